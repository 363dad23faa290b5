"""GPU edge cases against the oracle: empty and ragged receiver sets (with
and without history, where an empty frame keeps the world cache by retain),
a multi-bounce frame whose receivers see nothing, and a screen whose extent
is not a multiple of the kernels' 16x16 tiles."""
import numpy as np
import pytest

import bevy_penumbra_b200 as bp
import oracle
from tests.helpers import packed, synthetic_screen, to_device, from_device, empty_device
from tests.test_gpu_cascades import compare_levels, cornell_floor_receivers

pytestmark = pytest.mark.gpu


def settings(frame, **kw):
    return bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=3,
                               frame_index=frame, **kw).sanitized()


def test_ragged_and_empty_frames_match_oracle():
    pos, nrm = cornell_floor_receivers(16)
    ragged = slice(0, 37)  # 111 interval rays: not a multiple of a warp
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed("cornell"))
    oscene = oracle.OracleScene.from_packed(packed("cornell"))
    view = bp.SplitView(ctx, max_receivers=len(pos), max_cells=1 << 14, max_entries=1 << 22, max_rays=len(pos) * 3)
    d_pos, d_nrm = to_device(pos[ragged]), to_device(nrm[ragged])
    s0 = settings(0)
    view.trace_merge(scene, s0, d_pos.data_ptr(), d_nrm.data_ptr(), 37)
    assert view.stats().error_flags == 0
    prev = oracle.OracleFrame(oscene, s0.to_c(), pos[ragged], nrm[ragged], max_cells=1 << 14, max_entries=1 << 22)
    compare_levels(s0, [view.read_level(l) for l in range(4)], prev, exact=False)
    # An empty frame with history: every cell is retained with its records.
    s1 = settings(1)
    view.trace_merge(scene, s1, d_pos.data_ptr(), d_nrm.data_ptr(), 0)
    st = view.stats()
    assert st.error_flags == 0 and st.interval_rays == 0
    empty = np.zeros((0, 4), np.float32)
    cur = oracle.OracleFrame(oscene, s1.to_c(), empty, empty, previous=prev, max_cells=1 << 14,
                             max_entries=1 << 22)
    compare_levels(s1, [view.read_level(l) for l in range(4)], cur, exact=False)
    assert st.cells[0] == prev.level(0, s0.direction_count(0))[0].shape[0]
    # Without history an empty frame holds nothing.
    s2 = settings(2, history_frames=0)
    view.trace_merge(scene, s2, d_pos.data_ptr(), d_nrm.data_ptr(), 0)
    assert all(view.stats().cells[l] == 0 for l in range(4))


@pytest.mark.parametrize("count", [1, 63, 64, 65])
def test_warp_boundary_receiver_counts_match_oracle(count):
    """Receiver counts at the warp boundaries of the ray, query and record
    lists (one ray per receiver: 1, 63, 64 and 65 interval rays), the analogue
    of the reference's compaction boundary counts
    (gpu_compact_direction_group_boundaries, src/transport_tests.rs:4109-4261):
    every frame's records and sample counts equal the oracle's."""
    pos, nrm = cornell_floor_receivers(16)
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed("cornell"))
    oscene = oracle.OracleScene.from_packed(packed("cornell"))
    s = bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=1,
                            frame_index=0).sanitized()
    view = bp.SplitView(ctx, max_receivers=count, max_cells=1 << 14, max_entries=1 << 22, max_rays=count)
    d_pos, d_nrm = to_device(pos[:count]), to_device(nrm[:count])
    view.trace_merge(scene, s, d_pos.data_ptr(), d_nrm.data_ptr(), count)
    st = view.stats()
    assert st.error_flags == 0 and st.interval_rays == count
    expected = oracle.OracleFrame(oscene, s.to_c(), pos[:count], nrm[:count], max_cells=1 << 14,
                                  max_entries=1 << 22)
    compare_levels(s, [view.read_level(l) for l in range(4)], expected, exact=False)


def test_multi_bounce_without_hits():
    """Receivers whose rays leave the scene record no surfaces: the secondary
    cache seeds nothing and the primary frame equals the plain one."""
    n = 64
    pos = np.zeros((n, 4), np.float32)
    pos[:, 0] = np.linspace(-50.0, -40.0, n, dtype=np.float32)  # far outside the Cornell box
    pos[:, 1] = 50.0
    pos[:, 3] = 1.0
    nrm = np.zeros_like(pos)
    nrm[:, 1] = 1.0  # facing away from the box
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed("cornell"))
    view = bp.SplitView(ctx, max_receivers=n, max_cells=1 << 12, max_entries=1 << 20, max_rays=n * 3)
    d_pos, d_nrm = to_device(pos), to_device(nrm)
    s = settings(0, multi_bounce=True)
    for frame in range(2):
        s.frame_index = frame
        view.trace_merge(scene, s, d_pos.data_ptr(), d_nrm.data_ptr(), n)
        sec = view.secondary()
        assert view.stats().error_flags == 0 and sec.stats().error_flags == 0
        assert sec.stats().interval_rays == 0 and sec.stats().cells[0] == 0


def test_screen_filter_ragged_extent():
    W, H = 77, 45
    s = bp.RadianceCascades(probe_spacing=0.25, normal_bias=0.005).sanitized()
    ctx = bp.LuxContext()
    screen = bp.ScreenFilter(ctx, W, H)
    out = empty_device(W * H * 16)
    history = None
    prev_clip = None
    for frame, eye in enumerate([(0.0, 1.2, 2.5), (0.02, 1.2, 2.5)]):
        irr, pos, nrm, ident, clip = synthetic_screen(W, H, eye, (0.0, 0.3, 0.0), seed=30 + frame)
        prev = clip if prev_clip is None else prev_clip
        d = [to_device(a) for a in (irr, pos, nrm, ident)]
        screen.filter(s, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), d[3].data_ptr(), prev, out.data_ptr(),
                      spatial_filter_steps=2)
        g_irr, g_meta = screen.read_history()
        history, o_out = oracle.screen_filter(s.to_c(), irr, pos, nrm, ident, prev, history=history,
                                              spatial_filter_steps=2)
        np.testing.assert_array_equal(g_irr.view(np.uint32), history[..., 0:4].view(np.uint32))
        np.testing.assert_array_equal(g_meta.view(np.uint32), history[..., 4:8].view(np.uint32))
        ctx.synchronize()
        np.testing.assert_allclose(from_device(out, np.float32, (H, W, 4)), o_out, rtol=1e-5, atol=1e-6)
        prev_clip = clip


def test_read_rate_probe_reports_l2_above_hbm_and_rejects_bad_sizes():
    ctx = bp.LuxContext()
    l2 = bp.measure_read_rate(ctx, 32 << 20, 64)
    hbm = bp.measure_read_rate(ctx, 1 << 30, 2)
    assert np.isfinite(l2) and np.isfinite(hbm) and hbm > 100.0
    assert l2 > hbm
    for nbytes, passes in ((1 << 10, 1), ((32 << 20) + 8, 1), (32 << 20, 0), (32 << 20, 5000)):
        with pytest.raises(bp.LuxError):
            bp.measure_read_rate(ctx, nbytes, passes)
