"""The learned-cache form of a Split frame (lux_view_set_cache): rays past
the cutoff answered by the cache, rotating validation with fallback, online
training inside the frame."""
import numpy as np
import pytest

import bevy_penumbra_b200 as bp
from tests.helpers import packed, to_device
from tests.test_gpu_batch import floor_receivers

pytestmark = pytest.mark.gpu

SETTINGS = dict(probe_spacing=0.25, interval_length=0.4, levels=8, interval_ratio=2.0, rays_per_receiver=8,
                emissive_samples=4)


def setup(n=4096):
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed("atrium65536"))
    pos, nrm = floor_receivers(n, 21, extent=6.0)
    rays = n * SETTINGS["rays_per_receiver"]
    view = bp.SplitView(ctx, max_receivers=n, max_cells=1 << 16, max_entries=1 << 25, max_rays=rays)
    return ctx, scene, view, to_device(pos), to_device(nrm), n


def test_cache_frames_run_and_train():
    ctx, scene, view, d_pos, d_nrm, n = setup()
    cache = bp.LearnedCache(ctx, batch=4096)
    cache.set_bounds((-8, -1, -8), (8, 11, 8))
    view.set_cache(cache, cutoff_level=2, validate_period=4, error_bound=4.0, train_samples=8192,
                   fallback_frames=4)
    for frame in range(24):
        settings = bp.RadianceCascades(frame_index=frame, **SETTINGS).sanitized()
        view.trace_merge(scene, settings, d_pos.data_ptr(), d_nrm.data_ptr(), n)
        st = view.stats()
        cs = view.cache_stats()
        assert st.error_flags == 0
        assert st.interval_rays == n * SETTINGS["rays_per_receiver"]
        assert cs.validated_rays > 0 and cs.trained_samples > 0
        assert cs.cached_rays + cs.fallback_rays <= st.interval_rays
    assert cache.stats().error_flags == 0
    assert cache.stats().steps == 24 * 2
    assert cs.cached_rays > 0.3 * st.interval_rays
    # Records exist at every level up to the cutoff and the cutoff level is
    # answered; no level past it is built (the cutoff level takes the tail).
    levels = [view.read_level(l) for l in range(3)]
    assert all(len(k) > 0 for k, _, _, _ in levels)
    assert levels[2][3].sum() > 0
    assert len(view.read_level(3)[0]) == 0


def test_cutoff_past_last_level_is_plain():
    """A cutoff at or beyond the last level leaves nothing to the cache: the
    frame equals the plain frame bit for bit on hit ids."""
    ctx, scene, view, d_pos, d_nrm, n = setup(1024)
    settings = bp.RadianceCascades(frame_index=5, **SETTINGS).sanitized()
    view.trace_merge(scene, settings, d_pos.data_ptr(), d_nrm.data_ptr(), n)
    plain = view.read_hits(n * SETTINGS["rays_per_receiver"])
    cache = bp.LearnedCache(ctx, batch=4096)
    view.set_cache(cache, cutoff_level=8)
    view.trace_merge(scene, settings, d_pos.data_ptr(), d_nrm.data_ptr(), n)
    hits = view.read_hits(n * SETTINGS["rays_per_receiver"])
    np.testing.assert_array_equal(plain["triangle"], hits["triangle"])
    np.testing.assert_array_equal(plain["distance"].view(np.uint32), hits["distance"].view(np.uint32))
    view.set_cache(None)


def test_set_cache_rejects_bad_modes():
    ctx, scene, view, d_pos, d_nrm, n = setup(256)
    cache = bp.LearnedCache(ctx, batch=4096)
    with pytest.raises(bp.LuxError):
        view.set_cache(cache, cutoff_level=0)
    with pytest.raises(bp.LuxError):
        view.set_cache(cache, validate_period=0)
    other = bp.LuxContext()
    foreign = bp.LearnedCache(other, batch=4096)
    with pytest.raises(bp.LuxError):
        view.set_cache(foreign)
