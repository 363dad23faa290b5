"""GPU cascade frame parity: trace + deposit + merge + pack + resolve of
liblux against the CPU oracle on identical seeded inputs."""
import numpy as np
import pytest

import bevy_penumbra_b200 as bp
from bevy_penumbra_b200 import scenes
import oracle
from tests.helpers import cornell_dense_settings, empty_device, from_device, packed, to_device

pytestmark = pytest.mark.gpu

RTOL = 1e-4   # merged cascade radiance: relative tolerance
ATOL = 1e-6


def key_of(k):
    """(x, y, z, lod) of a cell key (w = level << 12 | lod << 18)."""
    return (int(k[0]), int(k[1]), int(k[2]), (int(k[3]) >> 18) & 31)


def by_key(keys):
    return {key_of(k): i for i, k in enumerate(keys)}


def run_frame(name, settings, pos, nrm, max_cells=1 << 16, max_entries=1 << 24, tuning=None):
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed(name))
    rays = len(pos) * settings.rays_per_receiver if settings.layout == bp.LAYOUT_SPLIT else 1 << 20
    view = bp.SplitView(ctx, max_receivers=len(pos), max_cells=max_cells, max_entries=max_entries, max_rays=rays)
    if tuning:
        view.set_tuning(**tuning)
    d_pos, d_nrm = to_device(pos), to_device(nrm)
    view.trace_merge(scene, settings, d_pos.data_ptr(), d_nrm.data_ptr(), len(pos))
    st = view.stats()
    assert st.error_flags == 0
    levels = [view.read_level(l) for l in range(settings.levels)]
    probes = view.read_probes()
    return ctx, scene, view, st, levels, probes


def oracle_frame(name, settings, pos, nrm):
    return oracle.OracleFrame(oracle.OracleScene.from_packed(packed(name)), settings.to_c(), pos, nrm)


def compare_levels(settings, gpu_levels, ofr, exact):
    for level in range(settings.levels):
        keys, merged, raw, samples = gpu_levels[level]
        okeys, omerged, oraw, osamples = ofr.level(level, settings.direction_count(level))
        assert len(keys) == len(okeys), f"level {level}: cell count"
        index = by_key(okeys)
        order = np.array([index[key_of(k)] for k in keys], dtype=np.int64)
        np.testing.assert_array_equal(samples, osamples[order], err_msg=f"level {level} samples")
        if exact:
            np.testing.assert_array_equal(raw.view(np.uint32), oraw[order].view(np.uint32))
            np.testing.assert_array_equal(merged.view(np.uint32), omerged[order].view(np.uint32))
        else:
            np.testing.assert_allclose(raw, oraw[order], rtol=RTOL, atol=ATOL, err_msg=f"level {level} raw")
            np.testing.assert_allclose(merged, omerged[order], rtol=RTOL, atol=ATOL, err_msg=f"level {level} merged")
    return order


def test_dense_cornell_frame_matches_oracle():
    settings = cornell_dense_settings()
    pos, nrm = scenes.dense_plane_probes(64, 0.1, 10)
    ctx, scene, view, st, levels, (pkeys, tables) = run_frame("cornell", settings, pos, nrm)
    assert st.interval_rays == 262_144
    assert [st.cells[l] for l in range(4)] == [4096, 1024, 256, 64]
    ofr = oracle_frame("cornell", settings, pos, nrm)
    ost = ofr.stats()
    assert st.shadow_rays == ost.shadow_rays
    assert st.deposits == ost.deposits
    compare_levels(settings, levels, ofr, exact=True)
    index = by_key(levels[0][0])
    otables = ofr.probes()
    okeys = ofr.level(0, 16)[0]
    order = np.array([by_key(pkeys)[key_of(k)] for k in okeys])
    np.testing.assert_allclose(tables[order], otables, rtol=RTOL, atol=ATOL)
    # Some probes see lit surfaces and some see the emitter.
    assert np.mean(levels[0][1][..., 3] > 0) > 0.2
    assert float(np.max(tables[..., :3])) > 0.0


def test_dense_cornell_resolve_matches_oracle():
    settings = cornell_dense_settings()
    pos, nrm = scenes.dense_plane_probes(64, 0.1, 10)
    ctx, scene, view, st, levels, probes = run_frame("cornell", settings, pos, nrm)
    rng = np.random.default_rng(3)
    n = 8192
    ppos = np.zeros((n, 4), np.float32)
    ppos[:, 0] = rng.uniform(-3.0, 3.0, n)
    ppos[:, 1] = rng.uniform(0.95, 1.15, n)
    ppos[:, 2] = rng.uniform(-3.0, 3.0, n)
    pn = rng.normal(size=(n, 3))
    pn /= np.linalg.norm(pn, axis=1, keepdims=True)
    pnrm = np.zeros((n, 4), np.float32)
    pnrm[:, :3] = pn
    d_p, d_n, d_o = to_device(ppos), to_device(pnrm), empty_device(n * 16)
    view.resolve(settings, d_p.data_ptr(), d_n.data_ptr(), n, d_o.data_ptr())
    ctx.synchronize()
    out = from_device(d_o, np.float32, (n, 4))
    expected = oracle_frame("cornell", settings, pos, nrm).resolve(ppos, pnrm)
    np.testing.assert_allclose(out, expected, rtol=RTOL, atol=ATOL)
    assert np.mean(out[:, 3] >= 1.0) > 0.5
    # frame_host gives the same irradiance from host buffers.
    host = view.frame_host(scene, settings, pos, nrm, ppos, pnrm)
    np.testing.assert_allclose(host, expected, rtol=RTOL, atol=ATOL)


def cornell_floor_receivers(n=32):
    k = (np.arange(n, dtype=np.float32) + np.float32(0.5)) / np.float32(n) * np.float32(1.9) - np.float32(0.95)
    x, z = np.meshgrid(k, k, indexing="ij")
    pos = np.zeros((n * n, 4), np.float32)
    pos[:, 0] = x.ravel()
    pos[:, 2] = z.ravel()
    nrm = np.zeros_like(pos)
    nrm[:, 1] = 1.0
    return pos, nrm


@pytest.mark.parametrize("rays,sort,depth,tile,mode", [(1, 0, 64, 32, 0), (8, 0, 64, 32, 0), (8, 1, 64, 32, 0),
                                                        (8, 1, 32, 32, 0), (8, 0, 64, 128, 0), (8, 1, 64, 256, 0),
                                                        (8, 0, 64, 32, 1), (8, 1, 64, 32, 1)])
def test_split_cornell_frame_matches_oracle(rays, sort, depth, tile, mode):
    """mode 1: the refill schedulers (a lane takes a new ray as soon as its
    walk ends) for both trace passes."""
    settings = bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=rays,
                                   frame_index=3).sanitized()
    pos, nrm = cornell_floor_receivers()
    ctx, scene, view, st, levels, (pkeys, tables) = run_frame("cornell", settings, pos, nrm,
                                                              tuning=dict(sort_rays=sort, sort_queries=sort,
                                                                          stack_depth=depth, tile_rays=tile,
                                                                          closest_mode=mode, shadow_mode=mode))
    ofr = oracle_frame("cornell", settings, pos, nrm)
    ost = ofr.stats()
    assert st.interval_rays == len(pos) * rays
    assert st.deposits == ost.deposits and st.shadow_rays == ost.shadow_rays
    compare_levels(settings, levels, ofr, exact=False)
    okeys = ofr.level(0, 32)[0]
    order = np.array([by_key(pkeys)[key_of(k)] for k in okeys])
    np.testing.assert_allclose(tables[order], ofr.probes(), rtol=RTOL, atol=ATOL)


def test_split_atrium_frame_matches_oracle():
    settings = bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=8, interval_ratio=2.0,
                                   rays_per_receiver=4, emissive_samples=4, frame_index=1).sanitized()
    rng = np.random.default_rng(9)
    n = 2048
    pos = np.zeros((n, 4), np.float32)
    pos[:, 0] = rng.uniform(-18, 18, n)
    pos[:, 2] = rng.uniform(-18, 18, n)
    pos[:, 1] = 0.0
    nrm = np.zeros_like(pos)
    nrm[:, 1] = 1.0
    ctx, scene, view, st, levels, probes = run_frame("atrium65536", settings, pos, nrm, max_entries=1 << 26,
                                                     tuning=dict(sort_rays=1, sort_queries=1))
    ofr = oracle_frame("atrium65536", settings, pos, nrm)
    compare_levels(settings, levels, ofr, exact=False)


def test_dense_cornell_history_matches_oracle():
    """Two frames on one view: the second blends the first's records
    (mergeEntry's history); dense records are bit-exact."""
    settings = cornell_dense_settings(frame_index=0)
    pos, nrm = scenes.dense_plane_probes(64, 0.1, 10)
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed("cornell"))
    view = bp.SplitView(ctx, max_receivers=len(pos), max_cells=1 << 16, max_entries=1 << 24, max_rays=1 << 20)
    d_pos, d_nrm = to_device(pos), to_device(nrm)
    view.trace_merge(scene, settings, d_pos.data_ptr(), d_nrm.data_ptr(), len(pos))
    second = cornell_dense_settings(frame_index=1)
    view.trace_merge(scene, second, d_pos.data_ptr(), d_nrm.data_ptr(), len(pos))
    levels = [view.read_level(l) for l in range(second.levels)]
    oscene = oracle.OracleScene.from_packed(packed("cornell"))
    first = oracle.OracleFrame(oscene, settings.to_c(), pos, nrm)
    ofr = oracle.OracleFrame(oscene, second.to_c(), pos, nrm, previous=first)
    compare_levels(second, levels, ofr, exact=True)
    # History changed something against a fresh second frame.
    fresh = oracle.OracleFrame(oscene, second.to_c(), pos, nrm)
    assert np.any(fresh.level(0, 16)[1] != ofr.level(0, 16)[1])


def test_split_history_and_invalidation_match_oracle():
    settings = bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=4,
                                   frame_index=0).sanitized()
    pos, nrm = cornell_floor_receivers()
    ctx, scene, view, st, levels, _ = run_frame("cornell", settings, pos, nrm)
    d_pos, d_nrm = to_device(pos), to_device(nrm)
    oscene = oracle.OracleScene.from_packed(packed("cornell"))
    prev = oracle.OracleFrame(oscene, settings.to_c(), pos, nrm)
    box = np.array([-0.3, -0.1, -0.3, 0.3, 0.5, 0.3], np.float32)
    for frame, dirty in ((1, None), (2, box)):
        s = bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=4,
                                frame_index=frame).sanitized()
        if dirty is not None:
            view.invalidate_bounds(dirty[:3], dirty[3:])
        view.trace_merge(scene, s, d_pos.data_ptr(), d_nrm.data_ptr(), len(pos))
        assert view.stats().error_flags == 0
        cur = oracle.OracleFrame(oscene, s.to_c(), pos, nrm, previous=prev,
                                 dirty=None if dirty is None else dirty[None])
        compare_levels(s, [view.read_level(l) for l in range(4)], cur, exact=False)
        prev = cur
    # reset_history: the next frame is fresh.
    view.reset_history()
    s = bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=4,
                            frame_index=3).sanitized()
    view.trace_merge(scene, s, d_pos.data_ptr(), d_nrm.data_ptr(), len(pos))
    compare_levels(s, [view.read_level(l) for l in range(4)], oracle.OracleFrame(oscene, s.to_c(), pos, nrm),
                   exact=False)


def test_split_retain_matches_oracle():
    """retain: receivers move between frames; cells of earlier frames stay in
    the persistent world cache (their records carried, their parents merged
    over them), and a tight max_cells keeps whole age classes youngest first."""
    def st(frame):
        return bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=4,
                                   frame_index=frame).sanitized()
    pos, nrm = cornell_floor_receivers()
    sets = [pos[:, 0] < 0, pos[:, 0] >= 0, np.abs(pos[:, 0]) < 0.2]
    oscene = oracle.OracleScene.from_packed(packed("cornell"))
    dirs = st(0).direction_count(0)
    every = {tuple(k[:3]) for k in oracle_frame("cornell", st(0), pos, nrm).level(0, dirs)[0]}
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed("cornell"))
    for max_cells in (1 << 16, len(every) - 1):
        view = bp.SplitView(ctx, max_receivers=len(pos), max_cells=max_cells, max_entries=1 << 24,
                            max_rays=len(pos) * 4)
        prev = None
        for frame, sel in enumerate(sets):
            s = st(frame)
            d_pos, d_nrm = to_device(pos[sel]), to_device(nrm[sel])
            view.trace_merge(scene, s, d_pos.data_ptr(), d_nrm.data_ptr(), int(sel.sum()))
            assert view.stats().error_flags == 0
            cur = oracle.OracleFrame(oscene, s.to_c(), pos[sel], nrm[sel], previous=prev, max_cells=max_cells,
                                     max_entries=1 << 24)
            compare_levels(s, [view.read_level(l) for l in range(4)], cur, exact=False)
            prev = cur
        if max_cells == 1 << 16:  # everything seen so far is still cached
            assert {tuple(k[:3]) for k in view.read_level(0)[0]} == every


@pytest.mark.parametrize("cached_sky", [False, True])
def test_multi_bounce_matches_oracle(cached_sky):
    """multi_bounce: each frame the primary cache traces with the previous
    secondary probes' bounce light and records one hit surface per receiver;
    the secondary cache (spacing and intervals x4) traces from those surfaces
    without first-hit emission.  Primary and secondary records follow the
    oracle chain frame by frame.  With cached_hit_sky (under a sky) the
    secondary's escapes carry the sky and covered hits skip their sky
    samples."""
    from dataclasses import replace

    def st(frame):
        return bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=4,
                                   emissive_samples=8, frame_index=frame, multi_bounce=True,
                                   environment=(1.5, 1.0, 0.5) if cached_sky else (0.0, 0.0, 0.0),
                                   cached_hit_sky=cached_sky).sanitized()
    pos, nrm = cornell_floor_receivers()
    pos[:, 3] = 1.0
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed("cornell"))
    oscene = oracle.OracleScene.from_packed(packed("cornell"))
    view = bp.SplitView(ctx, max_receivers=len(pos), max_cells=1 << 16, max_entries=1 << 24, max_rays=len(pos) * 4)
    assert view.secondary() is None
    d_pos, d_nrm = to_device(pos), to_device(nrm)
    prim = sec = None
    caps = dict(max_cells=1 << 16, max_entries=1 << 24)
    for frame in range(3):
        s = st(frame)
        s2 = replace(s, probe_spacing=s.probe_spacing * 4.0, interval_length=s.interval_length * 4.0,
                     multi_bounce=False, cached_hit_sky=False)
        view.trace_merge(scene, s, d_pos.data_ptr(), d_nrm.data_ptr(), len(pos))
        stats = view.stats()
        assert stats.error_flags == 0
        p = oracle.OracleFrame(oscene, s.to_c(), pos, nrm, previous=prim, feedback=sec, record_hits=True,
                               cached_sky=cached_sky, **caps)
        q = oracle.OracleFrame(oscene, s2.to_c(), p.hit_pos, p.hit_nrm, previous=sec, feedback=sec, sparse=True,
                               skip_emission=True, cached_sky=cached_sky, **caps)
        assert stats.shadow_rays == p.stats().shadow_rays
        compare_levels(s, [view.read_level(l) for l in range(4)], p, exact=False)
        secondary = view.secondary()
        assert secondary is not None and secondary.stats().error_flags == 0
        compare_levels(s2, [secondary.read_level(l) for l in range(4)], q, exact=False)
        if sec is not None:  # the bounce light reaches the primary records
            unfed = oracle.OracleFrame(oscene, s.to_c(), pos, nrm, previous=prim, **caps)
            dirs = s.direction_count(0)
            assert np.any(p.level(0, dirs)[2][..., :3] > unfed.level(0, dirs)[2][..., :3] + 1e-4)
        prim, sec = p, q


def test_split_lod_frames_and_resolve_match_oracle():
    """Distance LODs: a perspective camera close to the Cornell floor puts
    the receivers into LODs 0-2 (both variants seeded in overlaps, rays
    deposited into the selected one with 2^lod interval ends); two frames
    with history and retain, then the resolve's LOD blend, follow the oracle."""
    import math
    from tests.test_lod import perspective_infinite_reverse, view_from_world

    def st(frame):
        return bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=4,
                                   frame_index=frame).sanitized()
    pos, nrm = cornell_floor_receivers()
    eye = np.array([0.9, 0.4, 0.9])
    clip = (perspective_infinite_reverse(math.radians(60.0), 16 / 9, 0.1)
            @ view_from_world(eye, (0.0, 0.0, 0.0))).astype(np.float32)
    cam = bp.camera_struct(clip, eye, 32, 16)
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed("cornell"))
    oscene = oracle.OracleScene.from_packed(packed("cornell"))
    view = bp.SplitView(ctx, max_receivers=len(pos), max_cells=1 << 16, max_entries=1 << 24, max_rays=len(pos) * 4)
    view.set_camera(clip, eye, 32, 16)
    d_pos, d_nrm = to_device(pos), to_device(nrm)
    caps = dict(max_cells=1 << 16, max_entries=1 << 24)
    prev = None
    for frame in range(2):
        s = st(frame)
        view.trace_merge(scene, s, d_pos.data_ptr(), d_nrm.data_ptr(), len(pos))
        assert view.stats().error_flags == 0
        cur = oracle.OracleFrame(oscene, s.to_c(), pos, nrm, previous=prev, camera=cam, **caps)
        compare_levels(s, [view.read_level(l) for l in range(4)], cur, exact=False)
        prev = cur
    lods = {key_of(k)[3] for k in view.read_level(0)[0]}
    assert len(lods) >= 2, lods
    rng = np.random.default_rng(5)
    n = 4096
    ppos = np.zeros((n, 4), np.float32)
    ppos[:, 0] = rng.uniform(-0.95, 0.95, n)
    ppos[:, 2] = rng.uniform(-0.95, 0.95, n)
    pnrm = np.zeros((n, 4), np.float32)
    pnrm[:, 1] = 1.0
    d_p, d_n, d_o = to_device(ppos), to_device(pnrm), empty_device(n * 16)
    view.resolve(st(1), d_p.data_ptr(), d_n.data_ptr(), n, d_o.data_ptr())
    ctx.synchronize()
    out = from_device(d_o, np.float32, (n, 4))
    np.testing.assert_allclose(out, prev.resolve(ppos, pnrm), rtol=RTOL, atol=ATOL)
    blends = [oracle.lod_blend(st(1).to_c(), cam, p[:3])[2] for p in ppos[:512]]
    assert any(0.0 < b < 1.0 for b in blends)  # some points blend two LODs


def test_split_frame_with_conventional_lights_matches_oracle():
    from tests.test_gpu_radiance import lit_cornell
    settings = bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=4,
                                   emissive_samples=8, frame_index=2).sanitized()
    pos, nrm = cornell_floor_receivers()
    scene_packed = lit_cornell()
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, scene_packed)
    view = bp.SplitView(ctx, max_receivers=len(pos), max_cells=1 << 16, max_entries=1 << 24, max_rays=len(pos) * 4)
    d_pos, d_nrm = to_device(pos), to_device(nrm)
    view.trace_merge(scene, settings, d_pos.data_ptr(), d_nrm.data_ptr(), len(pos))
    st = view.stats()
    assert st.error_flags == 0
    ofr = oracle.OracleFrame(oracle.OracleScene.from_packed(scene_packed), settings.to_c(), pos, nrm)
    compare_levels(settings, [view.read_level(l) for l in range(4)], ofr, exact=False)
    assert st.shadow_rays == ofr.stats().shadow_rays


def test_split_frame_with_environment_matches_oracle():
    """A constant sky: every hit adds cosine-proposal environment samples
    (visibility to 1e20) after its emissive estimate; the frame's levels and
    shadow-ray count follow the oracle."""
    settings = bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=4,
                                   emissive_samples=8, frame_index=4, environment=(1.5, 1.0, 0.5)).sanitized()
    pos, nrm = cornell_floor_receivers()
    ctx, scene, view, st, levels, probes = run_frame("cornell", settings, pos, nrm)
    ofr = oracle_frame("cornell", settings, pos, nrm)
    compare_levels(settings, levels, ofr, exact=False)
    assert st.shadow_rays == ofr.stats().shadow_rays
    plain = bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=4,
                                emissive_samples=8, frame_index=4).sanitized()
    dark = oracle_frame("cornell", plain, pos, nrm)
    assert ofr.stats().shadow_rays > dark.stats().shadow_rays
