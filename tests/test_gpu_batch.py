"""Batched frames (lux_batch_*): many scenes and views in one launch per
trace stage, captured as a CUDA graph.  Each view's results equal an
unbatched lux_view_trace_merge of the same view bit for bit on hit ids."""
import numpy as np
import pytest

import bevy_penumbra_b200 as bp
from bevy_penumbra_b200 import scenes
from tests.helpers import packed, to_device

pytestmark = pytest.mark.gpu

# History off: a batched and an unbatched frame of one view are compared
# frame by frame, so neither may blend the other's records.
SETTINGS = dict(probe_spacing=0.25, interval_length=0.4, levels=8, interval_ratio=2.0, rays_per_receiver=4,
                emissive_samples=4, history_frames=0)


def floor_receivers(n, seed, extent=2.4):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), np.float32)
    pos[:, 0] = rng.uniform(-extent, extent, n)
    pos[:, 2] = rng.uniform(-extent, extent, n)
    nrm = np.zeros_like(pos)
    nrm[:, 1] = 1.0
    return pos, nrm


def make_jobs(ctx):
    specs = [(scenes.batch_scene(31, 1000), 700), (scenes.batch_scene(32, 3001), 1500),
             (scenes.batch_scene(33, 24000), 333), (None, 2048), (scenes.batch_scene(34, 250), 0),
             (scenes.batch_scene(35, 90000), 1200)]
    jobs = []
    for k, (desc, n) in enumerate(specs):
        pk = packed("atrium65536") if desc is None else bp.PackedScene.from_desc(desc)
        scene = bp.GpuScene(ctx, pk)
        pos, nrm = floor_receivers(max(n, 1), 100 + k)
        d_pos, d_nrm = to_device(pos), to_device(nrm)
        view = bp.SplitView(ctx, max_receivers=max(n, 1), max_cells=1 << 15, max_entries=1 << 24,
                            max_rays=max(n, 1) * SETTINGS["rays_per_receiver"])
        jobs.append(dict(scene=scene, view=view, pos=d_pos, nrm=d_nrm, n=n))
    return jobs


def batch_args(jobs):
    return [(j["view"], j["scene"], j["pos"].data_ptr(), j["nrm"].data_ptr(), j["n"]) for j in jobs]


def snapshot(job, settings):
    view = job["view"]
    st = view.stats()
    rays = job["n"] * settings.rays_per_receiver
    hits = view.read_hits(rays) if rays else None
    levels = [view.read_level(l) for l in range(settings.levels)] if job["n"] else None
    return st, hits, levels


def assert_same(a, b, settings):
    (sa, ha, la), (sb, hb, lb) = a, b
    assert sa.error_flags == 0 and sb.error_flags == 0
    assert sa.interval_rays == sb.interval_rays
    assert sa.shadow_rays == sb.shadow_rays
    assert sa.deposits == sb.deposits and sa.unsupported == sb.unsupported
    assert sa.nodes_visited == sb.nodes_visited
    if ha is not None:
        np.testing.assert_array_equal(ha["triangle"], hb["triangle"])
        np.testing.assert_array_equal(ha["instance"], hb["instance"])
        np.testing.assert_array_equal(ha["errors"], hb["errors"])
        np.testing.assert_array_equal(ha["distance"].view(np.uint32), hb["distance"].view(np.uint32))
    if la is not None:
        for level in range(settings.levels):
            ka, ma, ra, ca = la[level]
            kb, mb, rb, cb = lb[level]
            # Dense cell ids follow atomic order: compare cells by key.
            assert len(ka) == len(kb)
            index = {tuple(k[:3]): i for i, k in enumerate(kb)}
            order = np.array([index[tuple(k[:3])] for k in ka], dtype=np.int64)
            mb, rb, cb = mb[order], rb[order], cb[order]
            np.testing.assert_array_equal(ca, cb)
            np.testing.assert_allclose(ra, rb, rtol=1e-4, atol=1e-6)
            np.testing.assert_allclose(ma, mb, rtol=1e-4, atol=1e-6)


@pytest.mark.parametrize("graph,sky,fused,tile", [(True, False, 0, 32), (False, False, 0, 64), (True, True, 0, 32),
                                                  (True, False, 1, 32), (False, True, 1, 128)])
def test_batch_matches_unbatched(graph, sky, fused, tile):
    """sky: a constant environment, whose next-event samples share the
    batched visibility pass with the emissive ones.  fused: the trace stage
    as one cooperative launch with grid barriers between its phases."""
    ctx = bp.LuxContext()
    jobs = make_jobs(ctx)
    batch = bp.Batch(ctx)
    batch.set_graph(graph)
    batch.set_tuning(16, 16, fused, tile)
    env = (1.0, 0.8, 0.6) if sky else (0.0, 0.0, 0.0)
    for frame in (1, 2):
        settings = bp.RadianceCascades(frame_index=frame, environment=env, **SETTINGS).sanitized()
        batch.trace_merge(batch_args(jobs), settings)
        got = [snapshot(j, settings) for j in jobs]
        for j, g in zip(jobs, got):
            j["view"].trace_merge(j["scene"], settings, j["pos"].data_ptr(), j["nrm"].data_ptr(), j["n"])
            assert_same(g, snapshot(j, settings), settings)
    info = batch.info()
    assert info.jobs == len(jobs)
    assert info.interval_rays == sum(j["n"] for j in jobs) * SETTINGS["rays_per_receiver"]
    if graph:
        assert info.graph_captures == 1 and info.graph_launches == 2
    else:
        assert info.graph_captures == 0
    batch.status()
    # Each pass runs once over all six jobs: setup, the sequence sort, the
    # trace stage (one launch fused, five not), corners, one merge per level
    # and the pack; the count does not grow with the job count.
    levels = SETTINGS["levels"]
    assert 10 + levels <= info.kernels_per_frame <= 2 * levels + (8 if fused else 12)


def test_batch_launches_do_not_grow_with_jobs():
    ctx = bp.LuxContext()
    jobs = make_jobs(ctx)
    batch = bp.Batch(ctx)
    batch.set_tuning(16, 16, 1)
    settings = bp.RadianceCascades(frame_index=1, **SETTINGS).sanitized()
    batch.trace_merge(batch_args(jobs[:2]), settings)
    two = batch.info().kernels_per_frame
    batch.trace_merge(batch_args(jobs), settings)
    assert batch.info().kernels_per_frame == two


def test_fused_trace_wait_runs_out_and_recovers():
    """A grid-barrier wait that cannot complete (one arrival short) gives up
    after its limit: lux_batch_status reports LUX_ERR_TIMEOUT, every job's
    view carries LUX_VIEW_ERR_TIMEOUT, and the next frame (wait restored)
    equals an unbatched frame."""
    ctx = bp.LuxContext()
    jobs = make_jobs(ctx)[:3]
    batch = bp.Batch(ctx)
    batch.set_tuning(16, 16, 1)
    batch.set_wait(50_000_000, missing_arrivals=1)
    settings = bp.RadianceCascades(frame_index=1, **SETTINGS).sanitized()
    batch.trace_merge(batch_args(jobs), settings)
    with pytest.raises(bp.LuxError) as err:
        batch.status()
    assert err.value.status == 7  # LUX_ERR_TIMEOUT
    for j in jobs:
        assert j["view"].stats().error_flags & 16
    batch.set_wait(1_000_000_000, 0)
    settings = bp.RadianceCascades(frame_index=2, **SETTINGS).sanitized()
    batch.trace_merge(batch_args(jobs), settings)
    batch.status()
    got = [snapshot(j, settings) for j in jobs]
    for j, g in zip(jobs, got):
        j["view"].trace_merge(j["scene"], settings, j["pos"].data_ptr(), j["nrm"].data_ptr(), j["n"])
        assert_same(g, snapshot(j, settings), settings)


@pytest.mark.parametrize("fused", [0, 1])
def test_batch_with_history_matches_unbatched(fused):
    """History on: each frame's records blend the view's previous frame
    (retain, history mapping, mass-weighted merge) in the batched passes as
    in unbatched frames of twin views, also across an invalidation box, and
    the graph is captured once."""
    ctx = bp.LuxContext()
    batched, single = make_jobs(ctx), make_jobs(ctx)
    batch = bp.Batch(ctx)
    batch.set_tuning(16, 16, fused)
    base = dict(SETTINGS, history_frames=24)
    for frame in (1, 2, 3, 4):
        if frame == 3:
            for j in batched + single:
                j["view"].invalidate_bounds((-1.0, -0.5, -1.0), (0.5, 1.0, 0.5))
        settings = bp.RadianceCascades(frame_index=frame, **base).sanitized()
        batch.trace_merge(batch_args(batched), settings)
        for j in single:
            j["view"].trace_merge(j["scene"], settings, j["pos"].data_ptr(), j["nrm"].data_ptr(), j["n"])
        for a, b in zip(batched, single):
            assert_same(snapshot(a, settings), snapshot(b, settings), settings)
    assert batch.info().graph_captures == 1


def test_batch_recaptures_on_new_configuration():
    ctx = bp.LuxContext()
    jobs = make_jobs(ctx)
    batch = bp.Batch(ctx)
    settings = bp.RadianceCascades(frame_index=1, **SETTINGS).sanitized()
    batch.trace_merge(batch_args(jobs), settings)
    batch.trace_merge(batch_args(jobs[:3]), settings)
    assert batch.info().graph_captures == 2
    got = snapshot(jobs[1], settings)
    jobs[1]["view"].trace_merge(jobs[1]["scene"], settings, jobs[1]["pos"].data_ptr(), jobs[1]["nrm"].data_ptr(),
                                jobs[1]["n"])
    assert_same(got, snapshot(jobs[1], settings), settings)


def test_batch_rejects_bad_jobs():
    ctx = bp.LuxContext()
    jobs = make_jobs(ctx)[:2]
    batch = bp.Batch(ctx)
    settings = bp.RadianceCascades(**SETTINGS).sanitized()
    args = batch_args(jobs)
    with pytest.raises(bp.LuxError):
        batch.trace_merge([args[0], args[0]], settings)  # a view twice
    with pytest.raises(bp.LuxError):
        batch.trace_merge([], settings)
    with pytest.raises(bp.LuxError):
        batch.trace_merge(args, bp.RadianceCascades(layout=bp.LAYOUT_DENSE, **SETTINGS).sanitized())
