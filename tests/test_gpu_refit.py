"""lux_scene_refit on the device: the refit words equal the oracle's refit
bit for bit, and traversal / cascade frames on the refit scene match the
oracle on the same words."""
import numpy as np
import pytest

import bevy_penumbra_b200 as bp
import oracle
from tests.helpers import EMPTY, empty_device, from_device, packed, rays_for, scene_desc, to_device
from tests.refit_cases import atrium_select, move_instances, slot_transforms
from tests.test_refit import random_rays, same_hits

pytestmark = pytest.mark.gpu


def gpu_hits(ctx, scene, rays, any_hit=False):
    d_rays = to_device(rays)
    d_hits = empty_device(len(rays) * bp.HIT_DTYPE.itemsize)
    bp.trace_rays(ctx, scene, d_rays.data_ptr(), len(rays), d_hits.data_ptr(), any_hit=any_hit)
    return from_device(d_hits, bp.HIT_DTYPE, (len(rays),))


def refit_pair(name, seed):
    desc = scene_desc(name)
    p0 = packed(name)
    select = atrium_select(desc) if name.startswith("atrium") else None
    moved = move_instances(desc, seed=seed, select=select)
    m = slot_transforms(moved, p0)
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, p0)
    scene.refit(m)
    osc = oracle.OracleScene.from_packed(p0)
    osc.refit(m)
    return ctx, scene, osc, moved, p0


@pytest.mark.parametrize("name", ["traversal24", "atrium65536"])
def test_refit_words_match_oracle(name):
    ctx, scene, osc, _, _ = refit_pair(name, 21)
    np.testing.assert_array_equal(scene.read_words(), osc.words())


@pytest.mark.parametrize("name", ["traversal24", "atrium65536"])
def test_refit_traversal_matches_oracle(name):
    ctx, scene, osc, moved, p0 = refit_pair(name, 22)
    rays = rays_for(moved) if name == "traversal24" else random_rays(20000, (-7, 0.2, -7), (7, 9.5, 7), 6)
    gpu = gpu_hits(ctx, scene, rays)
    cpu, _ = osc.trace_rays(rays)
    assert same_hits(gpu, p0.instance_order, cpu, p0.instance_order) > 1000
    assert not np.any(gpu["errors"]) and not np.any(cpu["errors"])
    occ = gpu_hits(ctx, scene, rays, any_hit=True)
    ocpu, _ = osc.trace_rays(rays, any_hit=True)
    np.testing.assert_array_equal(occ["triangle"] != EMPTY, ocpu["triangle"] != EMPTY)


def test_refit_round_trip_restores_hits():
    name = "atrium65536"
    desc = scene_desc(name)
    p0 = packed(name)
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, p0)
    rays = random_rays(20000, (-7, 0.2, -7), (7, 9.5, 7), 7)
    before = gpu_hits(ctx, scene, rays)
    scene.refit(slot_transforms(move_instances(desc, 5, atrium_select(desc)), p0))
    moved = gpu_hits(ctx, scene, rays)
    assert np.any(moved["distance"] != before["distance"])
    scene.refit(slot_transforms(desc, p0))
    after = gpu_hits(ctx, scene, rays)
    same_hits(before, p0.instance_order, after, p0.instance_order)


def test_refit_rejects_bad_input():
    p0 = packed("traversal24")
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, p0)
    m = slot_transforms(scene_desc("traversal24"), p0)
    with pytest.raises(bp.LuxError):
        scene.refit(m[:-1])
    bad = m.copy()
    bad[2, :, :3] = 0.0
    with pytest.raises(bp.LuxError):
        scene.refit(bad)
    # A rejected refit leaves the scene usable at its previous pose.
    scene.refit(m)


def test_split_frame_after_refit_matches_oracle():
    settings = bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=8, interval_ratio=2.0,
                                   rays_per_receiver=4, emissive_samples=4, frame_index=2).sanitized()
    ctx, scene, osc, _, p0 = refit_pair("atrium65536", 23)
    rng = np.random.default_rng(10)
    n = 2048
    pos = np.zeros((n, 4), np.float32)
    pos[:, 0] = rng.uniform(-7, 7, n)
    pos[:, 2] = rng.uniform(-7, 7, n)
    nrm = np.zeros_like(pos)
    nrm[:, 1] = 1.0
    view = bp.SplitView(ctx, max_receivers=n, max_cells=1 << 16, max_entries=1 << 26,
                        max_rays=n * settings.rays_per_receiver)
    d_pos, d_nrm = to_device(pos), to_device(nrm)
    view.trace_merge(scene, settings, d_pos.data_ptr(), d_nrm.data_ptr(), n)
    assert view.stats().error_flags == 0
    ofr = oracle.OracleFrame(oracle.OracleScene(osc.words(), p0.geometry_words, p0.lights), settings.to_c(), pos, nrm)
    from tests.test_gpu_cascades import compare_levels
    compare_levels(settings, [view.read_level(l) for l in range(settings.levels)], ofr, exact=False)
