"""GPU traversal parity (lux_trace_rays vs the CPU oracle and the f64 brute
force), the port of gpu_traversal_matches_brute_force_through_motion_and_asset_edits
(src/traversal_tests.rs:2067-2331) and check_gpu_for_layers
(src/traversal_tests.rs:1432-1519)."""
import numpy as np
import pytest

import bevy_penumbra_b200 as bp
import oracle
from tests.helpers import (EMPTY, check_against_f64, empty_device, from_device, packed, rays_for, scene_desc,
                           to_device)

pytestmark = pytest.mark.gpu


def gpu_trace(name, rays, any_hit=False):
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed(name))
    d_rays = to_device(rays)
    d_hits = empty_device(len(rays) * bp.HIT_DTYPE.itemsize)
    bp.trace_rays(ctx, scene, d_rays.data_ptr(), len(rays), d_hits.data_ptr(), any_hit=any_hit)
    ctx.synchronize()
    return from_device(d_hits, bp.HIT_DTYPE, (len(rays),))


@pytest.mark.parametrize("name", ["cornell", "traversal24"])
def test_closest_hits_bit_exact_against_oracle(name):
    rays = rays_for(scene_desc(name))
    gpu = gpu_trace(name, rays)
    oscene = oracle.OracleScene.from_packed(packed(name))
    cpu, _ = oscene.trace_rays(rays)
    hit = cpu["triangle"] != EMPTY
    # Hit/miss flag, triangle and instance are bit-exact; so is the distance.
    np.testing.assert_array_equal(gpu["triangle"], cpu["triangle"])
    np.testing.assert_array_equal(gpu["instance"], cpu["instance"])
    np.testing.assert_array_equal(gpu["errors"], cpu["errors"])
    np.testing.assert_array_equal(gpu["distance"][hit].view(np.uint32), cpu["distance"][hit].view(np.uint32))
    np.testing.assert_allclose(gpu["barycentric"][hit], cpu["barycentric"][hit], rtol=0, atol=0)
    failures, count = check_against_f64(oscene, rays, gpu, any_hit=False)
    assert not failures, failures[:12]
    if name == "traversal24":
        assert count > 500, "fixture must exercise many actual hits"


@pytest.mark.parametrize("name", ["cornell", "traversal24"])
def test_any_hit_matches_oracle(name):
    rays = rays_for(scene_desc(name))
    gpu = gpu_trace(name, rays, any_hit=True)
    oscene = oracle.OracleScene.from_packed(packed(name))
    cpu, _ = oscene.trace_rays(rays, any_hit=True)
    np.testing.assert_array_equal(gpu["triangle"] != EMPTY, cpu["triangle"] != EMPTY)
    np.testing.assert_array_equal(gpu["errors"] & 4, cpu["errors"] & 4)
    blocked = int(np.sum(gpu["triangle"] != EMPTY))
    if name == "traversal24":
        assert blocked > 500


def test_atrium_random_rays_match_oracle():
    name = "atrium65536"
    rng = np.random.default_rng(11)
    n = 20000
    rays = np.zeros(n, dtype=bp.RAY_DTYPE)
    rays["origin"] = rng.uniform((-7, 0.2, -7), (7, 9.5, 7), size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays["direction"] = d.astype(np.float32)
    rays["limit"] = 1e20
    gpu = gpu_trace(name, rays)
    oscene = oracle.OracleScene.from_packed(packed(name))
    cpu, _ = oscene.trace_rays(rays)
    hit = cpu["triangle"] != EMPTY
    assert hit.mean() > 0.5
    np.testing.assert_array_equal(gpu["triangle"], cpu["triangle"])
    np.testing.assert_array_equal(gpu["instance"], cpu["instance"])
    np.testing.assert_array_equal(gpu["distance"][hit].view(np.uint32), cpu["distance"][hit].view(np.uint32))


def test_tmin_interval_hits_match_oracle():
    name = "cornell"
    rng = np.random.default_rng(5)
    n = 4096
    rays = np.zeros(n, dtype=bp.RAY_DTYPE)
    rays["origin"] = rng.uniform((-0.9, 0.1, -0.9), (0.9, 1.9, 0.9), size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays["direction"] = d.astype(np.float32)
    rays["tmin"] = rng.uniform(0.0, 1.0, size=n).astype(np.float32)
    rays["limit"] = rng.uniform(0.5, 3.0, size=n).astype(np.float32)
    gpu = gpu_trace(name, rays)
    cpu, _ = oracle.OracleScene.from_packed(packed(name)).trace_rays(rays)
    np.testing.assert_array_equal(gpu["triangle"], cpu["triangle"])
    hit = cpu["triangle"] != EMPTY
    np.testing.assert_array_equal(gpu["distance"][hit].view(np.uint32), cpu["distance"][hit].view(np.uint32))
