"""The reference's forced-deep topologies on the device
(forced_deep_scene, src/traversal_tests.rs:1521-1592; check_gpu with
expected errors 1 / 2, :2271-2283) and the rejection of its malformed BLAS
fixtures at upload (:1594-1636).

The device walks a 4-wide BVH collapsed from the binary one and keeps one
pending entry per three binary levels, so the reference's 64-deep chain does
not exhaust its stack: there the hits equal the oracle's and no overflow bit
is set.  A 200-deep chain exhausts the 32- and 64-entry stacks as well as the
oracle's 49-entry one: the overflow bits then agree with the oracle's, and the
ordered-scan fallback of both keeps every hit."""
import numpy as np
import pytest

import bevy_penumbra_b200 as bp
import oracle
from tests import fault_topologies as ft
from tests.helpers import EMPTY, check_against_f64, empty_device, from_device, packed, rays_for, scene_desc, to_device
from tests.test_gpu_cascades import compare_levels

pytestmark = pytest.mark.gpu


def assert_same_overflow(gpu_errors, oracle_errors):
    """Equal error bits, except that the device may add bit 1 (its BLAS walk
    ran out of the stack it shares with the TLAS walk) where bit 2 is set."""
    g, o = gpu_errors.astype(np.uint32), oracle_errors.astype(np.uint32)
    extra = g & ~o
    assert np.all((extra & ~np.uint32(1)) == 0), np.unique(g[extra != 0])
    assert np.all((g[extra != 0] & 2) == 2)
    np.testing.assert_array_equal(g & ~np.uint32(1), o & ~np.uint32(1))
    np.testing.assert_array_equal(o & ~g, 0)


def gpu_trace(pk, rays, any_hit=False):
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, pk)
    d_rays = to_device(rays)
    d_hits = empty_device(len(rays) * bp.HIT_DTYPE.itemsize)
    bp.trace_rays(ctx, scene, d_rays.data_ptr(), len(rays), d_hits.data_ptr(), any_hit=any_hit)
    ctx.synchronize()
    return from_device(d_hits, bp.HIT_DTYPE, (len(rays),))


@pytest.mark.parametrize("blas", [True, False])
@pytest.mark.parametrize("internals", [64, 200])
def test_forced_deep_traversal_matches_oracle(blas, internals):
    deep = ft.forced_deep(packed("traversal24"), blas, internals)
    rays = rays_for(scene_desc("traversal24"))
    gpu = gpu_trace(deep, rays)
    oscene = oracle.OracleScene.from_packed(deep)
    cpu, _ = oscene.trace_rays(rays)
    hit = cpu["triangle"] != EMPTY
    assert hit.sum() > 500
    np.testing.assert_array_equal(gpu["triangle"], cpu["triangle"])
    np.testing.assert_array_equal(gpu["instance"], cpu["instance"])
    np.testing.assert_array_equal(gpu["distance"][hit].view(np.uint32), cpu["distance"][hit].view(np.uint32))
    expected = 1 if blas else 2
    if internals == 64:
        assert np.all(gpu["errors"] == 0)
    else:
        # Both walks overflow: every hit carries the overflow bit of the deep
        # tree.  The device's TLAS and BLAS walks share one stack, so an
        # instance entered from a nearly full TLAS stack can also exhaust it
        # in its BLAS walk (bit 1 beside bit 2); the reference's BLAS walk has
        # a stack of its own.  Either fallback keeps every hit.
        assert_same_overflow(gpu["errors"], cpu["errors"])
        assert np.all((gpu["errors"][hit] & expected) == expected)
    # The TLAS chain may also raise the BLAS bit on the device (shared stack).
    failures, _ = check_against_f64(oscene, rays, gpu, any_hit=False, expected_errors=expected if blas else 3)
    assert not failures, failures[:12]
    blocked = gpu_trace(deep, rays, any_hit=True)
    cblocked, _ = oscene.trace_rays(rays, any_hit=True)
    np.testing.assert_array_equal(blocked["triangle"] != EMPTY, cblocked["triangle"] != EMPTY)
    np.testing.assert_array_equal(blocked["errors"] & 4, cblocked["errors"] & 4)


def scattered_receivers(n, seed):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform((-12.0, -9.0, -3.0), (12.0, 9.0, 3.0), size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    nrm = np.zeros_like(pos)
    nrm[:, :3] = d
    return pos, nrm


@pytest.mark.parametrize("blas", [True, False])
@pytest.mark.parametrize("stack_depth", [32, 64])
def test_forced_deep_split_frame_matches_oracle(blas, stack_depth):
    """A Split frame over the 200-deep topology with either stack: interval
    hits (with their overflow bits) bit-exact, records within tolerance."""
    deep = ft.forced_deep(packed("traversal24"), blas, 200)
    settings = bp.RadianceCascades(probe_spacing=0.5, interval_length=0.5, levels=4, rays_per_receiver=4,
                                   emissive_samples=4, frame_index=2).sanitized()
    pos, nrm = scattered_receivers(512, 21)
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, deep)
    rays = len(pos) * settings.rays_per_receiver
    view = bp.SplitView(ctx, max_receivers=len(pos), max_cells=1 << 14, max_entries=1 << 22, max_rays=rays)
    view.set_tuning(stack_depth=stack_depth, sort_queries=1)
    d_pos, d_nrm = to_device(pos), to_device(nrm)
    view.trace_merge(scene, settings, d_pos.data_ptr(), d_nrm.data_ptr(), len(pos))
    st = view.stats()
    assert st.error_flags == 0
    ofr = oracle.OracleFrame(oracle.OracleScene.from_packed(deep), settings.to_c(), pos, nrm)
    ost = ofr.stats()
    assert st.shadow_rays == ost.shadow_rays
    assert st.deposits == ost.deposits and st.unsupported == ost.unsupported
    got, want = view.read_hits(rays), ofr.hits(rays)
    np.testing.assert_array_equal(got["triangle"], want["triangle"])
    np.testing.assert_array_equal(got["instance"], want["instance"])
    assert_same_overflow(got["errors"], want["errors"])
    np.testing.assert_array_equal(got["distance"].view(np.uint32), want["distance"].view(np.uint32))
    hit = got["triangle"] != EMPTY
    assert hit.sum() > 100
    assert np.all((got["errors"][hit] & (1 if blas else 2)) == (1 if blas else 2))
    compare_levels(settings, [view.read_level(l) for l in range(settings.levels)], ofr, exact=False)


@pytest.mark.parametrize("make", [
    lambda p: ft.forced_cyclic_blas(p, 1),
    lambda p: ft.forced_oversized_leaf(p, 0),
    ft.two_child_self_loop,
    ft.shared_subtree,
], ids=["cyclic_blas", "oversized_leaf", "two_child_self_loop", "shared_subtree"])
def test_malformed_topologies_fail_upload(make):
    ctx = bp.LuxContext()
    with pytest.raises(bp.LuxError) as e:
        bp.GpuScene(ctx, make(packed("traversal24")))
    assert e.value.status == 5  # LUX_ERR_MALFORMED_SCENE
