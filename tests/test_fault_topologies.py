"""Malformed and forced-deep BVH topologies on the host: the oracle against
the reference's stack-overflow expectations, and the upload's validation
(lux_scene_validate, the host half of lux_scene_upload) rejecting cycles,
shared subtrees and oversized leaves in bounded time."""
import time

import numpy as np
import pytest

import bevy_penumbra_b200 as bp
import oracle
from tests import fault_topologies as ft
from tests.helpers import EMPTY, check_against_f64, packed, rays_for, scene_desc

MALFORMED = 5  # LUX_ERR_MALFORMED_SCENE


def test_topologies_round_trip_the_words():
    """Words -> pack without changes reproduces the packer's streams."""
    p = packed("traversal24")
    q = ft.Words(p).pack()
    np.testing.assert_array_equal(q.scene_words, p.scene_words)


@pytest.mark.parametrize("blas", [True, False])
@pytest.mark.parametrize("internals", [64, 200])
def test_forced_deep_scenes_validate(blas, internals):
    status, message = bp.validate_scene(ft.forced_deep(packed("traversal24"), blas, internals))
    assert status == 0, message


@pytest.mark.parametrize("blas", [True, False])
def test_oracle_reports_stack_overflow_and_keeps_every_hit(blas):
    """check_gpu(.., forced_deep_scene(.., blas), expected 1 / 2)
    (src/traversal_tests.rs:2271-2283) against the oracle: every closest hit
    carries exactly the overflow bit (1: a BLAS stack, 2: the TLAS stack) and
    the f64 brute-force acceptance still holds."""
    expected = 1 if blas else 2
    deep = ft.forced_deep(packed("traversal24"), blas, 64)
    oscene = oracle.OracleScene.from_packed(deep)
    rays = rays_for(scene_desc("traversal24"))
    hits, _ = oscene.trace_rays(rays)
    hit = hits["triangle"] != EMPTY
    assert hit.sum() > 500
    assert np.all(hits["errors"][hit] == expected)
    assert np.all((hits["errors"] & ~np.uint32(expected)) == 0)
    failures, count = check_against_f64(oscene, rays, hits, any_hit=False, expected_errors=expected)
    assert not failures, failures[:12]
    # The same hits as the normal topology.
    plain, _ = oracle.OracleScene.from_packed(packed("traversal24")).trace_rays(rays)
    np.testing.assert_array_equal(hits["triangle"], plain["triangle"])
    np.testing.assert_array_equal(hits["instance"], plain["instance"])
    np.testing.assert_array_equal(hits["distance"][hit].view(np.uint32), plain["distance"][hit].view(np.uint32))
    blocked, _ = oscene.trace_rays(rays, any_hit=True)
    plain_blocked, _ = oracle.OracleScene.from_packed(packed("traversal24")).trace_rays(rays, any_hit=True)
    np.testing.assert_array_equal(blocked["triangle"] != EMPTY, plain_blocked["triangle"] != EMPTY)


@pytest.mark.parametrize("make", [
    lambda p: ft.forced_cyclic_blas(p, 1),
    lambda p: ft.forced_oversized_leaf(p, 0),
    ft.two_child_self_loop,
    ft.shared_subtree,
], ids=["cyclic_blas", "oversized_leaf", "two_child_self_loop", "shared_subtree"])
def test_malformed_topologies_are_rejected_quickly(make):
    bad = make(packed("traversal24"))
    t0 = time.perf_counter()
    status, message = bp.validate_scene(bad)
    elapsed = time.perf_counter() - t0
    assert status == MALFORMED, message
    assert elapsed < 0.5, elapsed
    assert message
