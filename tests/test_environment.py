"""Constant-environment next-event estimation in the oracle, pinned to the
reference's own regression (src/transport_tests.rs:1744-1880: an unoccluded
constant sky integrates to its radiance within 2.5% at 4096 samples; blocked
queries give supported black, denied queries unsupported black) and to the
cosineDirection frame of shaders/common.slang:407-412."""
import math

import numpy as np
import pytest

import oracle

SKY = (4.0, 2.0, 1.0)
ROUGHNESS = math.sqrt(0.4)


@pytest.mark.parametrize("position,sequence", [((0.0, 0.0, 0.0), 0), ((3.0, 2.0, 1.0), 1)])
def test_unoccluded_constant_sky_integrates_to_its_radiance(position, sequence):
    """checkEnvironment (src/transport_tests.rs:164-176) with tuning
    (1, sqrt(0.4), 0.001) and 4096 samples."""
    rgb, ok = oracle.environment_irradiance(SKY, position, (0.0, 1.0, 0.0), ROUGHNESS, 4096, sequence,
                                            probe_spacing=1.0, bias=0.001)
    assert ok
    for actual, expected in zip(rgb, SKY):
        assert abs(actual - expected) <= expected * 0.025, rgb


def test_blocked_and_denied_visibility():
    blocked, ok = oracle.environment_irradiance(SKY, (0, 0, 0), (0, 1, 0), ROUGHNESS, 32, 0, visibility=1)
    assert ok and np.all(blocked == 0.0)
    denied, ok = oracle.environment_irradiance(SKY, (0, 0, 0), (0, 1, 0), ROUGHNESS, 32, 0, visibility=2)
    assert not ok and np.all(denied == 0.0)


def test_black_environment_issues_no_queries():
    rgb, ok = oracle.environment_irradiance((0.0, 0.0, 0.0), (0, 0, 0), (0, 1, 0), ROUGHNESS, 32, 0, visibility=2)
    assert ok and np.all(rgb == 0.0)  # no query was made, so none could be denied


def test_estimate_is_linear_in_the_sky():
    a, _ = oracle.environment_irradiance(SKY, (0.3, 0.1, 0.7), (0, 1, 0), ROUGHNESS, 64, 9)
    b, _ = oracle.environment_irradiance(tuple(2.0 * c for c in SKY), (0.3, 0.1, 0.7), (0, 1, 0), ROUGHNESS, 64, 9)
    np.testing.assert_array_equal(b, 2.0 * a)  # power-of-two scaling is exact


def test_cosine_direction_frame():
    """results[24] of checkTransport: cosineDirection((0,1,0), (1,0)) is the
    unit tangent; every direction is unit length and above the normal."""
    t = oracle.cosine_direction_frame((0.0, 1.0, 0.0), 1.0, 0.0)
    assert abs(float(np.linalg.norm(t)) - 1.0) < 1e-6
    assert abs(float(t[1])) < 1e-6
    rng = np.random.default_rng(3)
    for _ in range(200):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        u1, u2 = rng.uniform(0.0, 1.0, 2)
        d = oracle.cosine_direction_frame(n, float(u1), float(u2))
        assert abs(float(np.linalg.norm(d)) - 1.0) < 1e-5
        assert float(np.dot(d, n)) >= -1e-6
        assert abs(float(np.dot(d, n)) - math.sqrt(1.0 - float(np.float32(u1)))) < 1e-5


def test_transport_random_is_open_unit_interval():
    vals = np.array([oracle.transport_random(s, lane) for s in range(0, 1 << 20, 4099) for lane in range(4)])
    assert np.all(vals > 0.0) and np.all(vals < 1.0)
    assert abs(vals.mean() - 0.5) < 0.02
