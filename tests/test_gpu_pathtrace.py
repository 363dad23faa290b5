"""lux_path_reference (the path-traced FP64 reference) against its oracle
restatement: every sample is the same FP32 computation on both sides, so the
per-point FP64 means agree to summation order; plus the rectangle-light
quadrature on the device and agreement of the two-vertex estimate with the
one-bounce lux_reference_irradiance estimator."""
import numpy as np
import pytest

import bevy_penumbra_b200 as bp
import oracle
from bevy_penumbra_b200 import scenes
from tests.helpers import empty_device, from_device, packed, to_device
from tests.test_pathtrace import rectangle_irradiance, rectangle_scene

pytestmark = pytest.mark.gpu


def points(name, n, seed):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), np.float32)
    nrm = np.zeros((n, 4), np.float32)
    if name == "cornell":
        pos[:, 0] = rng.uniform(-0.9, 0.9, n)
        pos[:, 2] = rng.uniform(-0.9, 0.9, n)
        pos[:, 1] = 0.001
    else:
        pos[:, 0] = rng.uniform(-7.0, 7.0, n)
        pos[:, 2] = rng.uniform(-7.0, 7.0, n)
        pos[:, 1] = 0.001
    nrm[:, 1] = 1.0
    return pos, nrm


def gpu_path(pk, settings, pos, nrm, spp, bounces, seed):
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, pk)
    d_p, d_n = to_device(pos), to_device(nrm)
    d_o = empty_device(len(pos) * 32)
    bp.path_reference(ctx, scene, settings, d_p.data_ptr(), d_n.data_ptr(), len(pos), spp, bounces, seed,
                      d_o.data_ptr())
    return from_device(d_o, np.float64, (len(pos), 4))


@pytest.mark.parametrize("name,bounces", [("cornell", 1), ("cornell", 3), ("atrium65536", 3), ("atrium65536", 5)])
def test_path_reference_matches_oracle(name, bounces):
    settings = bp.RadianceCascades(emissive_samples=16).sanitized()
    pos, nrm = points(name, 96, 4)
    got = gpu_path(packed(name), settings, pos, nrm, 256, bounces, 17)
    want = oracle.OracleScene.from_packed(packed(name)).path_reference(settings.to_c(), pos, nrm, 256, bounces, 17)
    np.testing.assert_array_equal(got[:, 3], want[:, 3])
    np.testing.assert_allclose(got[:, :3], want[:, :3], rtol=1e-9, atol=1e-12)
    assert np.mean(got[:, :3].sum(1) > 0) > 0.5


def test_rectangle_light_quadrature_on_device():
    pk = bp.PackedScene.from_desc(rectangle_scene())
    settings = bp.RadianceCascades(normal_bias=1e-4).sanitized()
    pos = np.array([[0.0, 0.0, 0.0, 0.0]], np.float32)
    nrm = np.array([[0.0, 1.0, 0.0, 0.0]], np.float32)
    got = gpu_path(pk, settings, pos, nrm, 32768, 1, 0x4E45)
    np.testing.assert_allclose(got[0, :3], rectangle_irradiance(), rtol=0.015)


def test_two_vertex_paths_agree_with_the_one_bounce_estimator():
    """Two diffuse vertices (direct light at the receiver + one bounce) is the
    transport lux_reference_irradiance estimates with cosine rays alone."""
    pk = packed("cornell")
    settings = bp.RadianceCascades(emissive_samples=16).sanitized()
    pos, nrm = points("cornell", 32, 9)
    path = gpu_path(pk, settings, pos, nrm, 65536, 2, 3)
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, pk)
    d_p, d_n, d_o = to_device(pos), to_device(nrm), empty_device(len(pos) * 32)
    bp.reference_irradiance(ctx, scene, settings, d_p.data_ptr(), d_n.data_ptr(), len(pos), 262144, 3,
                            d_o.data_ptr())
    one = from_device(d_o, np.float64, (len(pos), 4))
    lit = one[:, :3].sum(1) > 1e-3  # points inside a box see no light at all
    assert lit.sum() >= 24
    np.testing.assert_array_equal(path[~lit, :3].sum(1) < 1e-3, True)
    # Both are Monte Carlo estimates (the cosine-ray one sees the small
    # emitter only by chance, a few per cent of noise per point).  The
    # cosine rays start normal_bias (5 mm) above the point, which raises the
    # direct light of the emitter 2 m above by about 0.5 per cent (the
    # next-event geometry is taken at the point itself), and the bounce term
    # differs by about one per cent more (measured with 2^21 cosine rays per
    # point on the oracle: -1.5 per cent in all, -1.1 with a 0.5 mm bias).
    rel = (path[lit, :3].sum(1) - one[lit, :3].sum(1)) / one[lit, :3].sum(1)
    assert -0.03 < rel.mean() < 0.005, rel
    assert np.median(np.abs(rel)) < 0.04 and np.abs(rel).max() < 0.15, rel


def test_direct_light_agrees_with_the_cosine_estimator():
    """Black walls leave the direct light alone: next-event estimation at
    the receiver (one diffuse vertex) and cosine rays that see the emitter
    estimate the same irradiance once the rays' origin offset is small."""
    desc = scenes.cornell()
    for words in desc.materials:
        f = words.view(np.float32)
        if f[4] == 0.0:
            f[0:3] = 0.0
    pk = bp.PackedScene.from_desc(desc)
    settings = bp.RadianceCascades(emissive_samples=16, normal_bias=0.0005).sanitized()
    pos, nrm = points("cornell", 32, 9)
    path = gpu_path(pk, settings, pos, nrm, 1 << 18, 1, 3)
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, pk)
    d_p, d_n, d_o = to_device(pos), to_device(nrm), empty_device(len(pos) * 32)
    bp.reference_irradiance(ctx, scene, settings, d_p.data_ptr(), d_n.data_ptr(), len(pos), 1 << 23, 3,
                            d_o.data_ptr())
    one = from_device(d_o, np.float64, (len(pos), 4))
    lit = one[:, :3].sum(1) > 1e-3
    assert lit.sum() >= 24
    # Points in deep penumbra (a few per cent of the emitter visible) keep
    # about a per cent of noise in either estimate; the mean bounds a bias.
    rel = (path[lit, :3].sum(1) - one[lit, :3].sum(1)) / one[lit, :3].sum(1)
    assert abs(rel.mean()) < 0.006 and np.abs(rel).max() < 0.05, rel
