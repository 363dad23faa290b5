"""The FP64 reference irradiance (the error-report oracle) and the FP64
error reduction: the GPU reference equals its C restatement bit for bit, the
error reduction equals numpy, and the plain cascade's resolve lands near the
reference on the Cornell configuration."""
import ctypes as C

import numpy as np
import pytest

import bevy_penumbra_b200 as bp
from bevy_penumbra_b200 import _native as N
from bevy_penumbra_b200 import scenes
import oracle
from tests.helpers import cornell_dense_settings, empty_device, from_device, packed, to_device
from tests.test_gpu_cascades import cornell_floor_receivers

pytestmark = pytest.mark.gpu


def gpu_reference(ctx, scene, settings, pos, nrm, spp, seed):
    d_pos, d_nrm = to_device(pos), to_device(nrm)
    d_out = empty_device(len(pos) * 32)
    bp.reference_irradiance(ctx, scene, settings, d_pos.data_ptr(), d_nrm.data_ptr(), len(pos), spp, seed,
                            d_out.data_ptr())
    return from_device(d_out, np.float64, (len(pos), 4))


def test_reference_matches_oracle_bit_for_bit():
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed("cornell"))
    settings = bp.RadianceCascades(probe_spacing=0.25, emissive_samples=8).sanitized()
    pos, nrm = cornell_floor_receivers(8)
    gpu = gpu_reference(ctx, scene, settings, pos, nrm, 64, 5)
    rounds = N.lib().lux_reference_round_samples(len(pos), 64)
    cpu = oracle.OracleScene.from_packed(packed("cornell")).reference_irradiance(settings.to_c(), pos, nrm, 64, 5,
                                                                                 rounds)
    np.testing.assert_array_equal(gpu, cpu)
    assert np.all(gpu[:, 3] == 64) and np.mean(gpu[:, :3].sum(1) > 0) > 0.5  # floor points under the boxes see nothing


def test_error_stats_matches_numpy():
    ctx = bp.LuxContext()
    rng = np.random.default_rng(4)
    n = 5000
    est = rng.uniform(0, 2, size=(n, 4)).astype(np.float32)
    est[::7, 3] = 0.0  # unresolved points are skipped
    ref = rng.uniform(0, 2, size=(n, 4))
    ref[:, 3] = 16.0
    ref[::11, 3] = 0.0  # unsampled points are skipped
    d_est, d_ref = to_device(est), to_device(ref)
    got = bp.error_stats(ctx, d_est.data_ptr(), d_ref.data_ptr(), n)
    use = (est[:, 3] > 0) & (ref[:, 3] > 0)
    err = est[use, :3].astype(np.float64) - ref[use, :3]
    rmse = np.sqrt(np.mean(err ** 2))
    assert got["points"] == int(use.sum())
    np.testing.assert_allclose(got["rmse"], rmse, rtol=1e-12)
    np.testing.assert_allclose(got["mean_reference"], ref[use, :3].mean(), rtol=1e-12)
    np.testing.assert_allclose(got["max_abs_error"], np.abs(err).max(), rtol=0)


def test_dense_cornell_resolve_near_reference():
    """Config 1 (dense 64x64 probes, 4 levels, 16 directions x4): the resolved
    floor irradiance against 1024 spp of the FP64 reference.  The cascade's
    discretisation (direction bins, trilinear probes, octahedral tables)
    and one frame of next-event noise keep it from matching exactly; the
    bound pins the units and the scale."""
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed("cornell"))
    settings = cornell_dense_settings()
    pos, nrm = scenes.dense_plane_probes(64, 0.1, 10)
    view = bp.SplitView(ctx, max_receivers=len(pos), max_cells=1 << 16, max_entries=1 << 24, max_rays=1 << 20)
    d_pos, d_nrm = to_device(pos), to_device(nrm)
    view.trace_merge(scene, settings, d_pos.data_ptr(), d_nrm.data_ptr(), len(pos))
    # Resolve points on the probe plane (y = 1.05 m), facing up and down.
    rpos, rnrm = cornell_floor_receivers(24)
    rpos[:, 1] = 1.05
    rnrm[1::2, 1] = -1.0
    d_rp, d_rn = to_device(rpos), to_device(rnrm)
    d_est = empty_device(len(rpos) * 16)
    view.resolve(settings, d_rp.data_ptr(), d_rn.data_ptr(), len(rpos), d_est.data_ptr())
    ctx.synchronize()
    d_ref = empty_device(len(rpos) * 32)
    bp.reference_irradiance(ctx, scene, settings, d_rp.data_ptr(), d_rn.data_ptr(), len(rpos), 1024, 11,
                            d_ref.data_ptr())
    stats = bp.error_stats(ctx, d_est.data_ptr(), d_ref.data_ptr(), len(rpos))
    est = from_device(d_est, np.float32, (len(rpos), 4))
    ref = from_device(d_ref, np.float64, (len(rpos), 4))
    use = (est[:, 3] > 0) & (ref[:, 3] > 0)
    ratio = est[use, :3].sum() / ref[use, :3].sum()
    print("dense cornell resolve vs FP64 reference:", stats, "ratio", ratio)
    assert stats["points"] > 0.9 * len(rpos)
    assert 0.5 < ratio < 2.0
    assert stats["relative_rmse"] < 1.0
