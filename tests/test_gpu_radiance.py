"""lux_interval_radiance against the oracle's traceRayTracked +
outgoingTransportRadianceTracked restatement on identical rays."""
import ctypes as C

import numpy as np
import pytest

import bevy_penumbra_b200 as bp
import oracle
from tests.helpers import EMPTY, empty_device, from_device, packed, to_device

pytestmark = pytest.mark.gpu


def random_rays(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    rays = np.zeros(n, dtype=bp.RAY_DTYPE)
    rays["origin"] = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays["direction"] = d.astype(np.float32)
    rays["limit"] = 1e20
    return rays


def oracle_radiance(name, settings, rays):
    """name: a built-in scene name or a PackedScene."""
    osc = oracle.OracleScene.from_packed(packed(name) if isinstance(name, str) else name)
    s = settings.to_c()
    out = np.zeros((len(rays), 4), np.float32)
    hit = np.zeros(1, dtype=bp.HIT_DTYPE)
    rad = np.zeros(3, np.float32)
    for i in range(len(rays)):
        o = np.ascontiguousarray(rays["origin"][i])
        d = np.ascontiguousarray(rays["direction"][i])
        oracle.lib().orc_trace_closest(osc.handle, o.ctypes.data, d.ctypes.data, float(rays["tmin"][i]),
                                       float(rays["limit"][i]), hit.ctypes.data, None)
        ok = oracle.lib().orc_outgoing_radiance(osc.handle, C.byref(s), o.ctypes.data, d.ctypes.data, hit.ctypes.data,
                                                rad.ctypes.data, None, None)
        out[i] = (*rad, hit["distance"][0]) if ok else (0, 0, 0, -1)
    return out


@pytest.mark.parametrize("name,lo,hi,samples", [
    ("cornell", (-0.95, 0.05, -0.95), (0.95, 1.95, 0.95), 16),
    ("cornell", (-0.95, 0.05, -0.95), (0.95, 1.95, 0.95), 3),
    ("atrium65536", (-7, 0.2, -7), (7, 9.0, 7), 8),
])
def test_interval_radiance_bit_exact(name, lo, hi, samples):
    settings = bp.RadianceCascades(probe_spacing=0.25, emissive_samples=samples, frame_index=5).sanitized()
    rays = random_rays(4096, lo, hi, seed=samples)
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed(name))
    d_rays = to_device(rays)
    d_out = empty_device(len(rays) * 16)
    bp.interval_radiance(ctx, scene, settings, d_rays.data_ptr(), len(rays), d_out.data_ptr())
    ctx.synchronize()
    gpu = from_device(d_out, np.float32, (len(rays), 4))
    cpu = oracle_radiance(name, settings, rays)
    np.testing.assert_array_equal(gpu.view(np.uint32), cpu.view(np.uint32))
    assert np.mean(gpu[:, :3].sum(1) > 0) > 0.2, "many rays must see lit surfaces or emitters"


def lit_cornell():
    """The Cornell scene with a point, a spot and a directional light."""
    d = np.array([0.3, 1.0, 0.2])
    return packed("cornell").with_conventional_lights([
        bp.conventional_light((0.3, 1.5, 0.2), 5.0, (2.0, 2.0, 2.0)),
        bp.conventional_light((-0.5, 1.8, -0.5), 4.0, (1.0, 0.5, 0.2), direction=(0.0, -1.0, 0.0),
                              spot_scale=2.0, spot_offset=-1.0),
        bp.directional_light(d / np.linalg.norm(d), (0.5, 0.5, 0.5)),
    ])


@pytest.mark.parametrize("samples", [16, 2])
def test_interval_radiance_with_conventional_lights_bit_exact(samples):
    """conventionalLightResponseTracked: point, spot and directional lights
    with visibility rays, added after the emissive estimate."""
    settings = bp.RadianceCascades(probe_spacing=0.25, emissive_samples=samples, frame_index=3).sanitized()
    rays = random_rays(4096, (-0.95, 0.05, -0.95), (0.95, 1.95, 0.95), seed=11 + samples)
    scene_packed = lit_cornell()
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, scene_packed)
    d_rays = to_device(rays)
    d_out = empty_device(len(rays) * 16)
    bp.interval_radiance(ctx, scene, settings, d_rays.data_ptr(), len(rays), d_out.data_ptr())
    ctx.synchronize()
    gpu = from_device(d_out, np.float32, (len(rays), 4))
    osc = oracle.OracleScene.from_packed(scene_packed)
    s = settings.to_c()
    cpu = np.zeros_like(gpu)
    hit = np.zeros(1, dtype=bp.HIT_DTYPE)
    rad = np.zeros(3, np.float32)
    for i in range(len(rays)):
        o = np.ascontiguousarray(rays["origin"][i])
        dd = np.ascontiguousarray(rays["direction"][i])
        oracle.lib().orc_trace_closest(osc.handle, o.ctypes.data, dd.ctypes.data, 0.0, 1e20, hit.ctypes.data, None)
        ok = oracle.lib().orc_outgoing_radiance(osc.handle, C.byref(s), o.ctypes.data, dd.ctypes.data,
                                                hit.ctypes.data, rad.ctypes.data, None, None)
        cpu[i] = (*rad, hit["distance"][0]) if ok else (0, 0, 0, -1)
    np.testing.assert_array_equal(gpu.view(np.uint32), cpu.view(np.uint32))
    # The lights add light: brighter than the emitter-only scene on average.
    plain = oracle_radiance("cornell", settings, rays)
    assert gpu[:, :3].sum() > plain[:, :3].sum() * 1.05


@pytest.mark.parametrize("lights,samples", [(False, 8), (True, 8), (False, 2)])
def test_interval_radiance_with_environment_bit_exact(lights, samples):
    """environmentResponseTracked with a constant sky: max(1, samples / 2)
    cosine proposals per hit, each a visibility query to 1e20 through the
    Cornell box's open front, averaged and added after the emissive estimate
    (and before the conventional lights)."""
    settings = bp.RadianceCascades(probe_spacing=0.25, emissive_samples=samples, frame_index=7,
                                   environment=(4.0, 2.0, 1.0)).sanitized()
    rays = random_rays(4096, (-0.95, 0.05, -0.95), (0.95, 1.95, 0.95), seed=21 + samples)
    scene_packed = lit_cornell() if lights else packed("cornell")
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, scene_packed)
    d_rays = to_device(rays)
    d_out = empty_device(len(rays) * 16)
    bp.interval_radiance(ctx, scene, settings, d_rays.data_ptr(), len(rays), d_out.data_ptr())
    ctx.synchronize()
    gpu = from_device(d_out, np.float32, (len(rays), 4))
    cpu = oracle_radiance(scene_packed, settings, rays)
    np.testing.assert_array_equal(gpu.view(np.uint32), cpu.view(np.uint32))
    from dataclasses import replace
    dark = oracle_radiance(scene_packed, replace(settings, environment=(0.0, 0.0, 0.0)), rays)
    assert gpu[:, :3].sum() > dark[:, :3].sum() * 1.05  # sky light enters through the open front
    assert gpu[:, 0].sum() > gpu[:, 2].sum()  # with the sky's hue


def test_environment_next_event_slots_are_checked():
    """Emissive and environment samples share a hit's 16 next-event slots:
    32 emissive samples (16 per group) with a sky do not fit."""
    ctx = bp.LuxContext()
    scene = bp.GpuScene(ctx, packed("cornell"))
    rays = random_rays(32, (-0.5, 0.5, -0.5), (0.5, 1.5, 0.5), seed=1)
    d_rays = to_device(rays)
    d_out = empty_device(len(rays) * 16)
    ok = bp.RadianceCascades(probe_spacing=0.25, emissive_samples=16, environment=(1.0, 1.0, 1.0)).sanitized()
    bp.interval_radiance(ctx, scene, ok, d_rays.data_ptr(), len(rays), d_out.data_ptr())
    too_many = bp.RadianceCascades(probe_spacing=0.25, emissive_samples=32, environment=(1.0, 1.0, 1.0)).sanitized()
    with pytest.raises(bp.LuxError):
        bp.interval_radiance(ctx, scene, too_many, d_rays.data_ptr(), len(rays), d_out.data_ptr())
    ctx.synchronize()
