"""Conventional lights in the oracle's hit shading
(conventionalLightResponseTracked, shaders/cascades.slang:136-176)."""
import ctypes as C

import numpy as np

import bevy_penumbra_b200 as bp
import oracle
from tests.helpers import packed


def shade(scene_packed, origin, direction, settings):
    osc = oracle.OracleScene.from_packed(scene_packed)
    hit = np.zeros(1, dtype=bp.HIT_DTYPE)
    rad = np.zeros(3, np.float32)
    o = np.asarray(origin, np.float32)
    d = np.asarray(direction, np.float32)
    d = (d / np.linalg.norm(d)).astype(np.float32)
    oracle.lib().orc_trace_closest(osc.handle, o.ctypes.data, d.ctypes.data, 0.0, 1e20, hit.ctypes.data, None)
    s = settings.to_c()
    ok = oracle.lib().orc_outgoing_radiance(osc.handle, C.byref(s), o.ctypes.data, d.ctypes.data, hit.ctypes.data,
                                            rad.ctypes.data, None, None)
    assert ok
    return rad.copy()


def test_point_light_falloff_and_range():
    s = bp.RadianceCascades(probe_spacing=0.25, emissive_samples=2).sanitized()
    base = packed("cornell")
    ray = ((0.0, 1.0, 0.0), (0.0, -1.0, 0.0))  # hits the floor at the centre
    dark = shade(base, *ray, s)
    near = shade(base.with_conventional_lights([bp.conventional_light((0.0, 0.5, 0.0), 5.0, (1, 1, 1))]), *ray, s)
    far = shade(base.with_conventional_lights([bp.conventional_light((0.0, 1.0, 0.0), 5.0, (1, 1, 1))]), *ray, s)
    short = shade(base.with_conventional_lights([bp.conventional_light((0.0, 1.0, 0.0), 0.9, (1, 1, 1))]), *ray, s)
    assert np.all(near > dark) and np.all(far > dark)
    # Inverse square with the range fade: 4x closer distance squared, more light.
    assert np.all(near - dark > 3.0 * (far - dark))
    np.testing.assert_array_equal(short, dark)  # beyond the light's range


def test_spot_cone_and_occlusion():
    s = bp.RadianceCascades(probe_spacing=0.25, emissive_samples=2).sanitized()
    base = packed("cornell")
    ray = ((0.0, 1.0, 0.0), (0.0, -1.0, 0.0))
    dark = shade(base, *ray, s)
    down = bp.conventional_light((0.0, 1.5, 0.0), 5.0, (1, 1, 1), direction=(0.0, -1.0, 0.0), spot_scale=4.0,
                                 spot_offset=-3.0)
    away = bp.conventional_light((0.0, 1.5, 0.0), 5.0, (1, 1, 1), direction=(0.0, 1.0, 0.0), spot_scale=4.0,
                                 spot_offset=-3.0)
    assert np.all(shade(base.with_conventional_lights([down]), *ray, s) > dark)
    np.testing.assert_array_equal(shade(base.with_conventional_lights([away]), *ray, s), dark)
    # A light behind the back wall is occluded by it.
    outside = bp.conventional_light((0.0, 1.0, -5.0), 20.0, (50, 50, 50))
    np.testing.assert_array_equal(shade(base.with_conventional_lights([outside]), *ray, s), dark)
