"""C-ABI boundary and host-side mirror (no GPU needed)."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

import bevy_penumbra_b200 as bp
from bevy_penumbra_b200 import _native as N
from bevy_penumbra_b200 import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "lux.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lux_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(N.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # ... and the Python binding declares a signature for each.
    assert set(names) <= set(N.SIGNATURES), sorted(set(names) - set(N.SIGNATURES))


def test_abi_version():
    assert N.lib().lux_abi_version() == 1


def test_record_layouts_match_the_header():
    assert C.sizeof(N.LuxRay) == 32
    assert C.sizeof(N.LuxHit) == 32
    assert C.sizeof(N.LuxLight) == 96
    assert bp.RAY_DTYPE.itemsize == 32 and bp.HIT_DTYPE.itemsize == 32


def test_context_creation_reports_missing_device_without_crashing():
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a device is present")
    handle = C.c_void_p()
    status = N.lib().lux_context_create(None, C.byref(handle))
    assert status == 6  # LUX_ERR_NO_DEVICE


# --- settings mirror: invalid_settings_are_bounded and the presets
# (src/lib.rs:949-1013) ---------------------------------------------------------
def test_invalid_settings_are_bounded():
    s = bp.RadianceCascades(probe_spacing=math.nan, emissive_samples=2**32 - 1, intensity=math.inf,
                            normal_bias=-1.0, levels=99, rays_per_receiver=0,
                            sampling=bp.SamplingSettings(resolve_scale=99)).sanitized()
    assert s.probe_spacing == np.float32(0.25)
    assert s.emissive_samples == 32
    assert s.intensity == 1.0
    assert s.normal_bias == np.float32(0.00001)
    assert 1 <= s.levels <= N.LUX_MAX_LEVELS
    assert s.rays_per_receiver == 1
    assert s.sampling.resolve_scale == 8
    h = bp.RadianceCascades(temporal_blend=math.inf, split_transmittance_blend=5.0, history_frames=1000).sanitized()
    assert h.temporal_blend == np.float32(0.88)        # non-finite: the default
    assert h.split_transmittance_blend == np.float32(0.999)
    assert h.history_frames == 64


def test_low_end_preset_fields():
    c = N.LuxSettings()
    N.lib().lux_settings_low_end(C.byref(c))
    assert c.probe_spacing == 1.0 and abs(c.interval_length - 1.6) < 1e-7
    assert c.emissive_samples == 4 and c.resolve_scale == 2
    d = N.LuxSettings()
    N.lib().lux_settings_default(C.byref(d))
    assert d.probe_spacing == np.float32(0.25) and d.emissive_samples == 16 and d.levels == 4
    assert (d.base_columns, d.base_rows) == (8, 4)  # 2*BASE_THETA x BASE_THETA
    assert d.temporal_blend == np.float32(0.88) and d.transmittance_blend == np.float32(0.98)
    assert d.history_frames == 24 and c.temporal_blend == np.float32(0.95)
    lo = bp.RadianceCascades.low_end()
    assert lo.sampling.grid_divisor == 8 and lo.sampling.max_receiver_cells == 16_384


def test_cache_entry_limit_accepts_262144_and_clamps_larger_values():
    assert bp.SamplingSettings(max_cache_entries=262_144).sanitized().max_cache_entries == 262_144
    assert bp.SamplingSettings(max_cache_entries=2**32 - 1).sanitized().max_cache_entries == 262_144


def test_interval_rules():
    ref = bp.RadianceCascades(interval_length=0.25, levels=4)
    # splitIntervalEnd: tuning.y * 4^L (shaders/split.slang:224-227)
    assert [ref.interval_end(l) for l in range(4)] == [0.25, 1.0, 4.0, 16.0]
    dbl = bp.RadianceCascades(interval_length=0.05, interval_ratio=2.0,
                              interval_rule=bp.INTERVAL_LENGTHS_GEOMETRIC, levels=4)
    ends = [dbl.interval_end(l) for l in range(4)]
    np.testing.assert_allclose(ends, [0.05, 0.15, 0.35, 0.75], rtol=1e-6)
    assert [ref.direction_count(l) for l in range(4)] == [32, 128, 512, 2048]
    c16 = bp.RadianceCascades(base_columns=4, base_rows=4)
    assert [c16.direction_count(l) for l in range(4)] == [16, 64, 256, 1024]


# --- scene packer: sah_build_is_bounded_at_world_workload_size
# (src/scene.rs:3620-3674) and the word layout (src/scene.rs:2096-2117) ----------
def test_sah_build_is_bounded_at_world_workload_size():
    i = np.arange(250_000)
    x = np.where(i >= 249_900, 1000.0 + (i - 249_900) * 0.01, (i % 500) * 0.01).astype(np.float32)
    y = ((i // 500) * 0.01).astype(np.float32)
    pos = np.zeros((750_000, 3), np.float32)
    pos[0::3, 0], pos[0::3, 1] = x, y
    pos[1::3, 0], pos[1::3, 1] = x + np.float32(0.003), y
    pos[2::3, 0], pos[2::3, 1] = x, y + np.float32(0.003)
    idx = np.arange(750_000, dtype=np.uint32).reshape(-1, 3)
    mat = scenes.material_words((0.5, 0.5, 0.5))
    p = bp.PackedScene.pack(pos, idx, [0], [250_000], [0], np.eye(3, 4, dtype=np.float32)[None], [0], [0], mat[None])
    assert p.max_depth <= 48
    assert p.blas_cost < 3.0, "SAH should isolate the tiny distant cluster"
    # Every triangle reachable exactly once from the BLAS leaves.
    sw = p.scene_words
    tlas = p.tlas_nodes
    counted = 0
    stack = [tlas]
    while stack:
        n = stack.pop()
        cnt = int(sw[2 + 2 * n][3])
        if cnt:
            counted += cnt
        else:
            first = int(sw[1 + 2 * n][3])
            stack += [first, first + 1]
    assert counted == 250_000


def test_packed_words_follow_the_reference_layout():
    p = bp.PackedScene.from_desc(scenes.cornell())
    sw, gw = p.scene_words, p.geometry_words
    material_end, base, count, stride = sw[0]
    assert stride == 9 and count == 8
    assert base == 1 + 2 * p.tlas_nodes + 2 * p.blas_nodes
    assert material_end == base + 9 * count + 8 * 4
    # geometry header {1, vertex base, 5, vertices}; vertex base multiple of 5
    assert gw[0][0] == 1 and gw[0][2] == 5 and gw[0][1] % 5 == 0
    # instance word 8: {TLAS count + BLAS root, first, count, 0}
    for i in range(count):
        w8 = sw[base + 9 * i + 8]
        assert w8[0] >= p.tlas_nodes and w8[3] == 0
    # one emissive quad -> two emitter records with a monotone CDF ending at 1
    cdf = p.lights.view(np.float32)[:, 11]
    assert len(cdf) == 2 and cdf[-1] == 1.0 and np.all(np.diff(cdf) > 0)
    area = p.lights.view(np.float32)[:, 7]
    np.testing.assert_allclose(area.sum(), 0.5, rtol=1e-5)


def test_scenes_have_the_stated_triangle_counts():
    assert scenes.cornell().world_triangles() == 34
    assert scenes.atrium(triangles=262_144).world_triangles() == 262_144
    assert scenes.atrium(triangles=65_536).world_triangles() == 65_536
