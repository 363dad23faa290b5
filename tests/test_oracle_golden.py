"""The CPU oracle pinned against the reference's own known-answer tests.

Each test cites the reference test it ports.  Expected values are the
reference's asserted numbers, or the reference test's own CPU reference
functions restated here (resolve tables, dense SDF march, f64 brute force).
"""
import ctypes as C
import math

import numpy as np
import pytest

import bevy_penumbra_b200 as bp
import oracle
from oracle import f32
from tests.helpers import EMPTY, check_against_f64, packed, rays_for, scene_desc

L = oracle.lib


_alive = []


def _p(a):
    """Address of a numpy array, kept alive for the duration of the session
    (ctypes receives a bare pointer)."""
    _alive.append(a)
    return a.ctypes.data


def settings(**kw):
    return bp.RadianceCascades(**kw).to_c()


# ---------------------------------------------------------------------------
# Deposit (gpu_split_deposit_stops_at_first_hit_and_leaves_far_intervals_unfilled,
# src/transport_tests.rs:3637-3829)
# ---------------------------------------------------------------------------
def test_deposit_stops_at_first_hit_and_leaves_far_intervals_unfilled():
    s = settings(probe_spacing=0.25, interval_length=0.25, levels=4)
    end1 = L().orc_interval_end(C.byref(s), 1)
    assert end1 == np.float32(1.0)
    out = np.full((4, 4), 9.0, np.float32)
    written = L().orc_deposit_levels(C.byref(s), end1, 1, 0, _p(f32(4, 2, 1)), _p(out))
    assert written == 2
    np.testing.assert_array_equal(out[0], [0, 0, 0, 1])
    np.testing.assert_array_equal(out[1], [4, 2, 1, 0])
    np.testing.assert_array_equal(out[2], [9, 9, 9, 9])
    np.testing.assert_array_equal(out[3], [9, 9, 9, 9])


def test_unsupported_query_deposits_nothing():
    # temporalCases results[14] (src/split_merge_tests.rs:84-88, 1333-1337).
    s = settings(levels=4)
    out = np.zeros((4, 4), np.float32)
    assert L().orc_deposit_levels(C.byref(s), 20000.0, 1, 1, _p(f32(4, 2, 1)), _p(out)) == 0


@pytest.mark.parametrize("distance,hit,radiance,expected", [
    (1e20, 0, (0, 0, 0), (0.0, 0.0, 0.0, 1.0)),      # escape: supported zero
    (20000.0, 1, (4, 2, 1), (4.0, 2.0, 1.0, 1.0)),  # the final interval owns distant hits
])
def test_terminal_interval_owns_the_tail(distance, hit, radiance, expected):
    # temporalCases results[11], [12] (src/split_merge_tests.rs:60-83, 1324-1333).
    s = settings(levels=4)
    out = np.zeros((4, 4), np.float32)
    written = L().orc_deposit_levels(C.byref(s), distance, hit, 0, _p(f32(*radiance)), _p(out))
    assert written == 4
    merged = np.zeros(4, np.float32)
    children = np.zeros(128, np.float32)
    L().orc_merge_entry(_p(out[3].copy()), 1, _p(f32(0, 0, 0)), _p(children), 0, _p(merged))
    np.testing.assert_array_equal(merged, expected)


# ---------------------------------------------------------------------------
# Merge / support (supportCases, src/split_merge_tests.rs:89-192, asserted at
# src/split_merge_tests.rs:1359-1386 with tolerance 2e-4)
# ---------------------------------------------------------------------------
def close(actual, expected, tol=2e-4):
    assert abs(float(actual) - float(expected)) < tol, (actual, expected)


def corners(x0, x1):
    """8 corner records: x=0 corners get x0, x=1 corners get x1."""
    c = np.zeros((8, 4), np.float32)
    for corner in range(8):
        c[corner] = x1 if corner & 1 else x0
    return c


def interpolate(fraction, corner_records):
    out = np.zeros(4, np.float32)
    L().orc_interpolate_children(_p(f32(*fraction)), _p(np.ascontiguousarray(corner_records, np.float32)), _p(out))
    return out


def merge(interval, fraction, children4x8):
    out = np.zeros(4, np.float32)
    L().orc_merge_entry(_p(f32(*interval)), 1, _p(f32(*fraction)),
                        _p(np.ascontiguousarray(children4x8, np.float32)), 1, _p(out))
    return out


def test_fractional_support_interpolation():
    # result[0]: corners x=0 (2, w 1), x=1 (10, w 0.25), fraction (0.5, 0, 0).
    r = interpolate((0.5, 0, 0), corners((2, 2, 2, 1), (10, 10, 10, 0.25)))
    close(r[0], 3.6)
    close(r[3], 0.625)


def test_merge_preserves_fractional_support():
    # result[1]: parent J = 2, beta = 0.5 over four such children.
    child = corners((2, 2, 2, 1), (10, 10, 10, 0.25))
    r = merge((2, 2, 2, 0.5), (0.5, 0, 0), np.stack([child] * 4))
    close(r[0], 3.125 / 0.8125)
    close(r[3], 0.8125)


def test_fully_supported_merge_reduces_to_eq7():
    # result[2]: J + beta * mean(I) -> (6, 1).
    child = np.tile(np.array([8, 8, 8, 1], np.float32), (8, 1))
    r = merge((2, 2, 2, 0.5), (0.5, 0, 0), np.stack([child] * 4))
    close(r[0], 6.0)
    close(r[3], 1.0)


def test_missing_children_keep_opaque_black_supported():
    # result[3]
    r = merge((0, 0, 0, 0), (0.5, 0, 0), np.zeros((4, 8, 4), np.float32))
    np.testing.assert_array_equal(r, [0, 0, 0, 1])


def test_one_partial_child_keeps_fractional_mass():
    # result[4]: only child 0 corner 0 = (8, 0.25); fraction 0.
    children = np.zeros((4, 8, 4), np.float32)
    children[0, 0] = (8, 8, 8, 0.25)
    r = merge((2, 2, 2, 0.5), (0, 0, 0), children)
    close(r[0], 2.25 / 0.53125)
    close(r[3], 0.53125)


def test_support_weighting_keeps_hues_apart():
    # result[7]
    c = np.zeros((8, 4), np.float32)
    c[0] = (1, 0, 0, 0.25)
    c[1] = (0, 0, 1, 1)
    r = interpolate((0.5, 0, 0), c)
    close(r[0], 0.2)
    close(r[2], 0.8)
    close(r[3], 0.625)


def test_partial_children_weight_parent_radiance():
    # result[8]
    children = np.tile(np.array([0, 0, 1, 0.25], np.float32), (4, 8, 1))
    r = merge((0.5, 0, 0, 0.5), (0, 0, 0), children)
    close(r[0], 0.8)
    close(r[2], 0.2)
    close(r[3], 0.625)


@pytest.mark.parametrize("fx", [2e-6, 0.5e-6])
def test_sub_epsilon_support_is_preserved(fx):
    # results[9], [10]: corners 1, 3, 5, 7 = (6, 3, 1, 1).
    c = np.zeros((8, 4), np.float32)
    for corner in (1, 3, 5, 7):
        c[corner] = (6, 3, 1, 1)
    r = interpolate((fx, 0.5, 0.5), c)
    assert abs(r[0] - 6.0) < 2e-4
    assert abs(r[3] - fx) < 2e-8


# ---------------------------------------------------------------------------
# Resolve (gpu_world_resolve_normalizes_sparse_support_and_isolates_lods,
# src/world_resolve_tests.rs:736-981; CPU references
# src/world_resolve_tests.rs:77-309), orthographic / LOD 0 cases.
# ---------------------------------------------------------------------------
def ref_bin_direction(i):
    x, y = i % 8, i // 8
    phi = np.float32((x + 0.5) * (2 * math.pi) / 8.0)
    vertical = np.float32((y + 0.5) * 0.5 - 1.0)
    r = np.float32(math.sqrt(max(1.0 - vertical * vertical, 0.0)))
    return np.array([r * math.cos(phi), vertical, r * math.sin(phi)], np.float64)


def ref_decode_oct(u, v):
    p = np.array([u * 2 - 1, v * 2 - 1])
    n = np.array([p[0], p[1], 1 - abs(p[0]) - abs(p[1])])
    fold = min(max(-n[2], 0.0), 1.0)
    n[0] += -fold if n[0] >= 0 else fold
    n[1] += -fold if n[1] >= 0 else fold
    return n / np.linalg.norm(n)


def ref_encode_oct(n):
    n = np.asarray(n, np.float64)
    n = n / np.linalg.norm(n)
    n = n / (abs(n[0]) + abs(n[1]) + abs(n[2]))
    p = np.array([n[0], n[1]])
    if n[2] < 0:
        p = np.array([1 - abs(p[1]), 1 - abs(p[0])]) * np.array([1 if p[0] >= 0 else -1, 1 if p[1] >= 0 else -1])
    return p * 0.5 + 0.5


def ref_wrap(px, py):
    if px < 0:
        px, py = -px - 1, 5 - py
    elif px >= 6:
        px, py = 11 - px, 5 - py
    if py < 0:
        px, py = 5 - px, -py - 1
    elif py >= 6:
        px, py = 5 - px, 11 - py
    return px, py


def ref_probe_table(radiance, directions, support, pattern=None):
    """reference_probe_table (src/world_resolve_tests.rs:77-128)."""
    pattern = np.ones(32) if pattern is None else pattern
    table = np.zeros((36, 4))
    for texel in range(36):
        n = ref_decode_oct((texel % 6) / 6 + 0.5 / 6, (texel // 6) / 6 + 0.5 / 6)
        rs = np.zeros(3)
        nominal = observed = 0.0
        for d in range(32):
            cos = max(float(n @ ref_bin_direction(d)), 0.0)
            nominal += cos
            if not directions & (1 << d):
                continue
            w = cos * min(max(support, 0.0), 1.0)
            observed += w
            rs += np.asarray(radiance) * pattern[d] * w
        if observed <= 0 or nominal <= 0:
            continue
        scale = nominal * (4.0 / 32.0) / observed
        table[texel, :3] = rs * scale
        table[texel, 3] = min(max(observed / nominal, 0.0), 1.0)
    return table


def ref_angular_lookup(table, normal):
    """reference_angular_lookup (src/world_resolve_tests.rs:130-160)."""
    g = ref_encode_oct(normal) * 6.0 - 0.5
    base = np.floor(g).astype(int)
    f = g - np.floor(g)
    s = np.zeros(3)
    obs = 0.0
    for corner in range(4):
        b = (corner & 1, corner >> 1)
        ax = (1 - f[0]) if b[0] == 0 else f[0]
        ay = (1 - f[1]) if b[1] == 0 else f[1]
        px, py = ref_wrap(base[0] + b[0], base[1] + b[1])
        sample = table[py * 6 + px]
        w = ax * ay * min(max(sample[3], 0.0), 1.0)
        s += sample[:3] * w
        obs += w
    return (np.zeros(3), 0.0) if obs <= 0 else (s / obs, min(max(obs, 0.0), 1.0))


def ref_diffuse_lod0(probes, position, normal):
    """reference_diffuse_at_lod + reference_split_diffuse_source at LOD 0
    (src/world_resolve_tests.rs:162-260), one source."""
    grid = np.asarray(position, np.float64) - 0.5
    base = np.floor(grid).astype(int)
    f = grid - np.floor(grid)
    s = np.zeros(3)
    obs = pot = 0.0
    for corner in range(8):
        b = (corner & 1, (corner >> 1) & 1, (corner >> 2) & 1)
        w = 1.0
        for k in range(3):
            w *= (1 - f[k]) if b[k] == 0 else f[k]
        if not w > 0:
            continue
        pot += w
        key = (base[0] + b[0], base[1] + b[1], base[2] + b[2])
        if key not in probes:
            continue
        irr, cov = ref_angular_lookup(ref_probe_table(*probes[key]), normal)
        if cov <= 0:
            continue
        s += irr * w * cov
        obs += w * cov
    if obs <= 0 or pot <= 0:
        return np.zeros(3), 0.0
    return s / obs, min(max(obs / pot, 0.0), 1.0)


def insert_probes(probes, position, radiance, directions, corner_mask, support=1.0):
    """insert_probes (src/world_resolve_tests.rs:433-478) at LOD 0, spacing 1."""
    grid = np.floor(np.asarray(position, np.float64) - 0.5).astype(int)
    for corner in range(8):
        if not corner_mask & (1 << corner):
            continue
        key = (grid[0] + (corner & 1), grid[1] + ((corner >> 1) & 1), grid[2] + ((corner >> 2) & 1))
        probes[key] = (tuple(radiance), directions, support)


def oracle_resolve(probes, positions, normals):
    keys = np.zeros((len(probes), 4), np.int32)
    tables = np.zeros((len(probes), 36, 4), np.float32)
    for i, (key, (radiance, directions, support)) in enumerate(probes.items()):
        keys[i, :3] = key
        merged = np.zeros((32, 4), np.float32)
        for d in range(32):
            if directions & (1 << d):
                merged[d] = (*radiance, support)
        table = np.zeros((36, 4), np.float32)
        L().orc_pack_table(_p(merged), 8, 4, _p(table))
        tables[i] = table
    pos = np.zeros((len(positions), 4), np.float32)
    pos[:, :3] = positions
    nrm = np.zeros((len(positions), 4), np.float32)
    nrm[:, :3] = normals
    out = np.zeros((len(positions), 4), np.float32)
    L().orc_resolve_tables(_p(keys), len(probes), _p(tables), 1.0, _p(pos), _p(nrm), len(positions), _p(out))
    return out


def rclose(actual, expected):
    assert abs(actual - expected) <= max(abs(expected), 1.0) * 2e-4, (actual, expected)


def test_resolve_normalizes_sparse_support():
    probes = {}
    insert_probes(probes, (0, 0, 0), (2, 2, 2), 0xFFFFFFFF, 0xFF)
    insert_probes(probes, (4, 0, 0), (2, 2, 2), 0xFFFFFFFF, 0x33)
    insert_probes(probes, (8, 0, 0), (2, 2, 2), (0x33 << 16) | (0x33 << 24), 0xFF)
    insert_probes(probes, (16, 0, 0), (0, 0, 0), 0xFFFFFFFF, 0xFF)
    positions = [(0, 0, 0), (4, 0, 0), (8, 0, 0), (16, 0, 0), (20, 0, 0)]
    out = oracle_resolve(probes, positions, [(0, 1, 0)] * 5)
    for actual, position in zip(out, positions):
        expected, coverage = ref_diffuse_lod0(probes, position, np.array([0.0, 1.0, 0.0]))
        for a, e in zip(actual[:3], expected):
            rclose(a, e)
        rclose(actual[3], 1.0 + 0.25 * coverage if coverage > 0 else -1.0)
    assert np.all(out[3, :3] == 0) and out[3, 3] > 1.0, "supported black remains supported"
    assert out[4, 3] == -1.0, "missing probes remain unsupported"


def test_resolve_partial_black_support():
    probes = {}
    insert_probes(probes, (0, 0, 0), (0, 0, 0), 0xFFFFFFFF, 0xFF, support=0.125)
    out = oracle_resolve(probes, [(0, 0, 0)], [(0, 1, 0)])[0]
    expected, coverage = ref_diffuse_lod0(probes, (0, 0, 0), np.array([0.0, 1.0, 0.0]))
    assert 0 < coverage < 1
    assert np.all(out[:3] == 0)
    rclose(out[3], 1.0 + 0.25 * coverage)


def test_resolve_angular_lookup_and_south_pole_seam():
    probes = {}
    insert_probes(probes, (0, 0, 0), (2, 1, 3), 0xA55AC33C, 0xFF)
    normals = [np.array([0, 1, 0.0]), np.array([0.3, 0.2, 0.9]), np.array([0.001, 0.001, -1.0]),
               np.array([-0.001, -0.001, -1.0])]
    normals = [n / np.linalg.norm(n) for n in normals]
    out = oracle_resolve(probes, [(0, 0, 0)] * 4, normals)
    table = ref_probe_table((2, 1, 3), 0xA55AC33C, 1.0)
    for actual, n in zip(out, normals):
        expected, coverage = ref_angular_lookup(table, n)
        assert coverage > 0
        for a, e in zip(actual[:3], expected):
            rclose(a, e)
        rclose(actual[3], 1.0 + 0.25 * coverage)
    assert np.all(np.abs(out[2, :3] - out[3, :3]) < 0.02), "octahedral south-pole seam must be continuous"


def test_resolve_zero_coverage_is_unsupported():
    probes = {}
    insert_probes(probes, (0, 0, 0), (100, 100, 100), 0, 0xFF)
    out = oracle_resolve(probes, [(0, 0, 0)], [(0, 1, 0)])[0]
    np.testing.assert_array_equal(out, [0, 0, 0, -1])


def test_pack_table_matches_reference_probe_table():
    rng = np.random.default_rng(4)
    for _ in range(8):
        directions = int(rng.integers(0, 1 << 32))
        radiance = rng.uniform(0, 5, 3)
        support = float(rng.uniform(0.05, 1.0))
        merged = np.zeros((32, 4), np.float32)
        for d in range(32):
            if directions & (1 << d):
                merged[d] = (*radiance, support)
        table = np.zeros((36, 4), np.float32)
        L().orc_pack_table(_p(merged), 8, 4, _p(table))
        expected = ref_probe_table(radiance, directions, support)
        np.testing.assert_allclose(table, expected, rtol=2e-4, atol=2e-5)


# ---------------------------------------------------------------------------
# Dense 16^3 SDF cascade reference (src/transport_tests.rs:179-248, 3830-4107)
# ---------------------------------------------------------------------------
def dense_box(p, c, h):
    q = np.abs(p - c) - h
    return np.sqrt(np.sum(np.maximum(q, 0) ** 2, axis=-1)) + np.minimum(np.max(q, axis=-1), 0)


def dense_scene(p):
    d = dense_box(p, np.array([-3.0, 0, 0]), np.array([0.9, 0.9, 0.9]))
    m = np.ones(d.shape, np.int32)
    sphere = np.linalg.norm(p - np.array([3.0, 1.0, 0.0]), axis=-1) - 1.0
    for dist, mat in ((sphere, 2), (dense_box(p, np.array([0.0, 3, 0]), np.array([2.0, 0.04, 2])), 3),
                      (dense_box(p, np.array([0.0, 0, 4]), np.array([2.0, 0.5, 0.03])), 4)):
        better = dist < d
        d = np.where(better, dist, d)
        m = np.where(better, mat, m)
    return d, m


def dense_reference(level):
    theta = 4 << level
    dim = 16 >> level
    dirs = 32 << (2 * level)
    idx = np.arange(dirs)
    u = ((idx % (2 * theta)) + 0.5) / (2 * theta)
    v = ((idx // (2 * theta)) + 0.5) / theta
    phi = u * 2 * math.pi
    y = v * 2 - 1
    r = np.sqrt(np.maximum(1 - y * y, 0))
    direction = np.stack([r * np.cos(phi), y, r * np.sin(phi)], -1)
    cells = np.stack(np.meshgrid(np.arange(dim), np.arange(dim), np.arange(dim), indexing="ij"), -1)
    cells = cells.transpose(2, 1, 0, 3).reshape(-1, 3)  # probe = x + y*dim + z*dim^2
    origin = -8.0 + (cells + 0.5) * (1 << level)
    o = np.repeat(origin, dirs, axis=0)
    d = np.tile(direction, (len(origin), 1))
    near = float((1 << level) - 1)
    far = float((1 << (level + 1)) - 1)
    t = np.full(len(o), near + 0.001)
    interval = np.tile(np.array([0, 0, 0, 1.0]), (len(o), 1))
    active = np.ones(len(o), bool)
    for _ in range(96):
        active &= t <= far
        if not active.any():
            break
        dist, mat = dense_scene(o + d * t[:, None])
        hit = active & (dist < 0.001)
        interval[hit] = np.where((mat[hit] == 3)[:, None], [6.0, 2.0, 0.5, 0.0], [0, 0, 0, 0.0])
        active &= ~hit
        t = np.where(active, t + np.maximum(dist, 0.005), t)
    return interval, d, idx


def test_dense_sdf_cascade_intervals_match_f64_reference():
    offset = 0
    hits_by_material = set()
    for level in range(4):
        interval, direction, idx = dense_reference(level)
        n = len(interval)
        got_i = np.zeros((n, 4), np.float32)
        got_d = np.zeros((n, 4), np.float32)
        for k in range(n):
            a = np.zeros(4, np.float32)
            b = np.zeros(4, np.float32)
            L().orc_dense_sdf_record(offset + k, _p(a), _p(b))
            got_i[k] = a
            got_d[k] = b
        mismatch = got_i[:, 3] != interval[:, 3]
        # The f32 march and the f64 march may disagree only where a ray grazes
        # a surface within the marcher's 0.001 hit threshold.
        assert mismatch.mean() < 2e-3, (level, mismatch.sum())
        ok = ~mismatch
        assert np.all(np.abs(got_i[ok, :3] - interval[ok, :3]) < 1e-4)
        np.testing.assert_array_equal(got_d[:, 3], np.tile(idx, n // len(idx)).astype(np.float32))
        assert np.all(np.abs(got_d[:, :3] - direction) < 1e-5)
        hits_by_material.update(np.unique(interval[:, 3]).tolist())
        offset += n
    assert offset == 245_760
    assert 0.0 in hits_by_material and 1.0 in hits_by_material


@pytest.mark.parametrize("columns,rows", [(8, 4), (4, 4), (16, 8)])
def test_direction_index_round_trips_bin_direction(columns, rows):
    for level in range(4):
        cols, rws = columns << level, rows << level
        for index in range(cols * rws):
            u = np.float32((np.float32(index % cols) + np.float32(0.5)) / np.float32(cols))
            v = np.float32((np.float32(index // cols) + np.float32(0.5)) / np.float32(rws))
            assert L().orc_direction_index_uv(u, v, cols, rws) == index
        # poles and the azimuth seam stay inside the grid
        for u, v in ((0.0, 1.0), (0.0, 0.0), (0.9999999, 0.5), (1.0, 1.0)):
            assert L().orc_direction_index_uv(u, v, cols, rws) < cols * rws


def test_sincos_turns_accuracy():
    turns = np.linspace(-1.0, 2.0, 30001, dtype=np.float32)
    c = np.zeros(1, np.float32)
    s = np.zeros(1, np.float32)
    worst = 0.0
    for t in turns[::7]:
        L().orc_sincos_turns(float(t), _p(c), _p(s))
        worst = max(worst, abs(float(c[0]) - math.cos(2 * math.pi * float(t))),
                    abs(float(s[0]) - math.sin(2 * math.pi * float(t))))
    assert worst < 5e-7


def test_r2_and_hashes_are_the_reference_integers():
    out = np.zeros(2, np.float32)
    for index in (0, 1, 7, 123456, 0xFFFFFFFF):
        L().orc_r2(index, _p(out))
        px = (index * 3242174889) & 0xFFFFFFFF
        py = (index * 2447445414) & 0xFFFFFFFF
        assert out[0] == np.float32((px >> 8) / 16777216.0)
        assert out[1] == np.float32((py >> 8) / 16777216.0)

    def transport_hash(v):
        v ^= v >> 16
        v = (v * 0x7FEB352D) & 0xFFFFFFFF
        v ^= v >> 15
        v = (v * 0x846CA68B) & 0xFFFFFFFF
        v ^= v >> 16
        return v

    for v in (0, 1, 0x5A17C9E3, 0xDEADBEEF):
        assert L().orc_transport_hash(v) == transport_hash(v)
    key = np.array([3, -2, 7, 1 << 12], np.int32)
    k = key.view(np.uint32).astype(np.uint64)
    h = int((k[0] * 0x8DA6B343) ^ (k[1] * 0xD8163841) ^ (k[2] * 0xCB1AB31F) ^ (k[3] * 0x165667B1)) & 0xFFFFFFFF
    h ^= h >> 16
    h = (h * 0x7FEB352D) & 0xFFFFFFFF
    h ^= h >> 15
    assert L().orc_hash_key(_p(key), 1 << 20) == (h & ((1 << 20) - 1))


def test_ray_offset_moves_along_the_normal():
    out = np.zeros(3, np.float32)
    for p, n in (((1.0, 2.0, 3.0), (0, 1, 0)), ((0.01, -0.02, 5.0), (0, 0, -1)), ((-4.0, 0.0, 1e6), (1, 0, 0))):
        L().orc_ray_offset(_p(f32(*p)), _p(f32(*n)), 0.005, _p(out))
        delta = out.astype(np.float64) - np.array(p, np.float64)
        assert np.dot(delta, n) > 0
        assert np.all(np.isfinite(out))


# ---------------------------------------------------------------------------
# Traversal (check_gpu_for_layers acceptance, src/traversal_tests.rs:1432-1519,
# on the rays_for families, src/traversal_tests.rs:1040-1125)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", ["cornell", "traversal24"])
def test_oracle_traversal_accepts_against_f64_brute_force(name):
    rays = rays_for(scene_desc(name))
    oscene = oracle.OracleScene.from_packed(packed(name))
    closest, _ = oscene.trace_rays(rays)
    failures, count = check_against_f64(oscene, rays, closest, any_hit=False)
    assert not failures, failures[:12]
    shadow, _ = oscene.trace_rays(rays, any_hit=True)
    sfail, scount = check_against_f64(oscene, rays, shadow, any_hit=True)
    assert not sfail, sfail[:12]
    if name == "traversal24":
        assert count > 500 and scount > 500, "fixture must exercise many actual hits"


def test_oracle_bvh_walk_equals_brute_force_f32():
    rays = rays_for(scene_desc("traversal24"))
    oscene = oracle.OracleScene.from_packed(packed("traversal24"))
    hits, _ = oscene.trace_rays(rays)
    brute = np.zeros(1, dtype=bp.HIT_DTYPE)
    for i in range(0, len(rays), 5):
        o = np.ascontiguousarray(rays["origin"][i])
        d = np.ascontiguousarray(rays["direction"][i])
        L().orc_brute_closest(oscene.handle, _p(o), _p(d), 0.0, float(rays["limit"][i]), _p(brute))
        assert brute["triangle"][0] == hits["triangle"][i]
        assert brute["instance"][0] == hits["instance"][i]
        if hits["triangle"][i] != EMPTY:
            assert brute["distance"][0] == hits["distance"][i]
