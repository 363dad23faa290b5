"""World history (mergeEntry's bounded interval history,
shaders/split.slang:1478-1521, :1624-1725) in the oracle: the temporal cases
of gpu_split_merge_bounds_history_and_preserves_fractional_support
(src/split_merge_tests.rs:36-70, asserted at :1306-1360, tolerance 2e-4),
and history across oracle frames."""
import numpy as np
import pytest

import bevy_penumbra_b200 as bp
import oracle
from tests.helpers import packed

TOL = 2e-4


def settings(radiance_blend, beta_blend):
    s = bp.RadianceCascades(temporal_blend=radiance_blend, split_transmittance_blend=beta_blend,
                            history_frames=30).to_c()
    return s


class Record:
    """One cache entry advanced frame by frame (the KAT's advance())."""

    def __init__(self, st):
        self.st = st
        self.raw = np.zeros(4, np.float32)
        self.mass = np.zeros(2, np.float32)

    def advance(self, radiance, beta, count):
        self.raw, self.mass = oracle.history_blend(self.st, count, (radiance, radiance, radiance, beta),
                                                   self.raw, self.mass)


@pytest.mark.parametrize("j,beta", [(0.5, 0.75), (0.9, 0.95)])
def test_temporal_cases(j, beta):
    r = Record(settings(j, beta))
    for _ in range(512):
        r.advance(2.0, 0.0, 1)
    # Masses saturate at 1 / (1 - blend).
    assert abs(r.mass[0] - 1.0 / (1.0 - j)) < TOL
    assert abs(r.mass[1] - 1.0 / (1.0 - beta)) < TOL
    r.advance(0.0, 1.0, 1)
    assert abs(r.raw[0] - 2.0 * j) < TOL
    assert abs(r.raw[3] - (1.0 - beta)) < TOL
    raw2, mass2 = r.raw.copy(), r.mass.copy()
    for _ in range(200):
        r.advance(0.0, 1.0, 0)
    # Zero observations must not decay world state, mass or support.
    np.testing.assert_array_equal(r.raw, raw2)
    np.testing.assert_array_equal(r.mass, mass2)
    # Batched observations consume retention per observation.
    for _ in range(512):
        r.advance(2.0, 0.0, 1)
    r.advance(0.0, 1.0, 4)
    assert abs(r.raw[0] - 2.0 * j ** 4) < TOL
    assert abs(r.raw[3] - (1.0 - beta ** 4)) < TOL
    assert abs(r.mass[0] - 1.0 / (1.0 - j)) < TOL
    assert abs(r.mass[1] - 1.0 / (1.0 - beta)) < TOL


def test_beta_only_and_radiance_only_history():
    r = Record(settings(0.0, 0.9))
    for _ in range(512):
        r.advance(2.0, 0.0, 1)
    r.advance(0.0, 1.0, 1)
    assert abs(r.raw[0] - 0.0) < TOL and abs(r.raw[3] - 0.1) < TOL
    for _ in range(200):
        r.advance(0.0, 1.0, 0)
    assert abs(r.mass[0] - 0.0) < TOL and abs(r.mass[1] - 10.0) < TOL
    r = Record(settings(0.9, 0.0))
    for _ in range(512):
        r.advance(2.0, 0.0, 1)
    r.advance(0.0, 1.0, 1)
    assert abs(r.raw[0] - 1.8) < TOL and abs(r.raw[3] - 1.0) < TOL
    for _ in range(200):
        r.advance(0.0, 1.0, 0)
    assert abs(r.mass[0] - 10.0) < TOL and abs(r.mass[1] - 0.0) < TOL


def test_disabled_history_is_the_fresh_mean():
    r = Record(settings(0.0, 0.0))
    r.advance(2.0, 0.25, 3)
    r.advance(1.0, 0.5, 2)
    np.testing.assert_allclose(r.raw, [1.0, 1.0, 1.0, 0.5], rtol=0, atol=0)


def cornell_receivers(n=24):
    k = (np.arange(n, dtype=np.float32) + np.float32(0.5)) / np.float32(n) * np.float32(1.9) - np.float32(0.95)
    x, z = np.meshgrid(k, k, indexing="ij")
    pos = np.zeros((n * n, 4), np.float32)
    pos[:, 0], pos[:, 2] = x.ravel(), z.ravel()
    nrm = np.zeros_like(pos)
    nrm[:, 1] = 1.0
    return pos, nrm


def test_oracle_frames_accumulate_history():
    s = bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=2,
                            emissive_samples=4, temporal_blend=0.88, split_transmittance_blend=0.98,
                            history_frames=24)
    pos, nrm = cornell_receivers()
    scene = oracle.OracleScene.from_packed(packed("cornell"))
    f1 = oracle.OracleFrame(scene, s.sanitized().to_c(), pos, nrm)
    s2 = s.sanitized()
    s2.frame_index = 1
    fresh = oracle.OracleFrame(scene, s2.to_c(), pos, nrm)
    blended = oracle.OracleFrame(scene, s2.to_c(), pos, nrm, previous=f1)
    dirs = s.direction_count(0)
    k1, m1, r1, c1 = f1.level(0, dirs)
    kf, mf, rf, cf = fresh.level(0, dirs)
    kb, mb, rb, cb = blended.level(0, dirs)
    np.testing.assert_array_equal(kf, kb)
    np.testing.assert_array_equal(cf, cb)  # samples are this frame's
    seen = (c1 > 0) & (cf > 0)
    # Records observed in both frames mix the two frames' means.
    lo = np.minimum(r1[seen][:, :3], rf[seen][:, :3]) - 1e-6
    hi = np.maximum(r1[seen][:, :3], rf[seen][:, :3]) + 1e-6
    assert np.all((rb[seen][:, :3] >= lo) & (rb[seen][:, :3] <= hi))
    assert np.any(np.abs(rb[seen][:, :3] - rf[seen][:, :3]) > 1e-4)
    # Records seen only before keep their history in the blended frame.
    kept = (c1 > 0) & (cf == 0)
    if kept.any():
        np.testing.assert_array_equal(rb[kept], r1[kept])
    # An invalidation box over the whole scene leaves only fresh data.
    reset = oracle.OracleFrame(scene, s2.to_c(), pos, nrm, previous=f1, dirty=[[-10, -10, -10, 10, 10, 10]])
    kr, mr, rr, cr = reset.level(0, dirs)
    np.testing.assert_array_equal(rr, rf)
    np.testing.assert_array_equal(mr, mf)


def keyset(keys):
    return {tuple(k[:3]) for k in keys}


def test_oracle_retains_unseen_cells_youngest_first():
    """retain (shaders/split.slang:991-1054) over a persistent world cache:
    cells of the previous frame that no receiver seeded stay with their
    records; capacity keeps whole age classes, youngest first (commitCache's
    youngest-kept rule, :1919-1961)."""
    base = bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=2,
                               emissive_samples=4, temporal_blend=0.88, split_transmittance_blend=0.98,
                               history_frames=24)
    pos, nrm = cornell_receivers()
    left, strip = pos[:, 0] < 0, np.abs(pos[:, 0]) < 0.2
    scene = oracle.OracleScene.from_packed(packed("cornell"))
    dirs = base.direction_count(0)

    def st(frame):
        s = base.sanitized()
        s.frame_index = frame
        return s.to_c()

    f0 = oracle.OracleFrame(scene, st(0), pos[left], nrm[left])
    f1 = oracle.OracleFrame(scene, st(1), pos[~left], nrm[~left], previous=f0)
    seeded1 = keyset(oracle.OracleFrame(scene, st(1), pos[~left], nrm[~left]).level(0, dirs)[0])
    k0, m0, r0, c0 = f0.level(0, dirs)
    k1, m1, r1, c1 = f1.level(0, dirs)
    assert keyset(k1) == keyset(k0) | seeded1
    i0 = {key: i for i, key in enumerate(map(tuple, k0[:, :3]))}
    kept = [(i, i0[tuple(k[:3])]) for i, k in enumerate(k1) if tuple(k[:3]) not in seeded1]
    assert kept
    for i, j in kept:  # no fresh samples: the record carries over unchanged
        assert np.all(c1[i] == 0)
        np.testing.assert_array_equal(r1[i], r0[j])

    # Frame 2 seeds a strip; frame 1's own cells are one frame old, the cells
    # only frame 0 saw are two frames old.
    seeded2 = keyset(oracle.OracleFrame(scene, st(2), pos[strip], nrm[strip]).level(0, dirs)[0])
    age1 = seeded1 - seeded2
    age2 = keyset(k0) - seeded1 - seeded2
    assert age1 and age2
    full = len(seeded2) + len(age1) + len(age2)
    for max_cells, expect in ((full, seeded2 | age1 | age2), (full - 1, seeded2 | age1),
                              (len(seeded2) + len(age1) - 1, seeded2)):
        f2 = oracle.OracleFrame(scene, st(2), pos[strip], nrm[strip], previous=f1, max_cells=max_cells)
        assert keyset(f2.level(0, dirs)[0]) == expect, max_cells
    # An invalidation box over the scene drops every unseen cell.
    f2 = oracle.OracleFrame(scene, st(2), pos[strip], nrm[strip], previous=f1, dirty=[[-10, -10, -10, 10, 10, 10]])
    assert keyset(f2.level(0, dirs)[0]) == seeded2


def test_oracle_multi_bounce_roles():
    """Multi-bounce roles of an oracle frame: the primary records one hit
    surface per receiver (its ray frame % R), the secondary cache over those
    sparse receivers leaves out first-hit emission, and a feedback frame adds
    non-negative diffuse bounce light at hits."""
    s = bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=2,
                            emissive_samples=4).sanitized()
    s2 = bp.RadianceCascades(probe_spacing=1.0, interval_length=1.6, levels=4, rays_per_receiver=2,
                             emissive_samples=4).sanitized()
    pos, nrm = cornell_receivers(16)
    pos[:, 3] = 1.0
    scene = oracle.OracleScene.from_packed(packed("cornell"))
    dirs = s.direction_count(0)
    p0 = oracle.OracleFrame(scene, s.to_c(), pos, nrm, record_hits=True)
    plain = oracle.OracleFrame(scene, s.to_c(), pos, nrm)
    for a, b in zip(p0.level(0, dirs), plain.level(0, dirs)):
        np.testing.assert_array_equal(a, b)  # recording changes nothing
    have = p0.hit_pos[:, 3] == 1.0
    assert have.mean() > 0.5
    assert np.all(np.isfinite(p0.hit_pos[have])) and np.all(np.abs(p0.hit_pos[have, :3]) <= 2.0 + 1e-5)
    np.testing.assert_allclose(np.linalg.norm(p0.hit_nrm[have, :3], axis=1), 1.0, rtol=1e-5)
    assert np.all(p0.hit_pos[~have] == 0.0)
    # Secondary cache over the sparse hit set: absent receivers seed nothing.
    sec = oracle.OracleFrame(scene, s2.to_c(), p0.hit_pos, p0.hit_nrm, sparse=True, skip_emission=True)
    dense = oracle.OracleFrame(scene, s2.to_c(), p0.hit_pos[have], p0.hit_nrm[have])
    assert {tuple(k[:3]) for k in sec.level(0, dirs)[0]} == {tuple(k[:3]) for k in dense.level(0, dirs)[0]}
    lit = oracle.OracleFrame(scene, s2.to_c(), p0.hit_pos, p0.hit_nrm, sparse=True)
    _, _, raw_skip, _ = sec.level(0, dirs)
    _, _, raw_lit, _ = lit.level(0, dirs)
    assert np.all(raw_skip[..., :3] <= raw_lit[..., :3] + 1e-7)
    assert np.any(raw_skip[..., :3] < raw_lit[..., :3] - 1e-4)  # rays that see the emitter lose it
    # Bounce light from the secondary's probes only adds.
    fed = oracle.OracleFrame(scene, s.to_c(), pos, nrm, feedback=sec)
    _, _, raw_fed, samples_fed = fed.level(0, dirs)
    _, _, raw_plain, samples_plain = plain.level(0, dirs)
    np.testing.assert_array_equal(samples_fed, samples_plain)
    assert np.all(raw_fed[..., :3] >= raw_plain[..., :3] - 1e-7)
    assert np.any(raw_fed[..., :3] > raw_plain[..., :3] + 1e-4)


def test_oracle_cached_hit_sky_roles():
    """cached_hit_sky: the secondary cache's escaped rays carry the sky
    (outgoingEnvironmentEscape), and hits its previous frame covers take
    their sky light from its probes instead of environment samples, so they
    trace fewer visibility queries; without feedback nothing changes."""
    sky = (2.0, 1.5, 1.0)
    s = bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=4, rays_per_receiver=2,
                            emissive_samples=4, environment=sky).sanitized()
    s2 = bp.RadianceCascades(probe_spacing=1.0, interval_length=1.6, levels=4, rays_per_receiver=2,
                             emissive_samples=4, environment=sky).sanitized()
    pos, nrm = cornell_receivers(16)
    pos[:, 3] = 1.0
    scene = oracle.OracleScene.from_packed(packed("cornell"))
    dirs = s.direction_count(0)
    p0 = oracle.OracleFrame(scene, s.to_c(), pos, nrm, record_hits=True)
    plain = oracle.OracleFrame(scene, s2.to_c(), p0.hit_pos, p0.hit_nrm, sparse=True, skip_emission=True)
    cached = oracle.OracleFrame(scene, s2.to_c(), p0.hit_pos, p0.hit_nrm, sparse=True, skip_emission=True,
                                cached_sky=True)
    # First frame: no feedback, so every hit still samples the sky; escapes now carry it.
    assert cached.stats().shadow_rays == plain.stats().shadow_rays
    last = s2.levels - 1  # escapes deposit their radiance in the last level, which owns the tail
    _, _, raw_c, _ = cached.level(last, s2.direction_count(last))
    _, _, raw_p, _ = plain.level(last, s2.direction_count(last))
    assert np.all(raw_c[..., :3] >= raw_p[..., :3] - 1e-7)
    assert np.any(raw_c[..., :3] > raw_p[..., :3] + 1e-3)  # the open front's escapes
    # Next frame with the secondary's probes as feedback: covered hits skip the sky samples.
    fed = oracle.OracleFrame(scene, s.to_c(), pos, nrm, feedback=cached)
    fed_cached = oracle.OracleFrame(scene, s.to_c(), pos, nrm, feedback=cached, cached_sky=True)
    assert fed_cached.stats().shadow_rays < fed.stats().shadow_rays
    _, _, raw_fc, samples_fc = fed_cached.level(0, dirs)
    _, _, raw_f, samples_f = fed.level(0, dirs)
    np.testing.assert_array_equal(samples_fc, samples_f)
    assert np.all(np.isfinite(raw_fc))


def support_children():
    """The child records of supportCases stages 3-5: only child 0, corner 0
    carries (8, support 0.25); the parent sits at fraction 0."""
    children = np.zeros((4, 8, 4), np.float32)
    children[0, 0] = (8, 8, 8, 0.25)
    return children


def test_transparent_history_passes_partial_children():
    """supportCases result[5] (src/split_merge_tests.rs:136-142, asserted at
    :1370-1371 under run(0, 0.9)): no fresh observation, the previous record
    transparent (J 7, beta 1, transmittance mass 4): the radiance blend is
    off, so the interval has no support of its own and passes the partially
    supported child through."""
    st = settings(0.0, 0.9)
    r = oracle.merge_history_entry(st, (0, 0, 0, 1), 0, (7, 7, 7, 1), (0, 4), (0, 0, 0), support_children())
    assert abs(r[0] - 8.0) < TOL
    assert abs(r[3] - 0.0625) < TOL


def test_opaque_history_cannot_invent_support():
    """supportCases result[6] (src/split_merge_tests.rs:143-148, asserted at
    :1372): the previous record's beta set to 0 (opaque) with no radiance
    mass: nothing passes and nothing is supported."""
    st = settings(0.0, 0.9)
    r = oracle.merge_history_entry(st, (0, 0, 0, 1), 0, (7, 7, 7, 0), (0, 4), (0, 0, 0), support_children())
    np.testing.assert_array_equal(r, [0, 0, 0, 0])
