"""Split sample sequence order (the reference's rank / parents / prefix
passes, shaders/split.slang:788-963): receivers of one cascade-0 probe take
consecutive places in the R2 sequence, and the probes under every coarser
probe form one contiguous run (siblings adjacent, octant ordinal x + 2y + 4z),
so each probe's rays are consecutive sequence points."""
import numpy as np

import bevy_penumbra_b200 as bp
import oracle


def receivers(n, seed):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(-3.0, 3.0, (n, 3))
    pos[:, 3] = 1.0
    return pos


def cells(pos, spacing, level):
    return np.floor(pos[:, :3] / np.float32(spacing * (1 << level))).astype(np.int64)


def test_order_is_a_permutation_grouped_by_probe_and_parent():
    s = bp.RadianceCascades(probe_spacing=0.5, levels=4).sanitized()
    pos = receivers(3000, 1)
    order = oracle.sequence_order(s.to_c(), pos)
    assert sorted(order.tolist()) == list(range(len(pos)))
    by_place = np.argsort(order)
    for level in range(4):
        c = cells(pos, 0.5, level)[by_place]
        keys = [tuple(k) for k in c]
        seen, prev = set(), None
        for k in keys:  # every probe of this level is one contiguous run
            if k != prev:
                assert k not in seen, (level, k)
                seen.add(k)
            prev = k
    # Within a probe, receivers keep their index order.
    c0 = cells(pos, 0.5, 0)
    for key in {tuple(k) for k in c0[:50]}:
        members = np.flatnonzero((c0 == key).all(axis=1))
        np.testing.assert_array_equal(np.sort(order[members]), order[members])
        assert order[members].max() - order[members].min() == len(members) - 1


def test_siblings_follow_the_octant_ordinal():
    s = bp.RadianceCascades(probe_spacing=1.0, levels=2).sanitized()
    pos = np.zeros((8, 4), np.float32)
    for o in range(8):  # the eight children of parent cell (0, 0, 0), listed in reverse
        x, y, z = 7 - o & 1, (7 - o) >> 1 & 1, (7 - o) >> 2 & 1
        pos[o, :3] = (x + 0.5, y + 0.5, z + 0.5)
        pos[o, 3] = 1.0
    order = oracle.sequence_order(s.to_c(), pos)
    np.testing.assert_array_equal(order, np.arange(8)[::-1])


def test_absent_receivers_come_last():
    s = bp.RadianceCascades(probe_spacing=0.5, levels=4).sanitized()
    pos = receivers(200, 2)
    pos[::3, 3] = 0.0
    order = oracle.sequence_order(s.to_c(), pos, sparse=True)
    absent = pos[:, 3] == 0.0
    assert order[absent].min() == (~absent).sum()
    np.testing.assert_array_equal(order[absent], np.arange((~absent).sum(), len(pos)))
