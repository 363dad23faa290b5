"""Oracle refit (rigid pose update + refitTlas by depth,
shaders/acceleration.slang:61-88): a refit scene answers every ray exactly
like the scene packed from scratch at the new pose."""
import numpy as np
import pytest

import bevy_penumbra_b200 as bp
import oracle
from tests.helpers import EMPTY, packed, rays_for, scene_desc
from tests.refit_cases import atrium_select, move_instances, slot_transforms


def random_rays(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    rays = np.zeros(n, dtype=bp.RAY_DTYPE)
    rays["origin"] = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays["direction"] = d.astype(np.float32)
    rays["limit"] = 1e20
    return rays


def same_hits(a, order_a, b, order_b):
    """Hits agree bit for bit; instances compared by original instance id."""
    hit_a, hit_b = a["triangle"] != EMPTY, b["triangle"] != EMPTY
    np.testing.assert_array_equal(hit_a, hit_b)
    np.testing.assert_array_equal(a["triangle"], b["triangle"])
    np.testing.assert_array_equal(a["distance"][hit_a].view(np.uint32), b["distance"][hit_b].view(np.uint32))
    np.testing.assert_array_equal(order_a[a["instance"][hit_a]], order_b[b["instance"][hit_b]])
    return int(hit_a.sum())


@pytest.mark.parametrize("name", ["traversal24", "atrium65536"])
def test_oracle_refit_matches_fresh_pack(name):
    desc = scene_desc(name)
    p0 = packed(name)
    select = atrium_select(desc) if name.startswith("atrium") else None
    moved = move_instances(desc, seed=17, select=select)
    p1 = bp.PackedScene.from_desc(moved)
    refit = oracle.OracleScene.from_packed(p0)
    refit.refit(slot_transforms(moved, p0))
    fresh = oracle.OracleScene.from_packed(p1)
    rays = rays_for(moved) if name == "traversal24" else random_rays(20000, (-7, 0.2, -7), (7, 9.5, 7), 5)
    a, _ = refit.trace_rays(rays)
    b, _ = fresh.trace_rays(rays)
    hits = same_hits(a, p0.instance_order, b, p1.instance_order)
    assert hits > 1000
    occ_a, _ = refit.trace_rays(rays, any_hit=True)
    occ_b, _ = fresh.trace_rays(rays, any_hit=True)
    np.testing.assert_array_equal(occ_a["triangle"] != EMPTY, occ_b["triangle"] != EMPTY)


def test_oracle_refit_rejects_bad_pose():
    p0 = packed("traversal24")
    sc = oracle.OracleScene.from_packed(p0)
    m = slot_transforms(scene_desc("traversal24"), p0)
    with pytest.raises(ValueError):
        sc.refit(m[:-1])
    m[3, :, :3] = 0.0
    with pytest.raises(ValueError):
        sc.refit(m)


def test_oracle_refit_round_trip_restores_words():
    """Refitting back to the packed pose reproduces the packer's instance
    rows exactly and boxes that contain the packer's."""
    p0 = packed("traversal24")
    sc = oracle.OracleScene.from_packed(p0)
    desc = scene_desc("traversal24")
    sc.refit(slot_transforms(move_instances(desc, 3), p0))
    sc.refit(slot_transforms(desc, p0))
    words = sc.words()
    base, count, stride = int(p0.scene_words[0, 1]), int(p0.scene_words[0, 2]), int(p0.scene_words[0, 3])
    for i in range(count):
        rows = slice(base + i * stride, base + i * stride + 6)
        np.testing.assert_array_equal(words[rows], p0.scene_words[rows])
    # TLAS node boxes: refit boxes enclose the packer's boxes of the same nodes.
    n_tlas = base  # node words precede the instances; check the root
    lo0, hi0 = p0.scene_words[1, :3].view(np.float32), p0.scene_words[2, :3].view(np.float32)
    lo1, hi1 = words[1, :3].view(np.float32), words[2, :3].view(np.float32)
    assert n_tlas > 2
    assert np.all(lo1 <= lo0 + 1e-4) and np.all(hi1 >= hi0 - 1e-4)


def test_emissive_lights_follow_moved_emitters():
    """lux_emissive_lights_at at a new pose gives the records a fresh pack at
    that pose builds (position, normal, edges), keeping the CDF."""
    name = "atrium65536"
    desc = scene_desc(name)
    p0 = packed(name)
    emitters = [i for i in range(len(desc.instance_mesh)) if desc.instance_mesh[i] == 3]
    assert len(emitters) == 3
    moved = move_instances(desc, seed=31, select=lambda i: i in emitters)
    lights = p0.lights_at(slot_transforms(moved, p0))
    p1 = bp.PackedScene.from_desc(moved)
    def records(p, lt):
        flat = np.ascontiguousarray(lt).view(np.float32).reshape(len(lt), 24)
        src = np.ascontiguousarray(lt).view(np.uint32).reshape(len(lt), 24)[:, 20:22]
        return {(int(p.instance_order[s]), int(t)): flat[k] for k, (s, t) in enumerate(src)}
    a, b = records(p0, lights), records(p1, p1.lights)
    assert set(a) == set(b) and len(a) > 0
    for key in a:
        np.testing.assert_array_equal(a[key][0:3], b[key][0:3])      # position
        np.testing.assert_array_equal(a[key][8:11], b[key][8:11])    # direction (facing normal)
        np.testing.assert_array_equal(a[key][12:15], b[key][12:15])  # edge1
        np.testing.assert_array_equal(a[key][16:19], b[key][16:19])  # edge2
    # Unmoved records (and every CDF field) are unchanged.
    np.testing.assert_array_equal(np.ascontiguousarray(lights).view(np.float32).reshape(-1, 24)[:, [11, 15, 7]],
                                  np.ascontiguousarray(p0.lights).view(np.float32).reshape(-1, 24)[:, [11, 15, 7]])
