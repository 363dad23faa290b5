"""The oracle's own scene packer (oracle/orc_pack.c) against liblux's
(lux_scene_pack): two restatements of build_tree / node_words /
pack_instances / geometry_words / build_emissive_lights
(src/scene.rs:2398-2554, :1025-1038, :1071-1122, :809-823, :2311-2372)
written apart must produce identical words.  No GPU needed."""
import numpy as np
import pytest

import bevy_penumbra_b200 as bp
import oracle
from bevy_penumbra_b200 import scenes
from tests.helpers import scene_desc


@pytest.mark.parametrize("name", ["cornell", "traversal24", "atrium65536", "batch"])
def test_oracle_packer_words_equal_the_library_packer(name):
    desc = scenes.batch_scene(44, 5000) if name == "batch" else scene_desc(name)
    lib_packed = bp.PackedScene.from_desc(desc)
    orc_packed = oracle.OraclePacked.from_desc(desc)
    np.testing.assert_array_equal(orc_packed.scene_words, lib_packed.scene_words)
    np.testing.assert_array_equal(orc_packed.geometry_words, lib_packed.geometry_words)
    np.testing.assert_array_equal(orc_packed.lights, lib_packed.lights)
    np.testing.assert_array_equal(orc_packed.instance_order, lib_packed.instance_order)
    assert (orc_packed.tlas_nodes, orc_packed.blas_nodes) == (lib_packed.tlas_nodes, lib_packed.blas_nodes)
    assert orc_packed.max_depth == lib_packed.max_depth
    assert orc_packed.blas_cost == lib_packed.blas_cost


def test_coincident_centroids_split_in_order():
    """The median fallback (no binned split: every centroid coincides) keeps
    the elements' order and splits at len / 2 in both packers."""
    sc = scenes.SceneDesc(name="coincident")
    mat = sc.add_material(scenes.material_words((0.5, 0.5, 0.5)))
    # Every triangle spans the cube [-1, 1]^3: equal boxes, equal centroids.
    rng = np.random.default_rng(8)
    inner = rng.uniform(-0.9, 0.9, size=(37, 3)).astype(np.float32)
    verts = np.concatenate([np.array([[-1, -1, -1], [1, 1, 1]], np.float32), inner])
    idx = np.array([[0, 1, 2 + k] for k in range(37)], np.uint32)
    mesh = sc.add_mesh(scenes.Mesh(verts, idx))
    sc.add_instance(mesh, np.eye(3, 4, dtype=np.float32), flags=0, material=mat)
    a, b = bp.PackedScene.from_desc(sc), oracle.OraclePacked.from_desc(sc)
    np.testing.assert_array_equal(b.scene_words, a.scene_words)
    np.testing.assert_array_equal(b.geometry_words, a.geometry_words)
    # Leaf order is the input order: a root split at 18 | 19 down to leaves of <= 4.
    np.testing.assert_array_equal(b.geometry_words[1:38, 2], np.arange(2, 39))
