"""The reference's fault topologies for traversal, rebuilt on packed word
streams (test infrastructure).

* forced_deep: forced_deep_scene (src/traversal_tests.rs:1521-1592): the
  TLAS, or every BLAS, replaced by a valid binary tree whose first-child path
  is `internals` inner nodes deep, every node carrying the root's box and
  every leaf the whole element range, so a depth-first walk keeps one
  pending node per level and overflows its stack.  The reference uses 64
  inner nodes against its 49-entry stack; `internals` is a parameter here
  because the device walks a 4-wide BVH (one pending entry per three binary
  levels) whose stacks hold 32 or 64 entries.
* forced_cyclic_blas: forced_cyclic_blas_scene (:1594-1617): one instance's
  BLAS root becomes an inner node whose first child is itself.
* forced_oversized_leaf: forced_oversized_blas_leaf (:1618-1636): one
  instance's BLAS root becomes a leaf claiming u32::MAX - first elements.
* shared_subtree: a BVH whose every level's two inner nodes share one pair of
  children (a DAG that doubles the number of paths per level).
"""
from __future__ import annotations

import numpy as np

import bevy_penumbra_b200 as bp

INSTANCE_WORDS = 9


class Words:
    """A packed scene's word streams split into binary nodes, instance records
    and material words (the layout of src/scene.rs:2096-2117)."""

    def __init__(self, packed: bp.PackedScene):
        sw = packed.scene_words
        self.packed = packed
        _, base, count, stride = (int(v) for v in sw[0])
        assert stride == INSTANCE_WORDS
        self.tlas_count = int(packed.tlas_nodes)
        self.blas_count = int(packed.blas_nodes)
        assert 1 + 2 * (self.tlas_count + self.blas_count) == base
        nodes = [self._node(sw, i) for i in range(self.tlas_count + self.blas_count)]
        self.tlas = nodes[:self.tlas_count]
        # BLAS nodes with local child indices.
        self.blas = []
        for n in nodes[self.tlas_count:]:
            n = dict(n)
            if n["count"] == 0:
                n["first"] -= self.tlas_count
            self.blas.append(n)
        self.material_base = base + count * INSTANCE_WORDS
        self.instances = [sw[base + INSTANCE_WORDS * k: base + INSTANCE_WORDS * (k + 1)].copy() for k in range(count)]
        self.materials = sw[self.material_base:].copy()

    @staticmethod
    def _node(sw, i):
        a, b = sw[1 + 2 * i], sw[2 + 2 * i]
        return {"min": a[:3].copy(), "max": b[:3].copy(), "first": int(a[3]), "count": int(b[3])}

    def blas_root(self, k: int) -> int:
        """Local BLAS index of instance k's root."""
        return int(self.instances[k][8][0]) - self.tlas_count

    def pack(self) -> bp.PackedScene:
        t, b = len(self.tlas), len(self.blas)
        base = 1 + 2 * (t + b)
        material_base = base + INSTANCE_WORDS * len(self.instances)
        words = [np.array([material_base + len(self.materials), base, len(self.instances), INSTANCE_WORDS],
                          np.uint32)]

        def node_words(n, offset):
            first = n["first"] + (offset if n["count"] == 0 else 0)
            words.append(np.concatenate([n["min"], [first]]).astype(np.uint32))
            words.append(np.concatenate([n["max"], [n["count"]]]).astype(np.uint32))

        for n in self.tlas:
            node_words(n, 0)
        for n in self.blas:
            node_words(n, t)
        for inst in self.instances:
            w = inst.copy()
            w[7][3] = int(w[7][3]) - self.material_base + material_base
            words.extend(w)
        words.extend(self.materials)
        sw = np.stack(words).astype(np.uint32)
        p = self.packed
        out = bp.PackedScene(sw, p.geometry_words, p.lights, p.instance_order, p.blas_cost, p.max_depth, t, b)
        out.conventional = p.conventional
        return out


def chain(nodes: list, mn, mx, first: int, count: int, internals: int) -> int:
    """Appends the deep binary tree of forced_deep_scene; returns its root
    (local index).  Node 0 and the odd nodes below 2 x internals - 1 are
    inner nodes; every other node is a leaf over [first, first + count)."""
    root = len(nodes)
    for i in range(2 * internals + 1):
        internal = i == 0 or (i % 2 == 1 and i < 2 * internals - 1)
        nodes.append({"min": np.array(mn, np.uint32), "max": np.array(mx, np.uint32),
                      "first": root + (1 if i == 0 else i + 2) if internal else first,
                      "count": 0 if internal else count})
    return root


def forced_deep(packed: bp.PackedScene, blas: bool, internals: int = 64) -> bp.PackedScene:
    w = Words(packed)
    if blas:
        nodes, roots = [], {}
        for k, inst in enumerate(w.instances):
            first, count = int(inst[8][1]), int(inst[8][2])
            if first not in roots:
                bounds = w.blas[w.blas_root(k)]
                roots[first] = chain(nodes, bounds["min"], bounds["max"], first, count, internals)
        tlas_count = len(w.tlas)
        for inst in w.instances:
            inst[8][0] = tlas_count + roots[int(inst[8][1])]
        w.blas = nodes
    else:
        old = len(w.tlas)
        bounds = w.tlas[0]
        nodes = []
        chain(nodes, bounds["min"], bounds["max"], 0, len(w.instances), internals)
        w.tlas = nodes
        for inst in w.instances:
            inst[8][0] = int(inst[8][0]) - old + len(nodes)
    return w.pack()


def forced_cyclic_blas(packed: bp.PackedScene, instance: int) -> bp.PackedScene:
    w = Words(packed)
    j = w.blas_root(instance)
    b = w.blas[j]
    w.blas[j] = {"min": b["min"], "max": b["max"], "first": j, "count": 0}
    far = np.array([100.0, 100.0, 100.0], np.float32).view(np.uint32)
    far1 = np.array([101.0, 101.0, 101.0], np.float32).view(np.uint32)
    w.blas[j + 1] = {"min": far, "max": far1, "first": 0, "count": 1}
    return w.pack()


def forced_oversized_leaf(packed: bp.PackedScene, instance: int) -> bp.PackedScene:
    w = Words(packed)
    j = w.blas_root(instance)
    b = w.blas[j]
    first = int(w.instances[instance][8][1])
    w.blas[j] = {"min": b["min"], "max": b["max"], "first": first, "count": 0xFFFFFFFF - first}
    return w.pack()


def two_child_self_loop(packed: bp.PackedScene) -> bp.PackedScene:
    """TLAS node 0 and node 1 both inner nodes whose children are nodes 0 and 1."""
    w = Words(packed)
    assert len(w.tlas) >= 2
    for i in (0, 1):
        w.tlas[i] = dict(w.tlas[i], first=0, count=0)
    return w.pack()


def shared_subtree(packed: bp.PackedScene, levels: int = 90) -> bp.PackedScene:
    """A TLAS where nodes 2k + 1 and 2k + 2 are both inner nodes over the same
    children 2k + 3 and 2k + 4, `levels` deep: 2^levels root-to-leaf paths over
    2 x levels + 3 nodes."""
    w = Words(packed)
    root = w.tlas[0]
    n_inst = len(w.instances)
    nodes = [{"min": root["min"], "max": root["max"], "first": 1, "count": 0}]
    for k in range(levels):
        for _ in range(2):
            nodes.append({"min": root["min"], "max": root["max"], "first": 2 * k + 3, "count": 0})
    for _ in range(2):
        nodes.append({"min": root["min"], "max": root["max"], "first": 0, "count": n_inst})
    old = len(w.tlas)
    w.tlas = nodes
    for inst in w.instances:
        inst[8][0] = int(inst[8][0]) - old + len(nodes)
    return w.pack()
