"""Rigid pose updates shared by the refit tests: seeded moves of a scene's
instances (rotation about y plus a translation), returned both as a new
scene description and in a packed scene's instance-record (slot) order."""
from __future__ import annotations

import copy
import math

import numpy as np

from bevy_penumbra_b200 import scenes


def move_instances(desc: scenes.SceneDesc, seed: int, select=None) -> scenes.SceneDesc:
    """A copy of `desc` whose selected instances are turned about y by up to
    0.3 rad and shifted by up to 0.5 m (seeded)."""
    rng = np.random.default_rng(seed)
    out = copy.deepcopy(desc)
    for i, m in enumerate(desc.instance_transform):
        if select is not None and not select(i):
            continue
        phi = float(rng.uniform(-0.3, 0.3))
        c, s = math.cos(phi), math.sin(phi)
        rot = np.array([[c, 0.0, s], [0.0, 1.0, 0.0], [-s, 0.0, c]])
        m64 = m.astype(np.float64)
        new = np.zeros((3, 4))
        new[:, :3] = rot @ m64[:, :3]
        new[:, 3] = rot @ m64[:, 3] + rng.uniform(-0.5, 0.5, size=3)
        out.instance_transform[i] = new.astype(np.float32)
    return out


def slot_transforms(desc: scenes.SceneDesc, packed) -> np.ndarray:
    """desc's world_from_local rows in packed's instance-record order."""
    return np.stack([desc.instance_transform[int(i)] for i in packed.instance_order]).astype(np.float32)


def atrium_select(desc: scenes.SceneDesc):
    """Columns, arches and floor tiles move; emitters and the ceiling stay
    (so the emissive light records stay valid)."""
    column, arch, tile = 0, 1, 2
    return lambda i: desc.instance_mesh[i] in (column, arch, tile)
