"""Seeded synthetic scenes and receiver sets for the transport path.

No dataset or asset is used: every scene is generated from a seed with the
shapes and value ranges of the workloads the transport is measured on.

* ``cornell``  Cornell box, 34 triangles: five axis-aligned walls of a 2 m
  cube (white 0.75, red / green side walls 0.65), a short and a tall box
  rotated by seeded angles, and a 0.5 m^2 quad emitter of radiance 15.
* ``atrium``   procedural atrium of exactly ``triangles`` world triangles
  (default 262,144): instanced columns, arches and floor tiles with uniform
  jitter in [-0.02, 0.02] m, a coffered ceiling, three rectangular emitters of
  radiance U[5, 20] and albedo U[0.2, 0.8].
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

F32 = np.float32


def material_words(albedo, emission=(0.0, 0.0, 0.0), metallic=0.0, roughness=1.0, reflectance=0.5,
                   exposure_weight=1.0) -> np.ndarray:
    """One material as the reference's 8 uint4 words (material_words,
    src/material.rs:132): base colour, emission + alpha cutoff (-1 opaque),
    (metallic, roughness, reflectance, exposure weight), UV rows, texture
    slots (EMPTY = untextured)."""
    w = np.zeros(32, dtype=np.uint32)
    f = w.view(np.float32)
    f[0:3] = albedo
    f[3] = 1.0
    f[4:7] = emission
    f[7] = -1.0
    f[8:12] = (metallic, roughness, reflectance, exposure_weight)
    f[16:19] = (1.0, 0.0, 0.0)
    f[20:23] = (0.0, 1.0, 0.0)
    w[24:29] = 0xFFFFFFFF
    return w


@dataclass
class Mesh:
    positions: np.ndarray  # (V, 3) float32
    indices: np.ndarray    # (T, 3) uint32 local vertex ids


@dataclass
class SceneDesc:
    meshes: list = field(default_factory=list)
    instance_mesh: list = field(default_factory=list)
    instance_transform: list = field(default_factory=list)  # 3x4 row-major world_from_local
    instance_flags: list = field(default_factory=list)
    instance_material: list = field(default_factory=list)
    materials: list = field(default_factory=list)
    name: str = ""

    def add_mesh(self, mesh: Mesh) -> int:
        self.meshes.append(mesh)
        return len(self.meshes) - 1

    def add_material(self, words: np.ndarray) -> int:
        self.materials.append(words)
        return len(self.materials) - 1

    def add_instance(self, mesh: int, transform=None, flags: int = 8, material: int = 0) -> None:
        if transform is None:
            transform = np.eye(3, 4, dtype=np.float32)
        self.instance_mesh.append(mesh)
        self.instance_transform.append(np.asarray(transform, dtype=np.float32).reshape(3, 4))
        self.instance_flags.append(flags)
        self.instance_material.append(material)

    def world_triangles(self) -> int:
        return int(sum(len(self.meshes[m].indices) for m in self.instance_mesh))

    def arrays(self):
        """Flattened global vertex/index arrays and mesh ranges."""
        positions, indices, first, count = [], [], [], []
        vbase = tbase = 0
        for mesh in self.meshes:
            positions.append(np.asarray(mesh.positions, dtype=np.float32))
            indices.append(np.asarray(mesh.indices, dtype=np.uint32) + vbase)
            first.append(tbase)
            count.append(len(mesh.indices))
            vbase += len(mesh.positions)
            tbase += len(mesh.indices)
        return (np.concatenate(positions).astype(np.float32), np.concatenate(indices).astype(np.uint32),
                np.asarray(first, np.uint32), np.asarray(count, np.uint32))


def quad(p0, p1, p2, p3) -> Mesh:
    """Two triangles (p0 p1 p2), (p0 p2 p3); normal = (p1-p0) x (p2-p0)."""
    return Mesh(np.array([p0, p1, p2, p3], dtype=np.float32), np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32))


def box_mesh(size, bottom: bool = True) -> Mesh:
    """Axis-aligned box centred on x/z with its base at y = 0, outward normals."""
    sx, sy, sz = (s * 0.5 for s in (size[0], 0.0, size[2]))
    h = size[1]
    v = np.array([[-sx, 0, -sz], [sx, 0, -sz], [sx, 0, sz], [-sx, 0, sz],
                  [-sx, h, -sz], [sx, h, -sz], [sx, h, sz], [-sx, h, sz]], dtype=np.float32)
    faces = [
        [4, 7, 6, 5],  # top (+y)
        [0, 4, 5, 1],  # -z
        [1, 5, 6, 2],  # +x
        [2, 6, 7, 3],  # +z
        [3, 7, 4, 0],  # -x
    ]
    if bottom:
        faces.append([0, 1, 2, 3])  # -y
    tri = []
    for a, b, c, d in faces:
        tri += [[a, b, c], [a, c, d]]
    return Mesh(v, np.array(tri, dtype=np.uint32))


def rotation_y(angle: float, translation=(0.0, 0.0, 0.0)) -> np.ndarray:
    c, s = math.cos(angle), math.sin(angle)
    return np.array([[c, 0, s, translation[0]], [0, 1, 0, translation[1]], [-s, 0, c, translation[2]]],
                    dtype=np.float32)


def cornell(seed: int = 1) -> SceneDesc:
    """The 34-triangle Cornell box (see module docstring)."""
    rng = np.random.default_rng(seed)
    sc = SceneDesc(name="cornell")
    white = sc.add_material(material_words((0.75, 0.75, 0.75)))
    red = sc.add_material(material_words((0.65, 0.05, 0.05)))
    green = sc.add_material(material_words((0.05, 0.65, 0.05)))
    side = math.sqrt(0.5)
    light = sc.add_material(material_words((0.0, 0.0, 0.0), emission=(15.0, 15.0, 15.0)))
    # Room [-1, 1] x [0, 2] x [-1, 1], open at z = +1; normals point inward.
    floor = sc.add_mesh(quad((-1, 0, -1), (-1, 0, 1), (1, 0, 1), (1, 0, -1)))
    ceiling = sc.add_mesh(quad((-1, 2, -1), (1, 2, -1), (1, 2, 1), (-1, 2, 1)))
    back = sc.add_mesh(quad((-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1)))
    left = sc.add_mesh(quad((-1, 0, -1), (-1, 2, -1), (-1, 2, 1), (-1, 0, 1)))
    right = sc.add_mesh(quad((1, 0, -1), (1, 0, 1), (1, 2, 1), (1, 2, -1)))
    h = side * 0.5
    emitter = sc.add_mesh(quad((-h, 1.99, -h), (h, 1.99, -h), (h, 1.99, h), (-h, 1.99, h)))
    short_box = sc.add_mesh(box_mesh((0.6, 0.6, 0.6), bottom=False))
    tall_box = sc.add_mesh(box_mesh((0.6, 1.2, 0.6), bottom=True))
    for m in (floor, ceiling, back):
        sc.add_instance(m, material=white)
    sc.add_instance(left, material=red)
    sc.add_instance(right, material=green)
    sc.add_instance(emitter, material=light)
    a0, a1 = rng.uniform(-0.6, 0.6, size=2)
    sc.add_instance(short_box, rotation_y(float(a0), (0.35, 0.0, 0.35)), material=white)
    sc.add_instance(tall_box, rotation_y(float(a1), (-0.35, 0.0, -0.3)), material=white)
    assert sc.world_triangles() == 34
    return sc


def cylinder_mesh(radius: float, height: float, sides: int, rings: int) -> Mesh:
    ang = np.linspace(0.0, 2.0 * math.pi, sides, endpoint=False)
    ys = np.linspace(0.0, height, rings + 1)
    v = [(radius * math.cos(a), y, radius * math.sin(a)) for y in ys for a in ang]
    tri = []
    for r in range(rings):
        for s in range(sides):
            a = r * sides + s
            b = r * sides + (s + 1) % sides
            c = (r + 1) * sides + (s + 1) % sides
            d = (r + 1) * sides + s
            tri += [[a, d, c], [a, c, b]]
    top = len(v)
    v.append((0.0, height, 0.0))
    for s in range(sides):
        tri.append([top, (rings) * sides + (s + 1) % sides, rings * sides + s])
    return Mesh(np.array(v, dtype=np.float32), np.array(tri, dtype=np.uint32))


def arch_mesh(span: float, thickness: float, depth: float, segments: int) -> Mesh:
    """Semicircular arch of rectangular section between x = -span/2 and +span/2."""
    r_in = span * 0.5 - thickness * 0.5
    r_out = span * 0.5 + thickness * 0.5
    ang = np.linspace(math.pi, 0.0, segments + 1)
    v = []
    for a in ang:
        for r in (r_in, r_out):
            for z in (-depth * 0.5, depth * 0.5):
                v.append((r * math.cos(a), r * math.sin(a), z))
    tri = []
    for s in range(segments):
        base, nxt = 4 * s, 4 * (s + 1)
        # vertex order per ring: (in,-z) (in,+z) (out,-z) (out,+z)
        for (a, b) in ((0, 1), (3, 2), (2, 0), (1, 3)):
            p, q, r_, t = base + a, base + b, nxt + b, nxt + a
            tri += [[p, q, r_], [p, r_, t]]
    return Mesh(np.array(v, dtype=np.float32), np.array(tri, dtype=np.uint32))


def grid_mesh(quads: int, size_x: float, size_z: float, y: float, rng, jitter: float) -> Mesh:
    """`quads` quads of a near-square row-major grid (the last row may be
    partial), facing -y, vertex heights jittered by U[-jitter, jitter]."""
    nx = max(1, int(math.ceil(math.sqrt(quads))))
    nz = (quads + nx - 1) // nx
    xs = np.linspace(-size_x * 0.5, size_x * 0.5, nx + 1)
    zs = np.linspace(-size_z * 0.5, size_z * 0.5, nz + 1)
    v = np.array([(x, y, z) for z in zs for x in xs], dtype=np.float64)
    v[:, 1] += rng.uniform(-jitter, jitter, size=len(v))
    tri = []
    for q in range(quads):
        j, i = divmod(q, nx)
        a = j * (nx + 1) + i
        b, c, d = a + 1, a + nx + 2, a + nx + 1
        tri += [[a, c, b], [a, d, c]]  # normal -y (ceiling seen from below)
    return Mesh(v.astype(np.float32), np.array(tri, dtype=np.uint32))


def atrium(seed: int = 2, triangles: int = 262_144) -> SceneDesc:
    """Procedural atrium with exactly ``triangles`` world triangles."""
    rng = np.random.default_rng(seed)
    sc = SceneDesc(name="atrium")
    jit = lambda: rng.uniform(-0.02, 0.02, size=3)

    def albedo_material():
        return sc.add_material(material_words(tuple(rng.uniform(0.2, 0.8, size=3))))

    column = sc.add_mesh(cylinder_mesh(0.3, 6.0, 32, 16))          # 32*16*2 + 32 = 1056
    arch = sc.add_mesh(arch_mesh(4.0, 0.4, 0.6, 60))               # 60*4*2 = 480
    tile = sc.add_mesh(box_mesh((0.98, 0.05, 0.98), bottom=False))  # 10
    emitter_mesh = sc.add_mesh(quad((-1.0, 0.0, -1.0), (1.0, 0.0, -1.0), (1.0, 0.0, 1.0), (-1.0, 0.0, 1.0)))
    # Columns on an n x n grid with 4 m pitch (10 x 10 at full size).
    large = triangles >= 200_000
    pitch, n = 4.0, (10 if large else 4)
    tiles = 40 if large else 16
    for i in range(n):
        for j in range(n):
            t = np.eye(3, 4, dtype=np.float64)
            t[:, 3] = ((i - (n - 1) / 2) * pitch, 0.0, (j - (n - 1) / 2) * pitch) + jit()
            sc.add_instance(column, t, material=albedo_material())
    # Arches between neighbouring columns along x and along z.
    for i in range(n - 1):
        for j in range(n):
            cx = (i + 0.5 - (n - 1) / 2) * pitch
            cz = (j - (n - 1) / 2) * pitch
            sc.add_instance(arch, rotation_y(0.0, (cx, 6.0, cz)) + _jit3(jit), material=albedo_material())
            sc.add_instance(arch, rotation_y(math.pi / 2, (cz, 6.0, cx)) + _jit3(jit), material=albedo_material())
    # Floor tiles, 1 m pitch (40 x 40 m at full size).
    for i in range(tiles):
        for j in range(tiles):
            t = np.eye(3, 4, dtype=np.float64)
            t[:, 3] = (i - (tiles - 1) / 2, -0.05, j - (tiles - 1) / 2) + jit()
            sc.add_instance(tile, t, material=albedo_material())
    # Three emitters under the ceiling, radiance U[5, 20].
    for k in range(3):
        radiance = float(rng.uniform(5.0, 20.0))
        mat = sc.add_material(material_words((0.0, 0.0, 0.0), emission=(radiance, radiance, radiance)))
        t = np.eye(3, 4, dtype=np.float64)  # the quad faces -y
        t[:, 3] = ((k - 1) * pitch * n * 0.3, 9.5, rng.uniform(-0.15, 0.15) * pitch * n)
        sc.add_instance(emitter_mesh, t, material=mat)
    # Coffered ceiling fills the remaining triangle budget exactly.
    remaining = triangles - sc.world_triangles()
    if remaining < 2 or remaining % 2:
        raise ValueError(f"atrium triangle budget {triangles} cannot be met (remaining {remaining})")
    extent = pitch * n + 4.0
    ceiling = sc.add_mesh(grid_mesh(remaining // 2, extent, extent, 10.0, rng, 0.02))
    sc.add_instance(ceiling, material=albedo_material())
    assert sc.world_triangles() == triangles, (sc.world_triangles(), triangles)
    return sc


def full_scene(seed: int = 5, triangles: int = 1_048_576):
    """The full-form scene: the atrium layout at ``triangles`` world triangles
    with four emitters (radiance U[5, 20]) and eight rigid boxes on the floor.
    Returns (desc, emitter instances, box instances)."""
    rng = np.random.default_rng(seed)
    sc = SceneDesc(name="full")
    jit = lambda: rng.uniform(-0.02, 0.02, size=3)

    def albedo_material():
        return sc.add_material(material_words(tuple(rng.uniform(0.2, 0.8, size=3))))

    column = sc.add_mesh(cylinder_mesh(0.3, 6.0, 32, 16))
    arch = sc.add_mesh(arch_mesh(4.0, 0.4, 0.6, 60))
    tile = sc.add_mesh(box_mesh((0.98, 0.05, 0.98), bottom=False))
    emitter_mesh = sc.add_mesh(quad((-1.0, 0.0, -1.0), (1.0, 0.0, -1.0), (1.0, 0.0, 1.0), (-1.0, 0.0, 1.0)))
    box = sc.add_mesh(box_mesh((1.2, 1.2, 1.2), bottom=False))
    pitch, n, tiles = 4.0, 10, 40
    for i in range(n):
        for j in range(n):
            t = np.eye(3, 4, dtype=np.float64)
            t[:, 3] = ((i - (n - 1) / 2) * pitch, 0.0, (j - (n - 1) / 2) * pitch) + jit()
            sc.add_instance(column, t, material=albedo_material())
    for i in range(n - 1):
        for j in range(n):
            cx = (i + 0.5 - (n - 1) / 2) * pitch
            cz = (j - (n - 1) / 2) * pitch
            sc.add_instance(arch, rotation_y(0.0, (cx, 6.0, cz)) + _jit3(jit), material=albedo_material())
            sc.add_instance(arch, rotation_y(math.pi / 2, (cz, 6.0, cx)) + _jit3(jit), material=albedo_material())
    for i in range(tiles):
        for j in range(tiles):
            t = np.eye(3, 4, dtype=np.float64)
            t[:, 3] = (i - (tiles - 1) / 2, -0.05, j - (tiles - 1) / 2) + jit()
            sc.add_instance(tile, t, material=albedo_material())
    emitters = []
    for k in range(4):
        radiance = float(rng.uniform(5.0, 20.0))
        mat = sc.add_material(material_words((0.0, 0.0, 0.0), emission=(radiance, radiance, radiance)))
        t = np.eye(3, 4, dtype=np.float64)
        t[:, 3] = (rng.uniform(-12.0, 12.0), 9.5, rng.uniform(-12.0, 12.0))
        emitters.append(len(sc.instance_mesh))
        sc.add_instance(emitter_mesh, t, material=mat)
    boxes = []
    for k in range(8):
        boxes.append(len(sc.instance_mesh))
        sc.add_instance(box, rotation_y(float(rng.uniform(0, 2 * math.pi)),
                                        (float(rng.uniform(-16, 16)), 0.0, float(rng.uniform(-16, 16)))),
                        material=albedo_material())
    remaining = triangles - sc.world_triangles()
    if remaining < 2 or remaining % 2:
        raise ValueError(f"full scene triangle budget {triangles} cannot be met (remaining {remaining})")
    extent = pitch * n + 4.0
    ceiling = sc.add_mesh(grid_mesh(remaining // 2, extent, extent, 10.0, rng, 0.02))
    sc.add_instance(ceiling, material=albedo_material())
    assert sc.world_triangles() == triangles, (sc.world_triangles(), triangles)
    return sc, emitters, boxes


def emitter_orbits(desc: SceneDesc, emitters, seed: int = 5):
    """Seeded circular paths of the emitters at 0.5 m/s: (centre, radius,
    phase, direction) per emitter; the pose at time t is
    centre + radius (cos, 0, sin)(phase + direction 0.5 t / radius)."""
    rng = np.random.default_rng(seed + 1000)
    orbits = []
    for i in emitters:
        c = desc.instance_transform[i][:, 3].astype(np.float64)
        r = float(rng.uniform(2.0, 5.0))
        orbits.append((c, r, float(rng.uniform(0, 2 * math.pi)), 1.0 if rng.uniform() < 0.5 else -1.0))
    return orbits


def batch_scene(seed: int, triangles: int) -> SceneDesc:
    """One scene of the batched workload: a floor, 1-3 downward emitters
    (radiance U[5, 20]), seeded boxes and columns on the floor and a jittered
    ceiling grid that makes the world triangle count exactly ``triangles``
    (>= 200).  The room grows with the triangle count (about 6 m at 1k, 24 m
    at 200k)."""
    if triangles < 200:
        raise ValueError("batch scene needs at least 200 triangles")
    rng = np.random.default_rng(seed)
    sc = SceneDesc(name=f"batch{seed}")
    size = 6.0 + 18.0 * math.log(triangles / 1000.0 + 1.0) / math.log(201.0)
    height = 3.0 + 0.25 * size
    half = size * 0.5

    def albedo_material():
        return sc.add_material(material_words(tuple(rng.uniform(0.2, 0.8, size=3))))

    floor = sc.add_mesh(quad((-half, 0.0, -half), (-half, 0.0, half), (half, 0.0, half), (half, 0.0, -half)))
    sc.add_instance(floor, material=albedo_material())
    emitter = sc.add_mesh(quad((-0.5, 0.0, -0.5), (0.5, 0.0, -0.5), (0.5, 0.0, 0.5), (-0.5, 0.0, 0.5)))
    for _ in range(int(rng.integers(1, 4))):
        radiance = float(rng.uniform(5.0, 20.0))
        mat = sc.add_material(material_words((0.0, 0.0, 0.0), emission=(radiance, radiance, radiance)))
        t = np.eye(3, 4, dtype=np.float64)
        t[:, 3] = (rng.uniform(-0.3, 0.3) * size, height - 0.3, rng.uniform(-0.3, 0.3) * size)
        sc.add_instance(emitter, t, material=mat)
    budget = triangles - sc.world_triangles() - 2
    box = sc.add_mesh(box_mesh((1.0, 1.0, 1.0), bottom=False))  # 10 triangles
    column = sc.add_mesh(cylinder_mesh(0.25, 1.0, 12, 2))
    column_tris = len(sc.meshes[column].indices)
    spend = int(budget * 0.3)
    while spend >= column_tris:
        use_column = rng.uniform() < 0.4
        mesh, tris = (column, column_tris) if use_column else (box, 10)
        if tris > spend:
            break
        m = rotation_y(float(rng.uniform(0.0, 2.0 * math.pi)),
                       (float(rng.uniform(-0.45, 0.45) * size), 0.0, float(rng.uniform(-0.45, 0.45) * size)))
        m = m.astype(np.float64)
        m[:, :3] = m[:, :3] @ np.diag((rng.uniform(0.3, 1.5), rng.uniform(0.3, height * 0.6), rng.uniform(0.3, 1.5)))
        sc.add_instance(mesh, m.astype(np.float32), material=albedo_material())
        spend -= tris
    remaining = triangles - sc.world_triangles()
    if remaining % 2:
        sc.add_instance(sc.add_mesh(Mesh(np.array([[-half, 0.01, -half], [-half + 0.2, 0.01, -half],
                                                   [-half, 0.01, -half + 0.2]], np.float32),
                                         np.array([[0, 2, 1]], np.uint32))), material=albedo_material())
        remaining -= 1
    ceiling = sc.add_mesh(grid_mesh(remaining // 2, size, size, height, rng, 0.02))
    sc.add_instance(ceiling, material=albedo_material())
    assert sc.world_triangles() == triangles, (sc.world_triangles(), triangles)
    return sc


def batch_workload(seed: int = 3, scenes: int = 64):
    """The batched configuration: per scene (seed, triangle count log-uniform
    in [1k, 200k], view resolution from {320x180, 640x360, 1280x720})."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(scenes):
        tris = int(round(math.exp(rng.uniform(math.log(1000.0), math.log(200000.0)))))
        res = [(320, 180), (640, 360), (1280, 720)][int(rng.integers(0, 3))]
        out.append((seed * 1000 + k, tris, res))
    return out


def _jit3(jit):
    t = np.zeros((3, 4), dtype=np.float32)
    t[:, 3] = jit()
    return t


def dense_plane_probes(n: int = 64, spacing: float = 0.1, y_cell: int = 10):
    """Cascade-0 probe centres of an n x n horizontal grid (cell centres
    (k + 0.5) * spacing), as float4 positions and +y normals."""
    k = np.arange(n, dtype=np.int64) - n // 2
    kx, kz = np.meshgrid(k, k, indexing="ij")
    s = F32(spacing)
    pos = np.zeros((n * n, 4), dtype=np.float32)
    pos[:, 0] = (kx.ravel().astype(np.float32) + F32(0.5)) * s
    pos[:, 1] = (F32(y_cell) + F32(0.5)) * s
    pos[:, 2] = (kz.ravel().astype(np.float32) + F32(0.5)) * s
    nrm = np.zeros_like(pos)
    nrm[:, 1] = 1.0
    return pos, nrm


def camera_rays(width: int, height: int, eye, target, fov_y_deg: float = 60.0, stride: int = 1):
    """Primary rays through the centres of every `stride`-th pixel block."""
    eye = np.asarray(eye, dtype=np.float64)
    fwd = np.asarray(target, dtype=np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, (0.0, 1.0, 0.0))
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    tan = math.tan(math.radians(fov_y_deg) * 0.5)
    aspect = width / height
    xs = (np.arange(0, width, stride) + stride * 0.5) / width * 2.0 - 1.0
    ys = 1.0 - (np.arange(0, height, stride) + stride * 0.5) / height * 2.0
    gx, gy = np.meshgrid(xs, ys)
    d = fwd[None, None, :] + gx[..., None] * tan * aspect * right + gy[..., None] * tan * up
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    d = d.reshape(-1, 3).astype(np.float32)
    o = np.broadcast_to(eye.astype(np.float32), d.shape).copy()
    return o, d


def clip_from_world(eye, target, fov_y_deg: float, width: int, height: int, near: float = 0.05,
                    far: float = 1000.0) -> np.ndarray:
    """clip_from_world (row-major float32) of the look-at perspective camera
    camera_rays traces (view space -z forward, clip w = view depth)."""
    eye = np.asarray(eye, np.float64)
    fwd = np.asarray(target, np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, (0.0, 1.0, 0.0))
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    view = np.eye(4)
    view[0, :3], view[1, :3], view[2, :3] = right, up, -fwd
    view[:3, 3] = -view[:3, :3] @ eye
    t = math.tan(math.radians(fov_y_deg) * 0.5)
    proj = np.zeros((4, 4))
    proj[0, 0], proj[1, 1] = 1.0 / (t * width / height), 1.0 / t
    proj[2, 2], proj[2, 3] = -(far + near) / (far - near), -2.0 * far * near / (far - near)
    proj[3, 2] = -1.0
    return (proj @ view).astype(np.float32)
