"""Fixtures shared by the tests: scenes, the reference's traversal ray
families, and GPU buffer plumbing (torch is used for device memory only)."""
from __future__ import annotations

import math
from functools import lru_cache

import numpy as np

import bevy_penumbra_b200 as bp
from bevy_penumbra_b200 import scenes

EMPTY = 0xFFFFFFFF


def quat_xyz(a: float, b: float, c: float) -> np.ndarray:
    """Rotation matrix of Quat::from_euler(EulerRot::XYZ, a, b, c) = Rx(a) Ry(b) Rz(c)."""
    ca, sa, cb, sb, cc, sc = math.cos(a), math.sin(a), math.cos(b), math.sin(b), math.cos(c), math.sin(c)
    rx = np.array([[1, 0, 0], [0, ca, -sa], [0, sa, ca]])
    ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    rz = np.array([[cc, -sc, 0], [sc, cc, 0], [0, 0, 1]])
    return rx @ ry @ rz


def traversal_fixture() -> scenes.SceneDesc:
    """The 24-instance scene of gpu_traversal_matches_brute_force_through_motion_and_asset_edits
    (src/traversal_tests.rs:2067-2175): unit cubes and 2x2 panels, mixed cull
    modes, mirrored and extremely anisotropic instance scales."""
    sc = scenes.SceneDesc(name="traversal24")
    mat = sc.add_material(scenes.material_words((0.8, 0.6, 0.4), emission=(0.1, 0.2, 0.3)))
    cube = sc.add_mesh(scenes.Mesh(
        np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)], np.float32),
        np.array([[0, 1, 3], [0, 3, 2], [4, 6, 7], [4, 7, 5], [0, 4, 5], [0, 5, 1],
                  [2, 3, 7], [2, 7, 6], [0, 2, 6], [0, 6, 4], [1, 5, 7], [1, 7, 3]], np.uint32)))
    panel = sc.add_mesh(scenes.quad((-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0)))
    bare = sc.add_mesh(scenes.quad((-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0)))
    cull_flags = [8 | 16, 1, 2]  # None (double-sided, unlit), Back, Front
    for i in range(24):
        mesh = bare if i == 23 else (cube if i % 2 == 0 else panel)
        if i == 23:
            lin = np.eye(3)
            t = (-16.0, 0.0, -20.0)
        else:
            scale = (-0.001, 1000.0, 1.0) if i == 0 else ((-1.2 if i % 2 == 0 else 1.2), 0.6, 2.0)
            rot = np.eye(3) if i == 0 else quat_xyz(i * 0.03, i * 0.07, 0.2)
            lin = rot @ np.diag(scale)
            t = ((i % 6) * 4.0 - 10.0, (i // 6) * 5.0 - 7.5, 0.0)
        m = np.zeros((3, 4))
        m[:, :3] = lin
        m[:, 3] = t
        flags = cull_flags[i % 3] | (4 if np.linalg.det(lin) < 0 else 0)
        sc.add_instance(mesh, m.astype(np.float32), flags=flags, material=mat)
    return sc


@lru_cache(maxsize=None)
def packed(name: str) -> bp.PackedScene:
    if name == "cornell":
        return bp.PackedScene.from_desc(scenes.cornell())
    if name == "traversal24":
        return bp.PackedScene.from_desc(traversal_fixture())
    if name.startswith("atrium"):
        tris = int(name[len("atrium"):] or 262144)
        return bp.PackedScene.from_desc(scenes.atrium(triangles=tris))
    raise KeyError(name)


def scene_desc(name: str) -> scenes.SceneDesc:
    if name == "cornell":
        return scenes.cornell()
    if name == "traversal24":
        return traversal_fixture()
    if name.startswith("atrium"):
        return scenes.atrium(triangles=int(name[len("atrium"):] or 262144))
    raise KeyError(name)


def _normalize(v):
    v = np.asarray(v, dtype=np.float32)
    return (v / np.float32(np.sqrt(np.sum(v * v)))).astype(np.float32)


def rays_for(desc: scenes.SceneDesc) -> np.ndarray:
    """rays_for, src/traversal_tests.rs:1040-1125: targeted rays at triangle
    centres / longest-edge midpoints / vertices from +-{0.01, 1, 100} along
    the normal, 4096 LCG rays (seed 7) in a 100 m cube with limit 200, and
    exact axis-parallel rays through every instance's bounds centre.  The
    any-hit copies are returned by the caller with any_hit set."""
    rays = []
    for inst, mesh_id in enumerate(desc.instance_mesh):
        mesh = desc.meshes[mesh_id]
        m = desc.instance_transform[inst].astype(np.float64)
        lin = m[:, :3]
        identity = np.allclose(lin, np.eye(3))
        for tri in mesh.indices[:12]:
            local = mesh.positions[tri].astype(np.float64)
            world = (local @ lin.T + m[:, 3]).astype(np.float32)
            a, b, c = world
            n = np.cross(b - a, c - a)
            n = _normalize(n)
            center = ((a + b + c) / np.float32(3.0)).astype(np.float32)
            edges = [(local[0], local[1]), (local[1], local[2]), (local[2], local[0])]
            s, e = max(edges, key=lambda p: float(np.sum((p[1] - p[0]) ** 2)))
            mid = ((s + e) * 0.5 @ lin.T + m[:, 3]).astype(np.float32)
            targets = [center, mid, a] if identity else [center, mid]
            for target in targets:
                for sign in (-1.0, 1.0):
                    for dist in (0.01, 1.0, 100.0):
                        origin = (target + n * np.float32(sign * dist)).astype(np.float32)
                        d = target - origin
                        ln = np.sqrt(np.sum(d.astype(np.float64) ** 2))
                        if ln > 0 and np.all(np.isfinite(d)):
                            rays.append((origin, (d / ln).astype(np.float32), np.float32(dist * 1.1)))
    state = 7

    def rnd():
        nonlocal state
        state = (state * 1664525 + 1013904223) & 0xFFFFFFFF
        return np.float32((state >> 8) / 16777216.0)

    for _ in range(4096):
        o = (np.array([rnd(), rnd(), rnd()], np.float32) * np.float32(100.0) - np.float32(50.0)).astype(np.float32)
        d = (np.array([rnd(), rnd(), rnd()], np.float32) * np.float32(2.0) - np.float32(1.0)).astype(np.float32)
        rays.append((o, _normalize(d), np.float32(200.0)))
    for inst, mesh_id in enumerate(desc.instance_mesh):
        mesh = desc.meshes[mesh_id]
        m = desc.instance_transform[inst].astype(np.float64)
        world = mesh.positions.astype(np.float64) @ m[:, :3].T + m[:, 3]
        center = ((world.min(0) + world.max(0)) * 0.5).astype(np.float32)
        for d in np.vstack([np.eye(3), -np.eye(3)]).astype(np.float32):
            rays.append(((center - d * np.float32(100.0)).astype(np.float32), d, np.float32(200.0)))
    out = np.zeros(len(rays), dtype=bp.RAY_DTYPE)
    for i, (o, d, lim) in enumerate(rays):
        out[i]["origin"] = o
        out[i]["direction"] = d
        out[i]["limit"] = lim
    return out


def check_against_f64(oscene, rays, hits, any_hit: bool, expected_errors: int = 0):
    """check_gpu_for_layers acceptance (src/traversal_tests.rs:1432-1519):
    |t - t_ref| <= 2e-4 max(1, |t|) and (triangle, instance) among the f64
    candidates within tolerance.  Returns (failures, hit count)."""
    failures = []
    count = 0
    for i in range(len(rays)):
        t, tri, inst = oscene.brute_f64(rays[i]["origin"], rays[i]["direction"], rays[i]["limit"])
        h = hits[i]
        hit = int(h["triangle"]) != EMPTY
        if (int(h["errors"]) & ~expected_errors) != 0:
            failures.append((i, "errors", int(h["errors"])))
            continue
        if not hit:
            if len(t):
                failures.append((i, "missed", float(t[0])))
            continue
        count += 1
        dist = float(h["distance"])
        if any_hit:
            tol = 2e-4 * max(1.0, abs(dist))
            ok = len(t) > 0
            if not ok:
                failures.append((i, "any-hit without candidate"))
            continue
        if not len(t):
            failures.append((i, "spurious hit", dist))
            continue
        tol = 2e-4 * max(1.0, abs(dist))
        ok = abs(dist - t[0]) <= tol and any(
            abs(c - t[0]) <= tol and int(a) == int(h["triangle"]) and int(b) == int(h["instance"])
            for c, a, b in zip(t, tri, inst))
        if not ok:
            failures.append((i, "closest", dist, int(h["triangle"]), int(h["instance"]), float(t[0])))
    return failures, count


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def to_device(arr: np.ndarray):
    import torch
    a = np.ascontiguousarray(arr)
    t = torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).cuda()
    torch.cuda.synchronize()  # the library's stream does not order after torch's
    return t


def from_device(t, dtype, shape) -> np.ndarray:
    return t.cpu().numpy().view(dtype).reshape(shape)


def empty_device(nbytes: int):
    import torch
    t = torch.zeros(max(nbytes, 16), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()  # the fill must land before the library writes
    return t


def cornell_dense_settings(**kw) -> bp.RadianceCascades:
    """The Cornell cascade configuration: 64 x 64 probes at 0.1 m, 4 levels,
    16 directions at cascade 0 (4 x 4) growing x4, interval lengths doubling
    from 0.05 m."""
    base = dict(probe_spacing=0.1, interval_length=0.05, levels=4, base_columns=4, base_rows=4,
                interval_ratio=2.0, interval_rule=bp.INTERVAL_LENGTHS_GEOMETRIC, layout=bp.LAYOUT_DENSE,
                emissive_samples=16, normal_bias=0.005)
    base.update(kw)
    return bp.RadianceCascades(**base).sanitized()


def camera_clip(eye, target, fov_y_deg: float, width: int, height: int):
    """scenes.clip_from_world and the camera basis of scenes.camera_rays."""
    from bevy_penumbra_b200 import scenes
    eye = np.asarray(eye, np.float64)
    fwd = np.asarray(target, np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, (0.0, 1.0, 0.0))
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    t = np.tan(np.radians(fov_y_deg) * 0.5)
    return scenes.clip_from_world(eye, target, fov_y_deg, width, height, far=100.0), (fwd, right, up, t,
                                                                                     width / height)


def synthetic_screen(width: int, height: int, eye, target, seed: int = 0, fov_y_deg: float = 60.0):
    """An analytic G-buffer for the screen filter: a floor (identity 1), a box
    (identity 2) and a back wall (identity 3) seen through a pinhole camera;
    irradiance is a smooth field plus seeded noise with rawGiSupportAlpha
    (1 + 0.25 coverage; -1 unsupported; 0 without a surface).  Returns
    (irradiance, position (w = view depth), normal, identity, clip_from_world)."""
    clip, (fwd, right, up, t, aspect) = camera_clip(eye, target, fov_y_deg, width, height)
    eye = np.asarray(eye, np.float64)
    xs = (np.arange(width) + 0.5) / width * 2.0 - 1.0
    ys = 1.0 - (np.arange(height) + 0.5) / height * 2.0
    gx, gy = np.meshgrid(xs, ys)
    d = fwd + gx[..., None] * (t * aspect) * right + gy[..., None] * t * up
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    best = np.full((height, width), np.inf)
    nrm = np.zeros((height, width, 3))
    ident = np.zeros((height, width), np.uint32)
    with np.errstate(divide="ignore", invalid="ignore"):
        tf = -eye[1] / d[..., 1]  # floor y = 0
        hit = (tf > 1e-4) & (tf < best)
        best[hit], nrm[hit], ident[hit] = tf[hit], (0.0, 1.0, 0.0), 1
        tw = (-2.0 - eye[2]) / d[..., 2]  # back wall z = -2
        hit = (tw > 1e-4) & (tw < best)
        best[hit], nrm[hit], ident[hit] = tw[hit], (0.0, 0.0, 1.0), 3
        lo, hi = np.array([-0.4, 0.0, -0.4]), np.array([0.4, 0.8, 0.4])
        t0 = (lo - eye) / d
        t1 = (hi - eye) / d
        tn, tx = np.minimum(t0, t1), np.maximum(t0, t1)
        near, far = tn.max(-1), tx.min(-1)
        axis = tn.argmax(-1)
        hit = (near <= far) & (near > 1e-4) & (near < best)
        face = np.zeros((height, width, 3))
        np.put_along_axis(face, axis[..., None], 1.0, axis=-1)
        sign = -np.sign(np.take_along_axis(d, axis[..., None], -1))
        best[hit], nrm[hit], ident[hit] = near[hit], (face * sign)[hit], 2
    ok = np.isfinite(best)
    p = eye + d * np.where(ok, best, 0.0)[..., None]
    rng = np.random.default_rng(seed)
    field = 0.5 + 0.3 * np.sin(3.0 * p[..., 0]) * np.cos(2.0 * p[..., 2]) + 0.2 * p[..., 1] + 0.1 * ident
    noise = 1.0 + 0.1 * rng.standard_normal((height, width, 3))
    irr = np.zeros((height, width, 4), np.float32)
    irr[..., :3] = field[..., None] * noise * np.array([1.0, 0.9, 0.8])
    u = rng.random((height, width))
    coverage = np.where(u < 0.6, 1.0, rng.uniform(0.2, 1.0, (height, width)))
    irr[..., 3] = np.where(u > 0.9, -1.0, 1.0 + 0.25 * coverage)
    irr[~ok] = 0.0
    pos = np.zeros((height, width, 4), np.float32)
    pos[..., :3] = p
    pos[..., 3] = np.where(ok, best * (d @ fwd), 0.0)
    pos[~ok, :3] = 0.0
    normal = np.zeros((height, width, 4), np.float32)
    normal[..., :3] = nrm
    identity = np.zeros((height, width, 2), np.uint32)
    identity[..., 0] = ident
    return irr, pos, normal, identity, clip
