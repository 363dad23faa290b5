"""CPU oracle of bevy_lux's Split transport path (test infrastructure only).

Loaded by the tests, the smoke check and the CPU-baseline leg of bench.py as
the parity checker; the product (bevy_penumbra_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liblux_oracle.so")


def build(force: bool = False) -> str:
    sources = [os.path.join(HERE, n) for n in ("lux_oracle.c", "orc_pack.c", "lux_oracle.h")]
    if force or not os.path.exists(LIB) or max(os.path.getmtime(s) for s in sources) > os.path.getmtime(LIB):
        subprocess.run(["make", "-s", "-C", HERE, "-B" if force else "liblux_oracle.so"], check=True)
    return LIB


class Counters(C.Structure):
    _fields_ = [("nodes", C.c_uint64), ("triangles", C.c_uint64), ("instances", C.c_uint64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        h = C.CDLL(LIB)
        P = C.c_void_p
        U = C.c_uint32
        F = C.c_float
        sig = {
            "orc_sincos_turns": (None, [F, P, P]),
            "orc_decode_direction": (None, [F, F, P]),
            "orc_bin_direction": (None, [U, U, U, P]),
            "orc_direction_index_uv": (U, [F, F, U, U]),
            "orc_r2": (None, [U, P]),
            "orc_transport_hash": (U, [U]),
            "orc_hash_key": (U, [P, U]),
            "orc_ray_offset": (None, [P, P, F, P]),
            "orc_encode_normal": (None, [P, P]),
            "orc_decode_normal": (None, [P, P]),
            "orc_interval_end": (F, [P, U]),
            "orc_spacing": (F, [P, U]),
            "orc_scene_create": (P, [P, C.c_size_t, P, C.c_size_t, P, U, U]),
            "orc_scene_destroy": (None, [P]),
            "orc_scene_refit": (C.c_int, [P, P, C.c_uint32]),
            "orc_reference_irradiance": (None, [P, P, P, P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, P]),
            "orc_scene_words": (None, [P, P]),
            "orc_trace_closest": (None, [P, P, P, F, F, P, P]),
            "orc_trace_occluded": (C.c_int, [P, P, P, F, P, P]),
            "orc_brute_closest": (None, [P, P, P, F, F, P]),
            "orc_brute_f64": (U, [P, P, P, F, P, P, P, U]),
            "orc_trace_rays": (None, [P, P, U, C.c_int, P, C.c_int, P]),
            "orc_outgoing_radiance": (C.c_int, [P, P, P, P, P, P, P, P]),
            "orc_frame_run": (P, [P, P, P, P, U, C.c_int]),
            "orc_frame_run_history": (P, [P, P, P, P, U, C.c_int, P, P, U]),
            "orc_frame_run_retain": (P, [P, P, P, P, U, C.c_int, P, P, U, U, C.c_uint64]),
            "orc_frame_run_bounce": (P, [P, P, P, P, U, C.c_int, P, P, U, U, C.c_uint64, P, U, P, P, P]),
            "orc_lod_blend": (None, [P, P, P, P, P, P]),
            "orc_transport_random": (F, [U, U]),
            "orc_sequence_order": (None, [P, P, P, U, C.c_int, P]),
            "orc_cosine_direction_frame": (None, [P, F, F, P]),
            "orc_environment_response": (C.c_int, [P, P, F, F, U, U, P, P, P, P, F, P, C.c_int, P, P, P]),
            "orc_screen_filter": (None, [P, U, U, P, P, P, P, P, P, U, U, U, P, P, P]),
            "orc_history_blend": (None, [P, U, P, P, P, P, P]),
            "orc_merge_history_entry": (None, [P, P, U, P, P, P, P, C.c_int, P]),
            "orc_frame_destroy": (None, [P]),
            "orc_frame_cells": (U, [P, U]),
            "orc_scene_pack": (C.c_int, [P, U, P, U, P, P, U, P, P, P, P, U, P, U, P]),
            "orc_path_random": (F, [U, U, U, U]),
            "orc_cosine_direction": (None, [P, F, F, P]),
            "orc_path_sample": (C.c_int, [P, P, U, U, U, P, P, U, P]),
            "orc_path_reference": (None, [P, P, P, P, U, U, U, U, C.c_int, P]),
            "orc_packed_sizes": (None, [P, P, P, P, P, P, P, P]),
            "orc_packed_copy": (None, [P, P, P, P, P, U]),
            "orc_packed_destroy": (None, [P]),
            "orc_frame_read_hits": (C.c_uint64, [P, P, C.c_uint64]),
            "orc_frame_read_level": (None, [P, U, P, P, P, P]),
            "orc_frame_read_probes": (None, [P, P]),
            "orc_frame_stats": (None, [P, P]),
            "orc_frame_resolve": (None, [P, P, P, U, P]),
            "orc_resolve_tables": (None, [P, U, P, F, P, P, U, P]),
            "orc_deposit_levels": (U, [P, F, C.c_int, C.c_int, P, P]),
            "orc_merge_entry": (None, [P, U, P, P, C.c_int, P]),
            "orc_interpolate_children": (None, [P, P, P]),
            "orc_pack_table": (None, [P, U, U, P]),
            "orc_probe_lookup": (None, [P, P, P]),
            "orc_dense_sdf_record": (None, [U, P, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib


# LuxHit (include/lux.h) as a numpy record.
HIT_DTYPE = np.dtype([("distance", "<f4"), ("triangle", "<u4"), ("instance", "<u4"), ("errors", "<u4"),
                      ("barycentric", "<f4", (3,)), ("visited", "<u4")])


def _p(a: np.ndarray) -> int:
    return a.ctypes.data if a is not None and a.size else 0


def f32(*v) -> np.ndarray:
    return np.ascontiguousarray(np.array(v, dtype=np.float32).ravel())


class OraclePacked:
    """The oracle packer's word streams (orc_scene_pack): the attributes of
    bevy_penumbra_b200.PackedScene, built without liblux."""

    def __init__(self, positions, indices, mesh_first, mesh_count, instance_mesh, instance_transform,
                 instance_flags, instance_material, materials):
        a = lambda x, t: np.ascontiguousarray(x, dtype=t)
        positions = a(positions, np.float32).reshape(-1, 3)
        indices = a(indices, np.uint32).reshape(-1, 3)
        mesh_first, mesh_count = a(mesh_first, np.uint32), a(mesh_count, np.uint32)
        imesh, iflags, imat = a(instance_mesh, np.uint32), a(instance_flags, np.uint32), a(instance_material, np.uint32)
        ixf = a(instance_transform, np.float32).reshape(-1, 12)
        mats = a(materials, np.uint32).reshape(-1, 32)
        handle = C.c_void_p()
        rc = lib().orc_scene_pack(_p(positions), len(positions), _p(indices), len(indices), _p(mesh_first),
                                  _p(mesh_count), len(mesh_first), _p(imesh), _p(ixf), _p(iflags), _p(imat),
                                  len(imesh), _p(mats), len(mats), C.byref(handle))
        if rc != 0:
            raise ValueError("oracle packer: invalid scene")
        try:
            sw, gw = C.c_size_t(), C.c_size_t()
            nl, tn, bn, depth = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
            cost = C.c_double()
            lib().orc_packed_sizes(handle, C.byref(sw), C.byref(gw), C.byref(nl), C.byref(tn), C.byref(bn),
                                   C.byref(depth), C.byref(cost))
            self.scene_words = np.zeros((sw.value, 4), np.uint32)
            self.geometry_words = np.zeros((gw.value, 4), np.uint32)
            self.lights = np.zeros((nl.value, 24), np.uint32)
            self.instance_order = np.zeros(len(imesh), np.uint32)
            lib().orc_packed_copy(handle, _p(self.scene_words), _p(self.geometry_words), _p(self.lights),
                                  _p(self.instance_order), len(imesh))
        finally:
            lib().orc_packed_destroy(handle)
        self.tlas_nodes, self.blas_nodes = tn.value, bn.value
        self.max_depth, self.blas_cost = depth.value, cost.value
        self.conventional = 0

    @staticmethod
    def from_desc(desc) -> "OraclePacked":
        """A scene description of bevy_penumbra_b200.scenes (pure numpy)."""
        positions, indices, first, count = desc.arrays()
        return OraclePacked(positions, indices, first, count, desc.instance_mesh, np.stack(desc.instance_transform),
                            desc.instance_flags, desc.instance_material, np.stack(desc.materials))


class OracleScene:
    """Oracle view of the reference word streams."""

    def __init__(self, scene_words: np.ndarray, geometry_words: np.ndarray, lights: np.ndarray,
                 conventional: int = 0):
        self._keep = (np.ascontiguousarray(scene_words, np.uint32), np.ascontiguousarray(geometry_words, np.uint32),
                      np.ascontiguousarray(lights, np.uint32))
        sw, gw, lt = self._keep
        self.handle = lib().orc_scene_create(_p(sw), sw.size // 4, _p(gw), gw.size // 4, _p(lt), lt.size // 24,
                                             conventional)

    @staticmethod
    def from_packed(packed) -> "OracleScene":
        return OracleScene(packed.scene_words, packed.geometry_words, packed.lights,
                           getattr(packed, "conventional", 0))

    def trace_rays(self, rays: np.ndarray, any_hit: bool = False, threads: int = 0):
        """rays: structured RAY_DTYPE array -> HIT_DTYPE array, counters."""
        rays = np.ascontiguousarray(rays)
        hits = np.zeros(len(rays), dtype=HIT_DTYPE)
        cn = Counters()
        lib().orc_trace_rays(self.handle, _p(rays), len(rays), 1 if any_hit else 0, _p(hits),
                             threads or os.cpu_count() or 1, C.byref(cn))
        return hits, cn

    def brute_f64(self, origin, direction, limit, capacity: int = 64):
        t = np.zeros(capacity, np.float64)
        tri = np.zeros(capacity, np.uint32)
        inst = np.zeros(capacity, np.uint32)
        o = f32(*origin)
        d = f32(*direction)
        n = lib().orc_brute_f64(self.handle, _p(o), _p(d), float(limit), _p(t), _p(tri), _p(inst), capacity)
        n = min(int(n), capacity)
        return t[:n], tri[:n], inst[:n]

    def refit(self, world_from_local) -> None:
        """Pose update + TLAS refit (float[instances, 3, 4], slot order)."""
        m = np.ascontiguousarray(world_from_local, dtype=np.float32).reshape(-1, 12)
        rc = lib().orc_scene_refit(self.handle, _p(m), len(m))
        if rc != 0:
            raise ValueError("oracle refit: instance count mismatch or singular transform")

    def reference_irradiance(self, settings_c, position, normal, spp: int, seed: int, round_samples: int):
        """FP64 reference irradiance (double[count, 4]) at float4 points / normals."""
        pos = np.ascontiguousarray(position, np.float32)
        nrm = np.ascontiguousarray(normal, np.float32)
        out = np.zeros((len(pos), 4), np.float64)
        lib().orc_reference_irradiance(self.handle, C.byref(settings_c), _p(pos), _p(nrm), len(pos), spp, seed,
                                       round_samples, _p(out))
        return out

    def path_reference(self, settings_c, position, normal, spp: int, bounces: int, seed: int, threads: int = 0):
        """Path-traced reference (double[count, 4]: mean rgb, supported samples)."""
        pos = np.ascontiguousarray(position, np.float32)
        nrm = np.ascontiguousarray(normal, np.float32)
        out = np.zeros((len(pos), 4), np.float64)
        lib().orc_path_reference(self.handle, C.byref(settings_c), _p(pos), _p(nrm), len(pos), spp, bounces, seed,
                                 threads or os.cpu_count() or 1, _p(out))
        return out

    def path_sample(self, settings_c, position, normal, bounces: int, seed: int, p: int, s: int):
        """One path's radiance (rgb), or None when a trace was unsupported."""
        pos = np.ascontiguousarray(position, np.float32).reshape(-1)[:3].copy()
        nrm = np.ascontiguousarray(normal, np.float32).reshape(-1)[:3].copy()
        out = np.zeros(3, np.float32)
        ok = lib().orc_path_sample(self.handle, C.byref(settings_c), bounces, seed, p, _p(pos), _p(nrm), s, _p(out))
        return out if ok else None

    def words(self) -> np.ndarray:
        out = np.zeros(self._keep[0].shape, dtype=np.uint32).reshape(-1, 4)
        lib().orc_scene_words(self.handle, _p(out))
        return out

    def close(self):
        if self.handle:
            lib().orc_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OracleFrame:
    def __init__(self, scene: OracleScene, settings_c, pos: np.ndarray, nrm: np.ndarray, threads: int = 0,
                 previous: "OracleFrame | None" = None, dirty=None, max_cells: int = 0xFFFFFFFF,
                 max_entries: int = (1 << 64) - 1, feedback: "OracleFrame | None" = None, sparse: bool = False,
                 skip_emission: bool = False, record_hits: bool = False, camera=None, cached_sky: bool = False):
        """previous: the frame whose records serve as history; dirty: boxes
        (n, 6) = (lo xyz, hi xyz) whose nearby records take no history;
        max_cells / max_entries: the view capacities that bound the cells
        retained from `previous`.  Multi-bounce: feedback, the secondary frame
        whose cascade-0 probes add bounce light at hits; sparse, receivers
        with position.w == 0 are absent; skip_emission, hits add no emission of
        their own; record_hits, keep each receiver's hit surface (hits());
        cached_sky, cachedHitSky (escapes of a skip_emission frame carry the
        environment, hits the feedback frame covers take no sky samples).
        camera: a LuxCamera (bevy_penumbra_b200.camera_struct) for distance
        LODs, as SplitView.set_camera."""
        self.settings = settings_c
        pos = np.ascontiguousarray(pos, np.float32)
        nrm = np.ascontiguousarray(nrm, np.float32)
        self._previous = previous  # keeps the history frame alive
        boxes = np.ascontiguousarray(dirty if dirty is not None else np.zeros((0, 6)), np.float32).reshape(-1, 6)
        self._feedback = feedback
        self._camera = camera
        self.hit_pos = np.zeros((len(pos), 4), np.float32)
        self.hit_nrm = np.zeros((len(pos), 4), np.float32)
        flags = (1 if sparse else 0) | (2 if skip_emission else 0) | (4 if record_hits else 0) | \
            (8 if cached_sky else 0)
        self.handle = lib().orc_frame_run_bounce(scene.handle, C.byref(settings_c), _p(pos), _p(nrm), len(pos),
                                                 threads or os.cpu_count() or 1,
                                                 previous.handle if previous is not None else None, _p(boxes),
                                                 len(boxes), max_cells, max_entries,
                                                 feedback.handle if feedback is not None else None, flags,
                                                 _p(self.hit_pos), _p(self.hit_nrm),
                                                 C.addressof(camera) if camera is not None else None)

    def level(self, level: int, dirs: int):
        cells = lib().orc_frame_cells(self.handle, level)
        keys = np.zeros((cells, 4), np.int32)
        merged = np.zeros((cells, dirs, 4), np.float32)
        raw = np.zeros((cells, dirs, 4), np.float32)
        samples = np.zeros((cells, dirs), np.uint32)
        if cells:
            lib().orc_frame_read_level(self.handle, level, _p(keys), _p(merged), _p(raw), _p(samples))
        return keys, merged, raw, samples

    def hits(self, count: int) -> np.ndarray:
        """Closest hits of the frame's interval rays (Split layout), as the
        LuxHit records of lux_view_read_hits."""
        out = np.zeros(count, dtype=HIT_DTYPE)
        n = lib().orc_frame_read_hits(self.handle, _p(out), count)
        return out[:n]

    def probes(self):
        cells = lib().orc_frame_cells(self.handle, 0)
        tables = np.zeros((cells, 36, 4), np.float32)
        if cells:
            lib().orc_frame_read_probes(self.handle, _p(tables))
        return tables

    def stats(self):
        from bevy_penumbra_b200._native import LuxStats
        st = LuxStats()
        lib().orc_frame_stats(self.handle, C.byref(st))
        return st

    def resolve(self, pos: np.ndarray, nrm: np.ndarray) -> np.ndarray:
        pos = np.ascontiguousarray(pos, np.float32)
        nrm = np.ascontiguousarray(nrm, np.float32)
        out = np.zeros((len(pos), 4), np.float32)
        lib().orc_frame_resolve(self.handle, _p(pos), _p(nrm), len(pos), _p(out))
        return out

    def close(self):
        if self.handle:
            lib().orc_frame_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def lod_blend(settings_c, camera, position):
    """splitLodBlendForParameters of one point: (low, high, blend)."""
    low, high, blend = C.c_uint32(), C.c_uint32(), C.c_float()
    p = f32(*position)
    lib().orc_lod_blend(C.byref(settings_c), C.byref(camera) if camera is not None else None, _p(p), C.byref(low),
                        C.byref(high), C.byref(blend))
    return int(low.value), int(high.value), float(blend.value)


def sequence_order(settings_c, pos, sparse=False, camera=None):
    """Each Split receiver's place in the sample sequence (uint32[n])."""
    pos = np.ascontiguousarray(pos, np.float32)
    out = np.zeros(len(pos), np.uint32)
    lib().orc_sequence_order(C.byref(settings_c), C.byref(camera) if camera is not None else None, _p(pos),
                             len(pos), 1 if sparse else 0, _p(out))
    return out


def transport_random(seed, lane):
    """transportRandom (shaders/common.slang:292-295)."""
    return float(lib().orc_transport_random(seed & 0xFFFFFFFF, lane & 0xFFFFFFFF))


def cosine_direction_frame(normal, u1, u2):
    """cosineDirection (shaders/common.slang:407-412) of a unit normal."""
    out = np.zeros(3, np.float32)
    n = f32(*normal)
    lib().orc_cosine_direction_frame(_p(n), u1, u2, _p(out))
    return out


def environment_irradiance(environment, position, normal, roughness, count, sequence_base, visibility=0,
                           probe_spacing=1.0, bias=0.001, geometric_normal=None, view=None, diffuse=(1.0, 1.0, 1.0)):
    """environmentIrradiance (shaders/environment.slang:242-249) of a constant
    environment with every visibility query stubbed (0 visible, 1 blocked,
    2 unsupported): (rgb float32[3], supported)."""
    out = np.zeros(3, np.float32)
    env, p, n, dif = f32(*environment), f32(*position), f32(*normal), f32(*diffuse)
    g = n if geometric_normal is None else f32(*geometric_normal)
    v = n if view is None else f32(*view)
    ok = lib().orc_environment_response(None, _p(env), probe_spacing, bias, count, sequence_base, _p(p), _p(n),
                                        _p(g), _p(v), roughness, _p(dif), visibility, _p(out), None, None)
    return out, bool(ok)


SCREEN_WORDS = 18


def screen_filter(settings_c, irradiance, position, normal, identity, previous_clip_from_world, history=None,
                  dirty=None, scene_changed=False, spatial_filter_steps=3):
    """The screen temporal + denoise passes on (h, w, 4) float32 images and an
    (h, w, 2) uint32 identity image; history: the previous call's history
    (None: no screen history).  Returns (history, out (h, w, 4))."""
    h, w = irradiance.shape[:2]
    irradiance = np.ascontiguousarray(irradiance, np.float32)
    position = np.ascontiguousarray(position, np.float32)
    normal = np.ascontiguousarray(normal, np.float32)
    identity = np.ascontiguousarray(identity, np.uint32)
    prev = np.ascontiguousarray(previous_clip_from_world, np.float32).reshape(16)
    hin = np.zeros((h, w, SCREEN_WORDS), np.float32) if history is None else np.ascontiguousarray(history)
    hout = np.zeros((h, w, SCREEN_WORDS), np.float32)
    out = np.zeros((h, w, 4), np.float32)
    d = None if dirty is None else np.ascontiguousarray(dirty, np.float32).reshape(6)
    lib().orc_screen_filter(C.byref(settings_c), w, h, _p(irradiance), _p(position), _p(normal), _p(identity),
                            _p(prev), _p(d) if d is not None else None, 1 if scene_changed else 0,
                            spatial_filter_steps, 0 if history is None else 1, _p(hin), _p(hout), _p(out))
    return hout, out


def merge_history_entry(settings_c, interval, samples: int, old, old_mass, fraction, children4x8):
    """mergeEntry with history of one entry: the merged float4."""
    out = np.zeros(4, np.float32)
    o = f32(*old) if old is not None else None
    om = f32(*old_mass) if old_mass is not None else None
    ch = np.ascontiguousarray(children4x8, np.float32)
    lib().orc_merge_history_entry(C.byref(settings_c), _p(f32(*interval)), samples,
                                  _p(o) if o is not None else None, _p(om) if om is not None else None,
                                  _p(f32(*fraction)), _p(ch), 1, _p(out))
    return out


def history_blend(settings_c, samples: int, fresh, old=None, old_mass=None):
    """mergeEntry's history blend of one record: (J rgb, beta), (radiance mass, transmittance mass)."""
    fresh = f32(*fresh)
    out = np.zeros(4, np.float32)
    mass = np.zeros(2, np.float32)
    o = f32(*old) if old is not None else None
    om = f32(*old_mass) if old_mass is not None else None
    lib().orc_history_blend(C.byref(settings_c), samples, _p(fresh), _p(o) if o is not None else None,
                            _p(om) if om is not None else None, _p(out), _p(mass))
    return out, mass
