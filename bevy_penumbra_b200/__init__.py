"""bevy_penumbra_b200 - B200 Split Radiance Cascades transport for bevy_lux.

Host-side mirror of the reference's settings surface and plugin
(``RadianceCascades``, ``SamplingSettings``, ``RadianceCascadesPlugin``,
src/lib.rs:343-900) over the C ABI of liblux.so (include/lux.h).  Every
compute call goes to the sm_100a kernels of liblux; nothing here computes
transport on the host.

Typical frame (render(), src/render.rs:9124-9830):

    plugin = RadianceCascadesPlugin()
    ctx = plugin.build()                       # device context
    packed = PackedScene.from_desc(scenes.cornell())
    scene = GpuScene(ctx, packed)               # lux_scene_upload
    view = SplitView(ctx, max_receivers=4096, max_cells=8192, max_entries=1 << 22)
    view.trace_merge(scene, settings, receivers_pos, receivers_nrm)
    irradiance = view.resolve(settings, points_pos, points_nrm)
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field, replace

import numpy as np

from . import _native as N
from ._native import LuxError, check, lib

__all__ = [
    "SamplingSettings", "RadianceCascades", "RadianceCascadesPlugin", "RadianceCascadesStatus",
    "LuxContext", "PackedScene", "GpuScene", "SplitView", "Batch", "LuxError", "trace_rays", "interval_radiance", "reference_irradiance", "error_stats", "measure_read_rate", "LearnedCache", "CACHE_SAMPLE_DTYPE",
    "LAYOUT_SPLIT", "LAYOUT_DENSE", "INTERVAL_ENDS_GEOMETRIC", "INTERVAL_LENGTHS_GEOMETRIC",
]

LAYOUT_SPLIT = N.LUX_LAYOUT_SPLIT
LAYOUT_DENSE = N.LUX_LAYOUT_DENSE
INTERVAL_ENDS_GEOMETRIC = N.LUX_INTERVAL_ENDS_GEOMETRIC
INTERVAL_LENGTHS_GEOMETRIC = N.LUX_INTERVAL_LENGTHS_GEOMETRIC


@dataclass
class SamplingSettings:
    """SamplingSettings (src/lib.rs:343-413); this path reads resolve_scale."""
    grid_divisor: int = 0
    max_receiver_cells: int = 0
    max_updates_per_frame: int = 0
    max_cache_entries: int = 0
    max_traversal_queries: int = 0
    resolve_scale: int = 1

    @staticmethod
    def unlimited() -> "SamplingSettings":
        return SamplingSettings()

    @staticmethod
    def low_end() -> "SamplingSettings":
        return SamplingSettings(8, 16_384, 1_024, 16_384, 16_384, 2)

    def sanitized(self) -> "SamplingSettings":
        def clamp(v, lo, hi):
            return v if v == 0 else min(max(v, lo), hi)
        return SamplingSettings(
            clamp(self.grid_divisor, 1, 256), clamp(self.max_receiver_cells, 1, 131_072),
            clamp(self.max_updates_per_frame, 1, 131_072), clamp(self.max_cache_entries, 1, 262_144),
            clamp(self.max_traversal_queries, 1, 131_072), min(max(self.resolve_scale, 1), 8))


@dataclass
class RadianceCascades:
    """Per-camera settings (RadianceCascades, src/lib.rs:431-518) plus the
    cascade-shape extensions the reference hard-codes (levels, base direction
    grid, interval growth) and the probe layout."""
    probe_spacing: float = 0.25
    interval_length: float = 0.4
    normal_bias: float = 0.005
    intensity: float = 1.0
    environment: tuple = (0.0, 0.0, 0.0)
    emissive_samples: int = 16
    sampling: SamplingSettings = field(default_factory=SamplingSettings)
    exposure: float = 1.0
    levels: int = 4
    base_columns: int = 8
    base_rows: int = 4
    interval_ratio: float = 4.0
    interval_rule: int = INTERVAL_ENDS_GEOMETRIC
    layout: int = LAYOUT_SPLIT
    rays_per_receiver: int = 1
    frame_index: int = 0
    temporal_blend: float = 0.88
    split_transmittance_blend: float = 0.98
    history_frames: int = 24
    multi_bounce: bool = False
    cached_hit_sky: bool = False

    @staticmethod
    def low_end() -> "RadianceCascades":
        """RadianceCascades::low_end() (src/lib.rs:700-722), the fields this path reads."""
        return RadianceCascades(probe_spacing=1.0, interval_length=1.6, emissive_samples=4,
                                sampling=SamplingSettings.low_end(), temporal_blend=0.95)

    def to_c(self) -> N.LuxSettings:
        s = N.LuxSettings()
        s.probe_spacing = self.probe_spacing
        s.interval_length = self.interval_length
        s.normal_bias = self.normal_bias
        s.intensity = self.intensity
        for i in range(3):
            s.environment[i] = self.environment[i]
        s.exposure = self.exposure
        s.emissive_samples = _u32(self.emissive_samples)
        s.levels = _u32(self.levels)
        s.base_columns = _u32(self.base_columns)
        s.base_rows = _u32(self.base_rows)
        s.interval_ratio = self.interval_ratio
        s.interval_rule = _u32(self.interval_rule)
        s.layout = _u32(self.layout)
        s.rays_per_receiver = _u32(self.rays_per_receiver)
        s.frame_index = _u32(self.frame_index)
        s.resolve_scale = _u32(self.sampling.resolve_scale)
        s.temporal_blend = self.temporal_blend
        s.transmittance_blend = self.split_transmittance_blend
        s.history_frames = _u32(self.history_frames)
        s.multi_bounce = 1 if self.multi_bounce else 0
        s.cached_hit_sky = 1 if self.cached_hit_sky else 0
        return s

    @staticmethod
    def from_c(s: N.LuxSettings, sampling: SamplingSettings | None = None) -> "RadianceCascades":
        sampling = replace(sampling or SamplingSettings(), resolve_scale=int(s.resolve_scale))
        return RadianceCascades(
            probe_spacing=s.probe_spacing, interval_length=s.interval_length, normal_bias=s.normal_bias,
            intensity=s.intensity, environment=tuple(s.environment), emissive_samples=int(s.emissive_samples),
            sampling=sampling, exposure=s.exposure, levels=int(s.levels), base_columns=int(s.base_columns),
            base_rows=int(s.base_rows), interval_ratio=s.interval_ratio, interval_rule=int(s.interval_rule),
            layout=int(s.layout), rays_per_receiver=int(s.rays_per_receiver), frame_index=int(s.frame_index),
            temporal_blend=s.temporal_blend, split_transmittance_blend=s.transmittance_blend,
            history_frames=int(s.history_frames), multi_bounce=bool(s.multi_bounce),
            cached_hit_sky=bool(s.cached_hit_sky))

    def sanitized(self) -> "RadianceCascades":
        """RadianceCascades::sanitized() (src/lib.rs:731-759), evaluated by liblux."""
        s = self.to_c()
        lib().lux_settings_sanitize(C.byref(s))
        return RadianceCascades.from_c(s, self.sampling.sanitized())

    def interval_end(self, level: int) -> float:
        s = self.to_c()
        return float(lib().lux_interval_end(C.byref(s), level))

    def direction_count(self, level: int) -> int:
        s = self.to_c()
        return int(lib().lux_direction_count(C.byref(s), level))


def _u32(v) -> int:
    v = int(v)
    return v & 0xFFFFFFFF if v >= 0 else 0


class RadianceCascadesStatus:
    """Deduplicated failure strings (RadianceCascadesStatus::record_failure,
    src/lib.rs:225-230)."""

    def __init__(self):
        self._failures: list[str] = []

    def record_failure(self, message: str) -> None:
        if message not in self._failures:
            self._failures.append(message)

    def failures(self) -> list[str]:
        return list(self._failures)


@dataclass
class RadianceCascadesPlugin:
    """RadianceCascadesPlugin (src/lib.rs:795-900): budgets, and `build`
    creates the device context that render() would use.

    The budgets keep the reference's fields and defaults.  The reference
    spends them in its render plumbing (scene paging against
    `scene_gpu_budget_bytes`, src/render.rs:6925-6950; view settings adapted
    to `view_gpu_budget_bytes`, src/render.rs:416-450), which is outside this
    library: here a scene and a view take exactly the capacities the caller
    passes to GpuScene and SplitView, and allocation failures surface as
    LUX_ERR_OUT_OF_MEMORY."""
    scene_gpu_budget_bytes: int = 256 * 1024 * 1024
    view_gpu_budget_bytes: int = 2 * 1024 * 1024 * 1024
    device: int = 0

    @staticmethod
    def low_end() -> "RadianceCascadesPlugin":
        return RadianceCascadesPlugin(scene_gpu_budget_bytes=256 * 1024 * 1024,
                                      view_gpu_budget_bytes=512 * 1024 * 1024)

    def build(self, stream: int | None = None) -> "LuxContext":
        return LuxContext(self.device, stream)


class LuxContext:
    """A liblux context on one device (lux_context_create)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        desc = N.LuxDeviceDesc(device, stream or None)
        handle = C.c_void_p()
        check(lib().lux_context_create(C.byref(desc), C.byref(handle)))
        self.handle = handle
        self.status = RadianceCascadesStatus()

    def check(self, status: int) -> None:
        if status != N.LUX_OK:
            raw = lib().lux_last_error_message(self.handle)
            message = raw.decode() if raw else ""
            self.status.record_failure(message)
            raise LuxError(status, message)

    def synchronize(self) -> None:
        self.check(lib().lux_context_synchronize(self.handle))

    def close(self) -> None:
        if self.handle:
            lib().lux_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data if a is not None and a.size else 0


class PackedScene:
    """The reference's scene word streams (src/scene.rs:2096-2117, :809-823)
    produced by liblux's native packer (lux_scene_pack)."""

    def __init__(self, scene_words: np.ndarray, geometry_words: np.ndarray, lights: np.ndarray,
                 instance_order: np.ndarray | None = None, blas_cost: float = 0.0, max_depth: int = 0,
                 tlas_nodes: int = 0, blas_nodes: int = 0):
        self.scene_words = np.ascontiguousarray(scene_words, dtype=np.uint32).reshape(-1, 4)
        self.geometry_words = np.ascontiguousarray(geometry_words, dtype=np.uint32).reshape(-1, 4)
        self.lights = np.ascontiguousarray(lights, dtype=np.uint32).reshape(-1, 24)
        self.instance_order = instance_order
        self.blas_cost = blas_cost
        self.max_depth = max_depth
        self.tlas_nodes = tlas_nodes
        self.blas_nodes = blas_nodes
        self.conventional = 0  # leading conventional (point, spot, directional) light records

    def with_conventional_lights(self, records) -> "PackedScene":
        """A copy whose light list starts with these conventional light
        records (conventional_light / directional_light), before the emissive
        ones, as the reference orders them (src/scene.rs:2311-2372)."""
        recs = np.ascontiguousarray(np.asarray(records, dtype=np.uint32).reshape(-1, 24))
        out = PackedScene(self.scene_words, self.geometry_words, np.concatenate([recs, self.lights[self.conventional:]]),
                          self.instance_order, self.blas_cost, self.max_depth, self.tlas_nodes, self.blas_nodes)
        out.conventional = len(recs)
        return out

    @staticmethod
    def pack(positions, indices, mesh_first, mesh_count, instance_mesh, instance_transform, instance_flags,
             instance_material, materials) -> "PackedScene":
        L = lib()
        positions = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
        indices = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1, 3)
        mesh_first = np.ascontiguousarray(mesh_first, dtype=np.uint32)
        mesh_count = np.ascontiguousarray(mesh_count, dtype=np.uint32)
        imesh = np.ascontiguousarray(instance_mesh, dtype=np.uint32)
        ixf = np.ascontiguousarray(instance_transform, dtype=np.float32).reshape(-1, 12)
        iflags = np.ascontiguousarray(instance_flags, dtype=np.uint32)
        imat = np.ascontiguousarray(instance_material, dtype=np.uint32)
        mats = np.ascontiguousarray(materials, dtype=np.uint32).reshape(-1, 32)
        handle = C.c_void_p()
        status = L.lux_scene_pack(_ptr(positions), len(positions), _ptr(indices), len(indices), _ptr(mesh_first),
                                  _ptr(mesh_count), len(mesh_first), _ptr(imesh), _ptr(ixf), _ptr(iflags),
                                  _ptr(imat), len(imesh), _ptr(mats), len(mats), C.byref(handle))
        check(status)
        try:
            sw, gw, nl = C.c_size_t(), C.c_size_t(), C.c_size_t()
            tn, bn = C.c_uint32(), C.c_uint32()
            check(L.lux_packed_scene_sizes(handle, C.byref(sw), C.byref(gw), C.byref(nl), C.byref(tn),
                                           C.byref(bn)))
            scene_words = np.zeros((sw.value, 4), dtype=np.uint32)
            geometry_words = np.zeros((gw.value, 4), dtype=np.uint32)
            lights = np.zeros((nl.value, 24), dtype=np.uint32)
            check(L.lux_packed_scene_copy(handle, _ptr(scene_words), _ptr(geometry_words), _ptr(lights)))
            order = np.zeros(len(imesh), dtype=np.uint32)
            if len(imesh):
                check(L.lux_packed_scene_instance_order(handle, _ptr(order)))
            cost, depth = C.c_double(), C.c_uint32()
            check(L.lux_packed_scene_quality(handle, C.byref(cost), C.byref(depth)))
        finally:
            L.lux_packed_scene_destroy(handle)
        return PackedScene(scene_words, geometry_words, lights, order, cost.value, depth.value, tn.value, bn.value)

    def lights_at(self, world_from_local_slots) -> np.ndarray:
        """lux_emissive_lights_at: this scene's emissive light records at new
        rigid poses (float[instances, 3, 4] in instance-record order)."""
        m = np.ascontiguousarray(world_from_local_slots, dtype=np.float32).reshape(-1, 12)
        out = np.zeros_like(self.lights)
        check(lib().lux_emissive_lights_at(_ptr(self.geometry_words), len(self.geometry_words), _ptr(self.lights),
                                           len(self.lights), _ptr(m), len(m), _ptr(out)))
        return out

    @staticmethod
    def from_desc(desc) -> "PackedScene":
        positions, indices, first, count = desc.arrays()
        return PackedScene.pack(positions, indices, first, count, desc.instance_mesh,
                                np.stack(desc.instance_transform), desc.instance_flags, desc.instance_material,
                                np.stack(desc.materials))


def conventional_light(position, range_: float, color, direction=(0.0, 0.0, -1.0), spot_scale: float = 0.0,
                       spot_offset: float = 0.0) -> np.ndarray:
    """A point (spot_scale = 0) or spot light record (the Light layout of
    conventionalLightResponseTracked, shaders/cascades.slang:136-176):
    position.w = range, color.w = spot offset, direction.w = spot scale."""
    f = np.zeros(24, np.float32)
    f[0:3], f[3] = position, range_
    f[4:7], f[7] = color, spot_offset
    f[8:11], f[11] = direction, spot_scale
    return f.view(np.uint32)


def directional_light(direction_to_light, color) -> np.ndarray:
    """A directional light record: the direction to the source in
    position.xyz, position.w = 0."""
    f = np.zeros(24, np.float32)
    f[0:3] = direction_to_light
    f[4:7] = color
    return f.view(np.uint32)


def validate_scene(packed: PackedScene) -> tuple[int, str]:
    """lux_scene_validate: the status (and message) lux_scene_upload would
    return for these word streams, checked on the host without a device."""
    buf = C.create_string_buffer(512)
    status = lib().lux_scene_validate(_ptr(packed.scene_words), len(packed.scene_words),
                                      _ptr(packed.geometry_words), len(packed.geometry_words),
                                      _ptr(packed.lights), len(packed.lights), packed.conventional, buf, len(buf))
    return int(status), buf.value.decode()


class GpuScene:
    """A scene resident on the device (lux_scene_upload)."""

    def __init__(self, ctx: LuxContext, packed: PackedScene):
        self.ctx = ctx
        self.packed = packed
        handle = C.c_void_p()
        ctx.check(lib().lux_scene_upload(ctx.handle, _ptr(packed.scene_words), len(packed.scene_words),
                                         _ptr(packed.geometry_words), len(packed.geometry_words),
                                         _ptr(packed.lights), len(packed.lights), packed.conventional,
                                         C.byref(handle)))
        self.handle = handle

    def layout(self) -> dict:
        vals = [C.c_uint32() for _ in range(5)]
        self.ctx.check(lib().lux_scene_layout(self.handle, *[C.byref(v) for v in vals]))
        keys = ("nodes", "node_bytes", "triangles", "triangle_bytes", "instances")
        return {k: v.value for k, v in zip(keys, vals)}

    def refit(self, world_from_local, lights=None) -> None:
        """lux_scene_refit: new float[instances, 3, 4] poses in instance-record
        (slot) order; optional replacement light records (LuxLight dtype)."""
        m = np.ascontiguousarray(world_from_local, dtype=np.float32).reshape(-1, 12)
        lp, ln = (None, 0)
        if lights is not None:
            lights = np.ascontiguousarray(lights)
            lp, ln = _ptr(lights), len(lights)
        self.ctx.check(lib().lux_scene_refit(self.handle, _ptr(m), len(m), lp, ln))

    def read_words(self) -> np.ndarray:
        """lux_scene_read_words: the device scene words (uint32[words, 4])."""
        out = np.zeros((len(self.packed.scene_words), 4), dtype=np.uint32)
        self.ctx.check(lib().lux_scene_read_words(self.handle, _ptr(out), len(out)))
        return out

    def close(self) -> None:
        if self.handle:
            lib().lux_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


RAY_DTYPE = np.dtype([("origin", "<f4", 3), ("tmin", "<f4"), ("direction", "<f4", 3), ("limit", "<f4")])
HIT_DTYPE = np.dtype([("distance", "<f4"), ("triangle", "<u4"), ("instance", "<u4"), ("errors", "<u4"),
                      ("barycentric", "<f4", 3), ("visited", "<u4")])


def trace_rays(ctx: LuxContext, scene: GpuScene, rays_device_ptr: int, count: int, hits_device_ptr: int,
               any_hit: bool = False) -> None:
    """lux_trace_rays on device buffers of RAY_DTYPE / HIT_DTYPE records.

    The launch is ordered on the context's stream; this wrapper waits for it,
    so the hits can be read from any stream when it returns.  The rays must
    be complete in device memory before the call."""
    ctx.check(lib().lux_trace_rays(ctx.handle, scene.handle, rays_device_ptr, count, 1 if any_hit else 0,
                                   hits_device_ptr))
    ctx.synchronize()


def interval_radiance(ctx: LuxContext, scene: GpuScene, settings: RadianceCascades, rays_device_ptr: int,
                      count: int, out_device_ptr: int) -> None:
    """lux_interval_radiance: float4 (radiance rgb, hit distance | -1) per ray.
    Waits for the context's stream before returning (see trace_rays)."""
    s = settings.to_c()
    ctx.check(lib().lux_interval_radiance(ctx.handle, scene.handle, C.byref(s), rays_device_ptr, count,
                                          out_device_ptr))
    ctx.synchronize()


def reference_irradiance(ctx: LuxContext, scene: GpuScene, settings: RadianceCascades, position_ptr: int,
                         normal_ptr: int, count: int, spp: int, seed: int, out_ptr: int) -> None:
    """lux_reference_irradiance: FP64 Monte Carlo reference (device double4[count]:
    mean rgb, supported samples) at device float4 points / unit normals."""
    s = settings.to_c()
    ctx.check(lib().lux_reference_irradiance(ctx.handle, scene.handle, C.byref(s), position_ptr, normal_ptr, count,
                                             spp, seed, out_ptr))
    ctx.synchronize()


def path_reference(ctx: LuxContext, scene: GpuScene, settings: RadianceCascades, position_ptr: int, normal_ptr: int,
                   count: int, spp: int, bounces: int, seed: int, out_ptr: int) -> None:
    """lux_path_reference: FP64-accumulated path-traced reference (device
    double4[count]: mean rgb, supported samples) with `bounces` diffuse
    vertices at device float4 points / unit normals."""
    s = settings.to_c()
    ctx.check(lib().lux_path_reference(ctx.handle, scene.handle, C.byref(s), position_ptr, normal_ptr, count, spp,
                                       bounces, seed, out_ptr))
    ctx.synchronize()


def error_stats(ctx: LuxContext, estimate_ptr: int, reference_ptr: int, count: int) -> dict:
    """lux_error_stats: FP64 error of a float4 estimate against a double4 reference."""
    out = (C.c_double * 4)()
    ctx.check(lib().lux_error_stats(ctx.handle, estimate_ptr, reference_ptr, count, out))
    sq, ref_sum, used, mx = out[0], out[1], out[2], out[3]
    n = max(used, 1.0) * 3.0
    rmse = (sq / n) ** 0.5
    mean = ref_sum / n
    return {"rmse": rmse, "mean_reference": mean, "relative_rmse": rmse / mean if mean > 0 else float("inf"),
            "points": int(used), "max_abs_error": mx}


def measure_read_rate(ctx: LuxContext, nbytes: int, passes: int) -> float:
    """lux_measure_read_rate: GB/s of one launch reading a device buffer of
    `nbytes` bytes `passes` times (inside L2: the L2 read rate)."""
    out = C.c_double(0.0)
    ctx.check(lib().lux_measure_read_rate(ctx.handle, int(nbytes), int(passes), C.byref(out)))
    return float(out.value)


def camera_struct(clip_from_world, position, viewport_height: int, target_pixels: int = 1) -> N.LuxCamera:
    """A LuxCamera for distance LODs (enabled)."""
    cam = N.LuxCamera()
    m = np.asarray(clip_from_world, np.float32).reshape(16)
    for i in range(16):
        cam.clip_from_world[i] = float(m[i])
    pos = np.asarray(position, np.float32).reshape(3)
    for a in range(3):
        cam.position[a] = float(pos[a])
    cam.viewport_height = int(viewport_height)
    cam.target_pixels = int(target_pixels)
    cam.enabled = 1
    return cam


class SplitView:
    """Per-view transport state (ViewBuffers) and one frame of
    seed -> trace -> deposit -> merge -> pack, then resolve."""

    def __init__(self, ctx: LuxContext, max_receivers: int, max_cells: int, max_entries: int,
                 max_rays: int | None = None):
        self.ctx = ctx
        if max_rays is None:
            max_rays = max(max_receivers, min(max_entries, 1 << 24))
        desc = N.LuxViewDesc(max_receivers, max_cells, max_entries, max_rays, 0)
        handle = C.c_void_p()
        ctx.check(lib().lux_view_create(ctx.handle, C.byref(desc), C.byref(handle)))
        self.handle = handle
        self.desc = desc
        self.settings: RadianceCascades | None = None
        self._owned = True

    def trace_merge(self, scene: GpuScene, settings: RadianceCascades, position_ptr: int, normal_ptr: int,
                    count: int) -> None:
        """Device pointers to float4 receiver positions / normals."""
        s = settings.to_c()
        rc = N.LuxReceivers(position_ptr, normal_ptr, count)
        self.ctx.check(lib().lux_view_trace_merge(self.handle, scene.handle, C.byref(s), C.byref(rc)))
        self.settings = settings

    def resolve(self, settings: RadianceCascades, position_ptr: int, normal_ptr: int, count: int,
                out_ptr: int) -> None:
        s = settings.to_c()
        self.ctx.check(lib().lux_view_resolve(self.handle, C.byref(s), position_ptr, normal_ptr, count, out_ptr))

    def frame_host(self, scene: GpuScene, settings: RadianceCascades, receiver_pos: np.ndarray,
                   receiver_nrm: np.ndarray, point_pos: np.ndarray, point_nrm: np.ndarray,
                   out: np.ndarray | None = None) -> np.ndarray:
        """One frame from host buffers (lux_view_frame_host)."""
        if out is None:
            out = np.zeros((len(point_pos), 4), dtype=np.float32)
        s = settings.to_c()
        self.ctx.check(lib().lux_view_frame_host(self.handle, scene.handle, C.byref(s), _ptr(receiver_pos),
                                                 _ptr(receiver_nrm), len(receiver_pos), _ptr(point_pos),
                                                 _ptr(point_nrm), len(point_pos), _ptr(out)))
        return out

    def set_timing(self, enable: bool = True) -> None:
        self.ctx.check(lib().lux_view_set_timing(self.handle, 1 if enable else 0))

    def tuning(self) -> N.LuxTuning:
        t = N.LuxTuning()
        self.ctx.check(lib().lux_view_get_tuning(self.handle, C.byref(t)))
        return t

    def set_tuning(self, **fields) -> None:
        t = self.tuning()
        for k, val in fields.items():
            setattr(t, k, int(val))
        self.ctx.check(lib().lux_view_set_tuning(self.handle, C.byref(t)))

    def timings(self) -> N.LuxTimings:
        t = N.LuxTimings()
        self.ctx.check(lib().lux_view_timings(self.handle, C.byref(t)))
        return t

    def stats(self) -> N.LuxStats:
        st = N.LuxStats()
        self.ctx.check(lib().lux_view_stats(self.handle, C.byref(st)))
        return st

    def read_level(self, level: int):
        """(keys int32[cells,4], merged f32[cells,dirs,4], raw f32[cells,dirs,4], samples u32[cells,dirs])."""
        st = self.stats()
        cells = int(st.cells[level])
        dirs = self.settings.direction_count(level)
        keys = np.zeros((cells, 4), dtype=np.int32)
        merged = np.zeros((cells, dirs, 4), dtype=np.float32)
        raw = np.zeros((cells, dirs, 4), dtype=np.float32)
        samples = np.zeros((cells, dirs), dtype=np.uint32)
        if cells:
            self.ctx.check(lib().lux_view_read_level(self.handle, level, _ptr(keys), _ptr(merged), _ptr(raw),
                                                     _ptr(samples)))
        return keys, merged, raw, samples

    def read_probes(self):
        st = self.stats()
        cells = int(st.cells[0])
        keys = np.zeros((cells, 4), dtype=np.int32)
        tables = np.zeros((cells, 36, 4), dtype=np.float32)
        if cells:
            self.ctx.check(lib().lux_view_read_probes(self.handle, _ptr(keys), _ptr(tables)))
        return keys, tables

    def set_cache(self, cache, cutoff_level: int = 3, validate_period: int = 16, error_bound: float = 0.25,
                  train_samples: int = 65536, fallback_frames: int = 32) -> None:
        """lux_view_set_cache: the learned-cache form (cache=None: plain)."""
        if cache is None:
            self.ctx.check(lib().lux_view_set_cache(self.handle, None))
            return
        m = N.LuxCacheMode()
        m.cache = cache.handle
        m.cutoff_level = cutoff_level
        m.validate_period = validate_period
        m.error_bound = error_bound
        m.train_samples = train_samples
        m.fallback_frames = fallback_frames
        self.ctx.check(lib().lux_view_set_cache(self.handle, C.byref(m)))

    def cache_stats(self) -> N.LuxCacheFrameStats:
        out = N.LuxCacheFrameStats()
        self.ctx.check(lib().lux_view_cache_stats(self.handle, C.byref(out)))
        return out

    def reset_history(self) -> None:
        """lux_view_reset_history: the next frame starts without history."""
        self.ctx.check(lib().lux_view_reset_history(self.handle))

    def invalidate_bounds(self, lo, hi) -> None:
        """lux_view_invalidate_bounds: records near this box take no history next frame."""
        lo = np.asarray(lo, np.float32)
        hi = np.asarray(hi, np.float32)
        self.ctx.check(lib().lux_view_invalidate_bounds(self.handle, _ptr(lo), _ptr(hi)))

    def read_hits(self, count: int) -> np.ndarray:
        """lux_view_read_hits: the last Split frame's first `count` interval-ray hits."""
        out = np.zeros(count, dtype=HIT_DTYPE)
        self.ctx.check(lib().lux_view_read_hits(self.handle, _ptr(out), count))
        return out

    def set_camera(self, clip_from_world=None, position=None, viewport_height: int = 0,
                   target_pixels: int = 1) -> None:
        """lux_view_set_camera: distance LODs of later Split frames and
        resolves from this camera (clip_from_world 4x4 row-major, world
        position, viewport height in pixels, probe footprint in pixels);
        None disables them."""
        if clip_from_world is None:
            self.ctx.check(lib().lux_view_set_camera(self.handle, None))
            return
        cam = camera_struct(clip_from_world, position, viewport_height, target_pixels)
        self.ctx.check(lib().lux_view_set_camera(self.handle, C.byref(cam)))

    def secondary(self) -> "SplitView | None":
        """lux_view_secondary: the multi-bounce secondary cache of this view
        (read-only; None before the first multi-bounce frame).  Its settings
        are this view's with probe spacing and interval length x4."""
        handle = C.c_void_p()
        self.ctx.check(lib().lux_view_secondary(self.handle, C.byref(handle)))
        if not handle.value:
            return None
        sec = SplitView.__new__(SplitView)
        sec.ctx = self.ctx
        sec.handle = handle
        sec.desc = self.desc
        sec.settings = replace(self.settings, multi_bounce=False, cached_hit_sky=False,
                               probe_spacing=self.settings.probe_spacing * 4.0,
                               interval_length=self.settings.interval_length * 4.0) if self.settings else None
        sec._owned = False
        sec._owner = self  # keeps the owning view alive
        return sec

    def close(self) -> None:
        if self.handle and getattr(self, "_owned", True):
            lib().lux_view_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many (view, scene, receivers) jobs per frame: one launch per trace
    stage over all jobs, the whole frame captured once as a CUDA graph and
    replayed (lux_batch_*)."""

    def __init__(self, ctx: LuxContext):
        self.ctx = ctx
        handle = C.c_void_p()
        ctx.check(lib().lux_batch_create(ctx.handle, C.byref(handle)))
        self.handle = handle

    def set_graph(self, enable: bool) -> None:
        self.ctx.check(lib().lux_batch_set_graph(self.handle, 1 if enable else 0))

    def set_tuning(self, closest_blocks_per_sm: int = 16, shadow_blocks_per_sm: int = 16, fused_trace: int = 0,
                   tile_rays: int = 32) -> None:
        t = N.LuxTuning()
        t.closest_blocks_per_sm = closest_blocks_per_sm
        t.shadow_blocks_per_sm = shadow_blocks_per_sm
        t.fused_trace = fused_trace
        t.tile_rays = tile_rays
        self.ctx.check(lib().lux_batch_set_tuning(self.handle, C.byref(t)))

    def set_wait(self, limit_ns: int, missing_arrivals: int = 0) -> None:
        """Bound of each grid-barrier wait of the fused trace launch;
        missing_arrivals > 0 makes the first wait run out (a test hook)."""
        self.ctx.check(lib().lux_batch_set_wait(self.handle, int(limit_ns), int(missing_arrivals)))

    def status(self) -> None:
        """Waits for the last frame; raises LuxError(LUX_ERR_TIMEOUT) when a
        grid-barrier wait of its fused trace launch ran out."""
        self.ctx.check(lib().lux_batch_status(self.handle))

    def trace_merge(self, jobs, settings: RadianceCascades) -> None:
        """jobs: sequence of (SplitView, GpuScene, position_ptr, normal_ptr, count)."""
        arr = (N.LuxBatchJob * len(jobs))()
        for k, (view, scene, pos, nrm, count) in enumerate(jobs):
            arr[k].view = view.handle
            arr[k].scene = scene.handle
            arr[k].receivers = N.LuxReceivers(pos, nrm, count)
            view.settings = settings
        s = settings.to_c()
        self.ctx.check(lib().lux_batch_trace_merge(self.handle, arr, len(jobs), C.byref(s)))

    def info(self) -> N.LuxBatchInfo:
        out = N.LuxBatchInfo()
        self.ctx.check(lib().lux_batch_info(self.handle, C.byref(out)))
        return out

    def close(self) -> None:
        if self.handle:
            lib().lux_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


CACHE_SAMPLE_DTYPE = np.dtype([("position", "<f4", 3), ("weight", "<f4"), ("direction", "<f4", 3), ("pad0", "<f4"),
                               ("normal", "<f4", 3), ("pad1", "<f4"), ("albedo", "<f4", 3), ("pad2", "<f4")])
CACHE_WEIGHTS = 4 * 64 * 64 + 16 * 64


class ScreenFilter:
    """Screen reconstruction after the world resolve (the reference's
    temporal + denoise passes, shaders/cascades.slang:310-690): owns the
    screen history of one view at the resolve extent."""

    def __init__(self, ctx: LuxContext, width: int, height: int):
        self.ctx = ctx
        self.width, self.height = int(width), int(height)
        handle = C.c_void_p()
        ctx.check(lib().lux_screen_create(ctx.handle, self.width, self.height, C.byref(handle)))
        self.handle = handle

    def filter(self, settings: RadianceCascades, irradiance_ptr: int, position_ptr: int, normal_ptr: int,
               identity_ptr: int, previous_clip_from_world, out_ptr: int, spatial_filter_steps: int = 3,
               scene_changed: bool = False, dirty=None) -> None:
        """Device pointers at the resolve extent: irradiance / position (w =
        view depth) / normal float4, identity uint32 x 2; out float4.
        previous_clip_from_world: 4x4 row-major; dirty: (lo xyz, hi xyz)."""
        f = N.LuxScreenFrame()
        f.irradiance, f.position, f.normal, f.identity = irradiance_ptr, position_ptr, normal_ptr, identity_ptr
        m = np.asarray(previous_clip_from_world, np.float32).reshape(16)
        for i in range(16):
            f.previous_clip_from_world[i] = float(m[i])
        if dirty is not None:
            d = np.asarray(dirty, np.float32).reshape(6)
            for a in range(3):
                f.dirty_lo[a], f.dirty_hi[a] = float(d[a]), float(d[3 + a])
            f.dirty = 1
        f.scene_changed = 1 if scene_changed else 0
        f.spatial_filter_steps = int(spatial_filter_steps)
        s = settings.to_c()
        self.ctx.check(lib().lux_screen_filter(self.handle, C.byref(s), C.byref(f), out_ptr))

    def reset(self) -> None:
        self.ctx.check(lib().lux_screen_reset(self.handle))

    def read_history(self):
        """(irradiance f32[h, w, 4], metadata f32[h, w, 4]: retained length,
        variance, support mask, surface flag)."""
        irr = np.zeros((self.height, self.width, 4), np.float32)
        meta = np.zeros((self.height, self.width, 4), np.float32)
        self.ctx.check(lib().lux_screen_read_history(self.handle, _ptr(irr), _ptr(meta)))
        return irr, meta

    def close(self) -> None:
        if self.handle:
            lib().lux_screen_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LearnedCache:
    """lux_cache_*: hash-grid encoded MLP radiance cache (tcgen05 BF16 MLP)."""

    def __init__(self, ctx: LuxContext, **desc):
        self.ctx = ctx
        d = N.LuxCacheDesc()
        lib().lux_cache_desc_default(C.byref(d))
        for k, v in desc.items():
            setattr(d, k, v)
        handle = C.c_void_p()
        ctx.check(lib().lux_cache_create(ctx.handle, C.byref(d), C.byref(handle)))
        self.handle = handle
        self.desc = d

    def set_bounds(self, lo, hi) -> None:
        lo = np.asarray(lo, np.float32)
        hi = np.asarray(hi, np.float32)
        self.ctx.check(lib().lux_cache_set_bounds(self.handle, _ptr(lo), _ptr(hi)))

    def train(self, samples_ptr: int, targets_ptr: int, count: int) -> None:
        self.ctx.check(lib().lux_cache_train(self.handle, samples_ptr, targets_ptr, count))

    def query(self, queries_ptr: int, count: int, out_ptr: int) -> None:
        self.ctx.check(lib().lux_cache_query(self.handle, queries_ptr, count, out_ptr))

    def encode(self, samples_ptr: int, count: int, out_ptr: int) -> None:
        self.ctx.check(lib().lux_cache_encode(self.handle, samples_ptr, count, out_ptr))

    def forward(self, encoded_ptr: int, count: int, out_ptr: int) -> None:
        self.ctx.check(lib().lux_cache_forward(self.handle, encoded_ptr, count, out_ptr))

    def weights(self) -> list:
        """FP32 master weights: 4 x [64, 64] hidden layers and the [16, 64] output layer ([out, in])."""
        w = np.zeros(CACHE_WEIGHTS, np.float32)
        self.ctx.check(lib().lux_cache_read_weights(self.handle, _ptr(w)))
        layers = [w[k * 4096:(k + 1) * 4096].reshape(64, 64) for k in range(4)]
        layers.append(w[4 * 4096:].reshape(16, 64))
        return layers

    def stats(self) -> N.LuxCacheStats:
        out = N.LuxCacheStats()
        self.ctx.check(lib().lux_cache_stats(self.handle, C.byref(out)))
        return out

    def table_size(self) -> int:
        return int(self.desc.levels) * (1 << int(self.desc.log2_table)) * 2

    def gradients(self, samples_ptr: int, targets_ptr: int, count: int):
        """lux_cache_gradients: (weight gradients as weights() layers, FP32
        hash-table gradients [levels, 2^log2_table, 2]) of one pass, no step."""
        w = np.zeros(CACHE_WEIGHTS, np.float32)
        t = np.zeros(self.table_size(), np.float32)
        self.ctx.check(lib().lux_cache_gradients(self.handle, samples_ptr, targets_ptr, count, _ptr(w), _ptr(t)))
        layers = [w[k * 4096:(k + 1) * 4096].reshape(64, 64) for k in range(4)]
        layers.append(w[4 * 4096:].reshape(16, 64))
        return layers, t.reshape(int(self.desc.levels), -1, 2)

    def table(self) -> np.ndarray:
        """The FP32 master hash table [levels, 2^log2_table, 2]."""
        t = np.zeros(self.table_size(), np.float32)
        self.ctx.check(lib().lux_cache_read_table(self.handle, _ptr(t)))
        return t.reshape(int(self.desc.levels), -1, 2)

    def close(self) -> None:
        if self.handle:
            lib().lux_cache_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
