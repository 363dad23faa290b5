"""ctypes binding of liblux.so (include/lux.h).

This is the binding a host engine adds to call the library; the Rust FFI
crate of bevy_lux would declare the same records and functions.  The
library is built in-tree by ``bevy_penumbra_b200.build``; importing this
module without it raises, so no code path silently runs without the CUDA
kernels.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblux.so")

LUX_OK = 0
STATUS_NAMES = {
    0: "LUX_OK", 1: "LUX_ERR_INVALID_ARGUMENT", 2: "LUX_ERR_CUDA", 3: "LUX_ERR_OUT_OF_MEMORY",
    4: "LUX_ERR_CAPACITY", 5: "LUX_ERR_MALFORMED_SCENE", 6: "LUX_ERR_NO_DEVICE", 7: "LUX_ERR_TIMEOUT",
    8: "LUX_ERR_INTERNAL",
}
LUX_EMPTY = 0xFFFFFFFF
LUX_HIT_QUERY_UNSUPPORTED = 4
LUX_LAYOUT_SPLIT = 0
LUX_LAYOUT_DENSE = 1
LUX_INTERVAL_ENDS_GEOMETRIC = 0
LUX_INTERVAL_LENGTHS_GEOMETRIC = 1
LUX_MAX_LEVELS = 12


class LuxError(RuntimeError):
    """A non-zero lux_status, with the context's last error message."""

    def __init__(self, status: int, message: str = ""):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


class LuxDeviceDesc(C.Structure):
    _fields_ = [("device", C.c_int32), ("stream", C.c_void_p)]


class LuxRay(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("tmin", C.c_float), ("direction", C.c_float * 3),
                ("limit", C.c_float)]


class LuxHit(C.Structure):
    _fields_ = [("distance", C.c_float), ("triangle", C.c_uint32), ("instance", C.c_uint32),
                ("errors", C.c_uint32), ("barycentric", C.c_float * 3), ("visited", C.c_uint32)]


class LuxLight(C.Structure):
    _fields_ = [("position", C.c_float * 4), ("color", C.c_float * 4), ("direction", C.c_float * 4),
                ("edge1", C.c_float * 4), ("edge2", C.c_float * 4), ("source", C.c_uint32 * 4)]


class LuxSettings(C.Structure):
    _fields_ = [
        ("probe_spacing", C.c_float), ("interval_length", C.c_float), ("normal_bias", C.c_float),
        ("intensity", C.c_float), ("environment", C.c_float * 3), ("exposure", C.c_float),
        ("emissive_samples", C.c_uint32), ("levels", C.c_uint32), ("base_columns", C.c_uint32),
        ("base_rows", C.c_uint32), ("interval_ratio", C.c_float), ("interval_rule", C.c_uint32),
        ("layout", C.c_uint32), ("rays_per_receiver", C.c_uint32), ("frame_index", C.c_uint32),
        ("resolve_scale", C.c_uint32), ("temporal_blend", C.c_float), ("transmittance_blend", C.c_float),
        ("history_frames", C.c_uint32), ("multi_bounce", C.c_uint32),
        ("cached_hit_sky", C.c_uint32),
    ]


class LuxReceivers(C.Structure):
    _fields_ = [("position", C.c_void_p), ("normal", C.c_void_p), ("count", C.c_uint32)]


class LuxStats(C.Structure):
    _fields_ = [
        ("interval_rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("nodes_visited", C.c_uint64),
        ("triangles_tested", C.c_uint64), ("instances_visited", C.c_uint64), ("deposits", C.c_uint64),
        ("unsupported", C.c_uint64), ("shadow_nodes", C.c_uint64), ("shadow_triangles", C.c_uint64),
        ("shadow_instances", C.c_uint64), ("cells", C.c_uint32 * LUX_MAX_LEVELS),
        ("entries", C.c_uint64 * LUX_MAX_LEVELS), ("levels", C.c_uint32), ("error_flags", C.c_uint32),
    ]


class LuxViewDesc(C.Structure):
    _fields_ = [("max_receivers", C.c_uint32), ("max_cells", C.c_uint32), ("max_entries", C.c_uint64),
                ("max_rays", C.c_uint32), ("reserved", C.c_uint32)]


class LuxTimings(C.Structure):
    _fields_ = [("seed_ms", C.c_float), ("trace_ms", C.c_float), ("merge_ms", C.c_float),
                ("pack_ms", C.c_float), ("resolve_ms", C.c_float)]


class LuxTuning(C.Structure):
    _fields_ = [("closest_mode", C.c_uint32), ("shadow_mode", C.c_uint32), ("closest_blocks_per_sm", C.c_uint32),
                ("shadow_blocks_per_sm", C.c_uint32), ("sort_queries", C.c_uint32), ("sort_rays", C.c_uint32),
                ("stack_depth", C.c_uint32), ("fused_trace", C.c_uint32), ("tile_rays", C.c_uint32),
                ("reserved", C.c_uint32)]


class LuxCacheDesc(C.Structure):
    _fields_ = [("levels", C.c_uint32), ("log2_table", C.c_uint32), ("base_resolution", C.c_uint32),
                ("growth", C.c_float), ("learning_rate", C.c_float), ("batch", C.c_uint32), ("seed", C.c_uint32),
                ("reserved", C.c_uint32)]


class LuxCacheStats(C.Structure):
    _fields_ = [("steps", C.c_uint64), ("samples", C.c_uint64), ("last_loss", C.c_float),
                ("error_flags", C.c_uint32)]


class LuxCacheMode(C.Structure):
    _fields_ = [("cache", C.c_void_p), ("cutoff_level", C.c_uint32), ("validate_period", C.c_uint32),
                ("error_bound", C.c_float), ("train_samples", C.c_uint32), ("fallback_frames", C.c_uint32),
                ("reserved", C.c_uint32 * 3)]


class LuxCacheFrameStats(C.Structure):
    _fields_ = [("cached_rays", C.c_uint64), ("validated_rays", C.c_uint64), ("train_candidates", C.c_uint64),
                ("trained_samples", C.c_uint64), ("validated_cells", C.c_uint32), ("failed_cells", C.c_uint32),
                ("fallback_rays", C.c_uint32), ("validated_bias", C.c_float)]


class LuxBatchJob(C.Structure):
    _fields_ = [("view", C.c_void_p), ("scene", C.c_void_p), ("receivers", LuxReceivers)]


class LuxBatchInfo(C.Structure):
    _fields_ = [("jobs", C.c_uint32), ("graph_captures", C.c_uint32), ("graph_launches", C.c_uint64),
                ("interval_rays", C.c_uint64), ("kernels_per_frame", C.c_uint32), ("reserved", C.c_uint32)]


class LuxCamera(C.Structure):
    _fields_ = [("clip_from_world", C.c_float * 16), ("position", C.c_float * 3), ("viewport_height", C.c_uint32),
                ("target_pixels", C.c_uint32), ("enabled", C.c_uint32)]


class LuxScreenFrame(C.Structure):
    _fields_ = [("irradiance", C.c_void_p), ("position", C.c_void_p), ("normal", C.c_void_p),
                ("identity", C.c_void_p), ("previous_clip_from_world", C.c_float * 16),
                ("dirty_lo", C.c_float * 3), ("dirty_hi", C.c_float * 3), ("dirty", C.c_uint32),
                ("scene_changed", C.c_uint32), ("spatial_filter_steps", C.c_uint32), ("reserved", C.c_uint32)]


P = C.c_void_p
U32 = C.c_uint32
SZ = C.c_size_t

# name -> (restype, argtypes); every symbol include/lux.h declares.
SIGNATURES = {
    "lux_abi_version": (U32, []),
    "lux_context_create": (C.c_int, [C.POINTER(LuxDeviceDesc), C.POINTER(P)]),
    "lux_context_destroy": (C.c_int, [P]),
    "lux_last_error_message": (C.c_char_p, [P]),
    "lux_context_synchronize": (C.c_int, [P]),
    "lux_settings_default": (None, [C.POINTER(LuxSettings)]),
    "lux_settings_low_end": (None, [C.POINTER(LuxSettings)]),
    "lux_settings_sanitize": (None, [C.POINTER(LuxSettings)]),
    "lux_interval_end": (C.c_float, [C.POINTER(LuxSettings), U32]),
    "lux_direction_count": (U32, [C.POINTER(LuxSettings), U32]),
    "lux_scene_pack": (C.c_int, [P, U32, P, U32, P, P, U32, P, P, P, P, U32, P, U32, C.POINTER(P)]),
    "lux_packed_scene_sizes": (C.c_int, [P, C.POINTER(SZ), C.POINTER(SZ), C.POINTER(SZ), C.POINTER(U32),
                                         C.POINTER(U32)]),
    "lux_packed_scene_copy": (C.c_int, [P, P, P, P]),
    "lux_packed_scene_instance_order": (C.c_int, [P, P]),
    "lux_packed_scene_quality": (C.c_int, [P, C.POINTER(C.c_double), C.POINTER(U32)]),
    "lux_packed_scene_destroy": (None, [P]),
    "lux_scene_upload": (C.c_int, [P, P, SZ, P, SZ, P, U32, U32, C.POINTER(P)]),
    "lux_scene_validate": (C.c_int, [P, SZ, P, SZ, P, U32, U32, C.c_char_p, SZ]),
    "lux_scene_destroy": (C.c_int, [P]),
    "lux_scene_refit": (C.c_int, [P, P, U32, P, U32]),
    "lux_emissive_lights_at": (C.c_int, [P, SZ, P, U32, P, U32, P]),
    "lux_scene_read_words": (C.c_int, [P, P, SZ]),
    "lux_scene_layout": (C.c_int, [P, C.POINTER(U32), C.POINTER(U32), C.POINTER(U32), C.POINTER(U32),
                                   C.POINTER(U32)]),
    "lux_trace_rays": (C.c_int, [P, P, P, U32, U32, P]),
    "lux_interval_radiance": (C.c_int, [P, P, C.POINTER(LuxSettings), P, U32, P]),
    "lux_interval_radiance_noalloc": (C.c_int, [P, P, C.POINTER(LuxSettings), P, U32, P]),
    "lux_view_create": (C.c_int, [P, C.POINTER(LuxViewDesc), C.POINTER(P)]),
    "lux_view_destroy": (C.c_int, [P]),
    "lux_view_trace_merge": (C.c_int, [P, P, C.POINTER(LuxSettings), C.POINTER(LuxReceivers)]),
    "lux_view_resolve": (C.c_int, [P, C.POINTER(LuxSettings), P, P, U32, P]),
    "lux_view_frame_host": (C.c_int, [P, P, C.POINTER(LuxSettings), P, P, U32, P, P, U32, P]),
    "lux_view_stats": (C.c_int, [P, C.POINTER(LuxStats)]),
    "lux_view_set_timing": (C.c_int, [P, U32]),
    "lux_view_timings": (C.c_int, [P, C.POINTER(LuxTimings)]),
    "lux_view_set_tuning": (C.c_int, [P, C.POINTER(LuxTuning)]),
    "lux_view_get_tuning": (C.c_int, [P, C.POINTER(LuxTuning)]),
    "lux_view_read_level": (C.c_int, [P, U32, P, P, P, P]),
    "lux_view_read_probes": (C.c_int, [P, P, P]),
    "lux_view_read_hits": (C.c_int, [P, P, U32]),
    "lux_view_reset_history": (C.c_int, [P]),
    "lux_view_secondary": (C.c_int, [P, C.POINTER(C.c_void_p)]),
    "lux_view_set_camera": (C.c_int, [P, C.c_void_p]),
    "lux_view_invalidate_bounds": (C.c_int, [P, P, P]),
    "lux_view_set_cache": (C.c_int, [P, C.POINTER(LuxCacheMode)]),
    "lux_view_cache_stats": (C.c_int, [P, C.POINTER(LuxCacheFrameStats)]),
    "lux_reference_round_samples": (U32, [U32, U32]),
    "lux_reference_irradiance": (C.c_int, [P, P, C.POINTER(LuxSettings), P, P, U32, U32, U32, P]),
    "lux_error_stats": (C.c_int, [P, P, P, U32, C.POINTER(C.c_double)]),
    "lux_measure_read_rate": (C.c_int, [P, C.c_uint64, U32, C.POINTER(C.c_double)]),
    "lux_path_reference": (C.c_int, [P, P, C.POINTER(LuxSettings), P, P, U32, U32, U32, U32, P]),
    "lux_cache_desc_default": (None, [C.POINTER(LuxCacheDesc)]),
    "lux_cache_create": (C.c_int, [P, C.POINTER(LuxCacheDesc), C.POINTER(P)]),
    "lux_cache_destroy": (C.c_int, [P]),
    "lux_cache_set_bounds": (C.c_int, [P, P, P]),
    "lux_cache_train": (C.c_int, [P, P, P, U32]),
    "lux_cache_query": (C.c_int, [P, P, U32, P]),
    "lux_cache_stats": (C.c_int, [P, C.POINTER(LuxCacheStats)]),
    "lux_cache_encode": (C.c_int, [P, P, U32, P]),
    "lux_cache_read_weights": (C.c_int, [P, P]),
    "lux_cache_forward": (C.c_int, [P, P, U32, P]),
    "lux_cache_gradients": (C.c_int, [P, P, P, U32, P, P]),
    "lux_cache_read_table": (C.c_int, [P, P]),
    "lux_batch_create": (C.c_int, [P, C.POINTER(P)]),
    "lux_batch_destroy": (C.c_int, [P]),
    "lux_batch_set_graph": (C.c_int, [P, U32]),
    "lux_batch_set_tuning": (C.c_int, [P, C.POINTER(LuxTuning)]),
    "lux_batch_trace_merge": (C.c_int, [P, P, U32, P]),
    "lux_batch_info": (C.c_int, [P, C.POINTER(LuxBatchInfo)]),
    "lux_batch_status": (C.c_int, [P]),
    "lux_batch_set_wait": (C.c_int, [P, C.c_uint64, U32]),
    "lux_screen_create": (C.c_int, [P, C.c_uint32, C.c_uint32, C.POINTER(C.c_void_p)]),
    "lux_screen_destroy": (C.c_int, [P]),
    "lux_screen_reset": (C.c_int, [P]),
    "lux_screen_filter": (C.c_int, [P, C.POINTER(LuxSettings), C.POINTER(LuxScreenFrame), C.c_void_p]),
    "lux_screen_read_history": (C.c_int, [P, C.c_void_p, C.c_void_p]),
}

_lib = None


def lib() -> C.CDLL:
    """Loads liblux.so (raises if it was not built: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"liblux.so is not built at {LIB_PATH}; run bevy_penumbra_b200.build.build()")
        handle = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status: int, ctx=None) -> None:
    if status != LUX_OK:
        message = ""
        if ctx:
            raw = lib().lux_last_error_message(ctx)
            message = raw.decode() if raw else ""
        raise LuxError(status, message)
