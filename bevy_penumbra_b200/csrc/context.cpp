// context.cpp - contexts, error reporting and the RadianceCascades settings
// mirror (src/lib.rs:671-759).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <string>

#include "lux_internal.h"

lux_status lux_fail(LuxContext *ctx, lux_status status, const std::string &message) {
    if (ctx) ctx->last_error = message;
    return status;
}

lux_status lux_cuda_check(LuxContext *ctx, int err, const char *what) {
    if (err == cudaSuccess) return LUX_OK;
    std::string message = std::string(what) + ": " + cudaGetErrorString((cudaError_t)err);
    return lux_fail(ctx, err == cudaErrorMemoryAllocation ? LUX_ERR_OUT_OF_MEMORY : LUX_ERR_CUDA, message);
}

extern "C" uint32_t lux_abi_version(void) { return LUX_ABI_VERSION; }

extern "C" lux_status lux_context_create(const LuxDeviceDesc *desc, LuxContext **out) {
    if (!out) return LUX_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return LUX_ERR_NO_DEVICE;
    }
    int device = desc ? desc->device : 0;
    if (device < 0 || device >= count) return LUX_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) return LUX_ERR_CUDA;
    LuxContext *ctx = new (std::nothrow) LuxContext();
    if (!ctx) return LUX_ERR_OUT_OF_MEMORY;
    ctx->device = device;
    cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (desc && desc->stream) {
        ctx->stream = (cudaStream_t)desc->stream;
    } else {
        if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete ctx;
            return LUX_ERR_CUDA;
        }
        ctx->owns_stream = true;
    }
    *out = ctx;
    return LUX_OK;
}

extern "C" lux_status lux_context_destroy(LuxContext *ctx) {
    if (!ctx) return LUX_OK;
    if (ctx->scratch_mem) cudaFree(ctx->scratch_mem);
    if (ctx->owns_stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return LUX_OK;
}

extern "C" const char *lux_last_error_message(const LuxContext *ctx) {
    return ctx ? ctx->last_error.c_str() : "no context";
}

extern "C" lux_status lux_context_synchronize(LuxContext *ctx) {
    if (!ctx) return LUX_ERR_INVALID_ARGUMENT;
    return lux_cuda_check(ctx, (int)cudaStreamSynchronize(ctx->stream), "stream synchronize");
}

// RadianceCascades::default(), src/lib.rs:671-698 (temporal_blend 0.88,
// split_transmittance_blend 0.98, history_frames 24), plus the extension fields
// at the reference's fixed values (CASCADES = 4, BASE_THETA = 4, x4 ends).
extern "C" void lux_settings_default(LuxSettings *s) {
    if (!s) return;
    std::memset(s, 0, sizeof *s);
    s->probe_spacing = 0.25f;
    s->interval_length = 0.4f;
    s->normal_bias = 0.005f;
    s->intensity = 1.0f;
    s->exposure = 1.0f;
    s->emissive_samples = 16;
    s->levels = 4;
    s->base_columns = 8;
    s->base_rows = 4;
    s->interval_ratio = 4.0f;
    s->interval_rule = LUX_INTERVAL_ENDS_GEOMETRIC;
    s->layout = LUX_LAYOUT_SPLIT;
    s->rays_per_receiver = 1;
    s->frame_index = 0;
    s->resolve_scale = 1;
    s->temporal_blend = 0.88f;
    s->transmittance_blend = 0.98f;
    s->history_frames = 24;
}

// RadianceCascades::low_end(), src/lib.rs:700-722 (the fields this path reads).
extern "C" void lux_settings_low_end(LuxSettings *s) {
    if (!s) return;
    lux_settings_default(s);
    s->probe_spacing = 1.0f;
    s->interval_length = 1.6f;
    s->emissive_samples = 4;
    s->resolve_scale = 2;
    s->temporal_blend = 0.95f;
}

static float finite_clamp(float value, float fallback, float lo, float hi) {
    if (!std::isfinite(value)) return fallback;
    return value < lo ? lo : (value > hi ? hi : value);
}

static uint32_t clamp_u(uint32_t v, uint32_t lo, uint32_t hi) { return v < lo ? lo : (v > hi ? hi : v); }

// RadianceCascades::sanitized(), src/lib.rs:731-759 (blends clamped to
// 0.99 / 0.999, history_frames to 64); SamplingSettings
// resolve_scale clamp, src/lib.rs:388-407.
extern "C" void lux_settings_sanitize(LuxSettings *s) {
    if (!s) return;
    s->probe_spacing = finite_clamp(s->probe_spacing, 0.25f, 0.001f, 10000.0f);
    s->interval_length = finite_clamp(s->interval_length, 0.4f, 0.001f, 100000.0f);
    s->normal_bias = finite_clamp(s->normal_bias, 0.005f, 0.00001f, s->probe_spacing);
    s->intensity = finite_clamp(s->intensity, 1.0f, 0.0f, 100.0f);
    for (int c = 0; c < 3; ++c) s->environment[c] = finite_clamp(s->environment[c], 0.0f, 0.0f, 100000.0f);
    s->exposure = (std::isfinite(s->exposure) && s->exposure > 0.0f) ? s->exposure : 1.0f;
    s->emissive_samples = clamp_u(s->emissive_samples, 1, 32);
    s->resolve_scale = clamp_u(s->resolve_scale, 1, 8);
    s->levels = clamp_u(s->levels, 1, LUX_MAX_LEVELS);
    s->base_columns = clamp_u(s->base_columns, 1, 64);
    s->base_rows = clamp_u(s->base_rows, 1, 64);
    // The finest level's direction count must fit 32-bit indices.
    while (s->levels > 1 && ((uint64_t)s->base_columns * s->base_rows << (2 * (s->levels - 1))) > (1ull << 30))
        s->levels--;
    s->interval_ratio = finite_clamp(s->interval_ratio, 4.0f, 1.0f, 16.0f);
    if (s->interval_rule > LUX_INTERVAL_LENGTHS_GEOMETRIC) s->interval_rule = LUX_INTERVAL_ENDS_GEOMETRIC;
    if (s->layout > LUX_LAYOUT_DENSE) s->layout = LUX_LAYOUT_SPLIT;
    s->rays_per_receiver = clamp_u(s->rays_per_receiver, 1, 4096);
    s->temporal_blend = finite_clamp(s->temporal_blend, 0.88f, 0.0f, 0.99f);
    s->transmittance_blend = finite_clamp(s->transmittance_blend, 0.98f, 0.0f, 0.999f);
    s->history_frames = s->history_frames > 64u ? 64u : s->history_frames;
    s->multi_bounce = s->multi_bounce ? 1u : 0u;
    s->cached_hit_sky = s->cached_hit_sky && s->multi_bounce ? 1u : 0u;  // ignored without multi_bounce
}

// splitIntervalEnd, shaders/split.slang:224-227, generalised to a ratio and
// to geometric interval lengths.
extern "C" float lux_interval_end(const LuxSettings *s, uint32_t level) {
    if (!s) return 0.0f;
    if (s->interval_rule == LUX_INTERVAL_LENGTHS_GEOMETRIC) {
        float sum = 0.0f, term = 1.0f;
        for (uint32_t k = 0; k <= level; ++k) {
            sum += term;
            term *= s->interval_ratio;
        }
        return s->interval_length * sum;
    }
    float scale = 1.0f;
    for (uint32_t k = 0; k < level; ++k) scale *= s->interval_ratio;
    return s->interval_length * scale;
}

extern "C" uint32_t lux_direction_count(const LuxSettings *s, uint32_t level) {
    if (!s) return 0;
    return (s->base_columns << level) * (s->base_rows << level);
}
