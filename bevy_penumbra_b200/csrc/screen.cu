// screen.cu - screen reconstruction after the world resolve: the reference's
// temporal and denoise passes (shaders/cascades.slang:310-690, dispatched at
// src/render.rs:9836-9930) for the Split method's persistent world intervals.
//
// Temporal (one thread per pixel of the resolve extent): the current raw
// irradiance with its support alpha, a 3x3 same-surface neighbourhood mean
// and deviation, bilinear reprojection of the previous temporal output
// through the previous camera (validated by normal, raster identity, surface
// plane and the dirty box), variance clamping of the history and the
// persistent-interval blend by retained length and freshness.  Its output
// becomes the next frame's history.  Denoise: `spatial_filter_steps` passes
// of a 5x5 binomial kernel without its four far corners at strides 1, 2, 4,
// 8, weighted by normal^32, surface-plane distance and luminance against the
// temporal variance.
//
// Deviations (same in the oracle): positions come from the caller (world
// xyz with the view depth in w) instead of depth reconstruction, and the
// previous frame's positions are kept in the history instead of being
// reconstructed from the previous depth; no motion vectors (reprojection by
// the previous camera, the reference's static-world path); one summed source
// group, so the background channel, gradual-sun and source-change paths are
// not built; pow(x, 32) is five squarings.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "lux_internal.h"
#include "lux_math.cuh"

namespace {

struct ScreenParams {
    uint32_t width, height;
    float temporal_blend;    // history.x
    float capacity;          // history.w: history_frames
    float tolerance;         // surfaceTolerance: max(normal_bias * 2, probe_spacing * 0.02)
    float plane_scale;       // denoise: max(normal_bias * 2, probe_spacing * 0.05)
    uint32_t history_valid;  // stability.x
    uint32_t scene_changed;  // stability.y
    uint32_t dirty;
    float dirty_lo[3], dirty_hi[3];
    float prev[16];          // previous clip_from_world, row-major
    uint32_t step;           // denoise stride
};

// The screen history of one frame (the temporal output).
struct History {
    float4 *irr;   // rgb, depth or 0
    float4 *meta;  // retained length, variance, support mask, surface flag
    float4 *pos;   // world position, depth
    float4 *nrm;   // geometric normal
    uint2 *id;     // raster identity
};

struct Input {
    const float4 *irr, *pos, *nrm;
    const uint2 *id;
};

__device__ __forceinline__ float luminance(float3 c) { return (c.x * 0.2126f + c.y * 0.7152f) + c.z * 0.0722f; }

__device__ __forceinline__ float dot3(float4 a, float4 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

__device__ __forceinline__ bool finite3(float4 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

__device__ __forceinline__ float saturatef(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }

// surfacePlaneDistance, shaders/common.slang:585-591.
__device__ __forceinline__ float plane_distance(float4 delta, float4 target, float4 sample) {
    float4 avg = make_float4(target.x + sample.x, target.y + sample.y, target.z + sample.z, 0.0f);
    float len2 = dot3(avg, avg);
    if (!(len2 > 1e-20f) || !isfinite(len2)) return fabsf(dot3(delta, target));
    float inv = 1.0f / sqrtf(len2);
    float4 n = make_float4(avg.x * inv, avg.y * inv, avg.z * inv, 0.0f);
    return fabsf(dot3(delta, n));
}

// splitReceiverCompatible (shaders/cascades.slang:281-283): same raster
// surface (receiverSame) and normals within 0.97.
__device__ __forceinline__ bool compatible(bool a_surface, uint2 a_id, float4 a_n, bool b_surface, uint2 b_id,
                                           float4 b_n) {
    return a_surface && b_surface && a_id.x == b_id.x && a_id.y == b_id.y && dot3(a_n, b_n) > 0.97f;
}

__device__ __forceinline__ bool dirty_contains(const ScreenParams &P, float4 p) {
    return P.dirty && p.x >= P.dirty_lo[0] && p.y >= P.dirty_lo[1] && p.z >= P.dirty_lo[2] && p.x <= P.dirty_hi[0] &&
           p.y <= P.dirty_hi[1] && p.z <= P.dirty_hi[2];
}

__device__ __forceinline__ float lerpf(float a, float b, float t) { return a + t * (b - a); }

// temporal, shaders/cascades.slang:310-535 (persistent world intervals, no motion).
__global__ void __launch_bounds__(256) temporal_kernel(ScreenParams P, Input in, History H, History out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= (int)P.width || y >= (int)P.height) return;
    const size_t p = (size_t)y * P.width + x;
    float4 center = in.irr[p];
    const float4 position = in.pos[p];
    const float depth = position.w;
    if (!(depth > 0.0f)) {
        out.irr[p] = out.meta[p] = out.pos[p] = out.nrm[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        out.id[p] = make_uint2(0u, 0u);
        return;
    }
    const float4 gn = in.nrm[p];
    const uint2 id = in.id[p];
    bool current_finite = isfinite(center.w) && finite3(center);
    uint32_t current_mask = current_finite && center.w > 0.0f ? ((uint32_t)floorf(center.w) & 1u) : 0u;
    bool current_supported = current_mask != 0u && current_finite;
    float freshness = current_supported ? saturatef((center.w - floorf(center.w)) * 4.0f) : 0.0f;
    if (!current_supported) center.x = center.y = center.z = 0.0f;
    uint32_t output_mask = current_mask;
    // Same-surface 3x3 neighbourhood of the current raw values.
    float mx = 0.0f, my = 0.0f, mz = 0.0f, sx = 0.0f, sy = 0.0f, sz = 0.0f, count = 0.0f;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            int qx = x + dx, qy = y + dy;
            if (qx < 0 || qy < 0 || qx >= (int)P.width || qy >= (int)P.height) continue;
            size_t q = (size_t)qy * P.width + qx;
            float4 v = in.irr[q];
            if (v.w <= 0.0f) continue;
            uint32_t nmask = (uint32_t)floorf(v.w) & 1u;
            if (current_mask != 0u && nmask != current_mask) continue;
            float4 op = in.pos[q];
            if (op.w <= 0.0f) continue;
            float4 on = in.nrm[q];
            if (!compatible(true, id, gn, true, in.id[q], on)) continue;
            float4 delta = make_float4(op.x - position.x, op.y - position.y, op.z - position.z, 0.0f);
            if (dot3(gn, on) < 0.95f || plane_distance(delta, gn, on) > P.tolerance) continue;
            mx += v.x;
            my += v.y;
            mz += v.z;
            sx += v.x * v.x;
            sy += v.y * v.y;
            sz += v.z * v.z;
            count += 1.0f;
        }
    float cdiv = fmaxf(count, 1.0f);
    mx /= cdiv;
    my /= cdiv;
    mz /= cdiv;
    sx /= cdiv;
    sy /= cdiv;
    sz /= cdiv;
    float vx = fmaxf(0.0f, sx - mx * mx), vy = fmaxf(0.0f, sy - my * my), vz = fmaxf(0.0f, sz - mz * mz);
    float dvx = sqrtf(vx), dvy = sqrtf(vy), dvz = sqrtf(vz);
    // Reprojection through the previous camera.
    float4 hist = make_float4(0.0f, 0.0f, 0.0f, 0.0f), meta = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float total = 0.0f;
    uint32_t history_mask = 0u;
    const float *M = P.prev;
    float cx = ((M[0] * position.x + M[1] * position.y) + M[2] * position.z) + M[3];
    float cy = ((M[4] * position.x + M[5] * position.y) + M[6] * position.z) + M[7];
    float cw = ((M[12] * position.x + M[13] * position.y) + M[14] * position.z) + M[15];
    float u = (cx / cw) * 0.5f + 0.5f, v = 0.5f - (cy / cw) * 0.5f;
    bool projected = cw > 0.0f && isfinite(u) && isfinite(v);
    float px = u * (float)P.width, py = v * (float)P.height;
    if (projected && P.history_valid && !dirty_contains(P, position) && P.temporal_blend > 0.0f &&
        P.capacity > 0.0f && px >= 0.0f && py >= 0.0f && px < (float)P.width && py < (float)P.height) {
        float lx = px - 0.5f, ly = py - 0.5f;
        int bx = (int)floorf(lx), by = (int)floorf(ly);
        float lastx = (float)(P.width - 1u), lasty = (float)(P.height - 1u);
        float leftx = fminf((float)bx, lastx), lefty = fminf((float)by, lasty);
        float rightx = fminf((float)(bx + 1), lastx), righty = fminf((float)(by + 1), lasty);
        float fx = saturatef((lx - leftx) / fmaxf(rightx - leftx, 1.0f));
        float fy = saturatef((ly - lefty) / fmaxf(righty - lefty, 1.0f));
        for (int corner = 0; corner < 4; ++corner) {
            int ox = bx + (corner & 1), oy = by + (corner >> 1);
            if (ox < 0 || oy < 0 || ox >= (int)P.width || oy >= (int)P.height) continue;
            size_t o = (size_t)oy * P.width + ox;
            float4 old = H.irr[o], om = H.meta[o], onrm = H.nrm[o], opos = H.pos[o];
            if (om.x <= 0.0f || old.w <= 0.0f || !finite3(old) || dot3(gn, onrm) < 0.95f ||
                !compatible(true, id, gn, om.w > 0.0f, H.id[o], onrm))
                continue;
            if (dirty_contains(P, opos)) continue;
            float4 delta = make_float4(opos.x - position.x, opos.y - position.y, opos.z - position.z, 0.0f);
            if (plane_distance(delta, gn, onrm) > P.tolerance) continue;
            float wx = (corner & 1) ? fx : 1.0f - fx, wy = (corner >> 1) ? fy : 1.0f - fy;
            float weight = wx * wy;
            if (weight <= 0.0f) continue;
            if (om.z <= 0.0f) continue;  // no screen-history support
            history_mask = 1u;
            hist = make_float4(hist.x + old.x * weight, hist.y + old.y * weight, hist.z + old.z * weight,
                               hist.w + old.w * weight);
            meta = make_float4(meta.x + om.x * weight, meta.y + om.y * weight, meta.z + om.z * weight,
                               meta.w + om.w * weight);
            total += weight;
        }
    }
    const float capacity = fmaxf(P.capacity, 0.0f);
    float retained = current_supported ? freshness : 0.0f;
    float3 var3 = make_float3(vx, vy, vz);
    float out_var = current_supported ? luminance(var3) : 0.0f;
    if (total > 0.00001f) {
        hist = make_float4(hist.x / total, hist.y / total, hist.z / total, hist.w / total);
        meta = make_float4(meta.x / total, meta.y / total, meta.z / total, meta.w / total);
        output_mask = history_mask;
        float old_length = fminf(meta.x, capacity);
        float3 h3 = make_float3(hist.x, hist.y, hist.z);
        if (current_supported) {
            if (freshness <= 0.00001f) {
                center.x = hist.x;
                center.y = hist.y;
                center.z = hist.z;
                retained = old_length;
                out_var = meta.y;
            } else {
                bool complete = freshness >= 1.0f;
                float3 clipped = h3;
                if (count >= 2.0f && complete) {
                    float d = luminance(h3) - luminance(make_float3(center.x, center.y, center.z));
                    float tv = fmaxf(meta.y, d * d * 0.25f);
                    float st = sqrtf(tv);
                    float rx = 2.5f * fmaxf(dvx, st) + 0.0001f, ry = 2.5f * fmaxf(dvy, st) + 0.0001f,
                          rz = 2.5f * fmaxf(dvz, st) + 0.0001f;
                    clipped = make_float3(fminf(fmaxf(h3.x, fmaxf(0.0f, mx - rx)), mx + rx),
                                          fminf(fmaxf(h3.y, fmaxf(0.0f, my - ry)), my + ry),
                                          fminf(fmaxf(h3.z, fmaxf(0.0f, mz - rz)), mz + rz));
                }
                float hl = luminance(h3), cl = luminance(make_float3(center.x, center.y, center.z));
                float delta = hl - cl;
                float ll = luminance(clipped);
                float change = fabsf(ll - cl) / fmaxf(fmaxf(ll, cl), 0.001f);
                float reactive = P.scene_changed && complete ? 1.0f - change * change : 1.0f;
                float ref_l = fmaxf(fmaxf(hl, cl), 0.001f);
                float noise = sqrtf(fmaxf(meta.y, 0.0f)) / ref_l;
                float threshold = fminf(fmaxf(3.0f * noise, 0.05f), 0.25f);
                bool step = freshness > 0.0f && complete && P.scene_changed && change > threshold;
                if (step) old_length = 0.0f;
                float weight = fminf(P.temporal_blend, old_length / (old_length + 1.0f));
                weight = weight / fmaxf(weight + freshness * (1.0f - weight), 1e-8f);
                weight *= reactive;
                if (step) weight = 0.0f;
                center.x = lerpf(center.x, clipped.x, weight);
                center.y = lerpf(center.y, clipped.y, weight);
                center.z = lerpf(center.z, clipped.z, weight);
                retained = fminf(capacity, old_length + freshness);
                out_var = lerpf(luminance(var3), meta.y, weight) + (weight * (1.0f - weight)) * (delta * delta);
            }
        } else {
            center.x = hist.x;
            center.y = hist.y;
            center.z = hist.z;
            retained = old_length;
            out_var = meta.y;
        }
    }
    center.w = current_supported || retained > 0.0f ? depth : 0.0f;
    out.irr[p] = center;
    out.meta[p] = make_float4(retained, out_var, (float)output_mask, 1.0f);
    out.pos[p] = position;
    out.nrm[p] = gn;
    out.id[p] = id;
}

// denoise, shaders/cascades.slang:618-690: one a-trous pass at stride P.step.
// `src` / `src_mask` are the previous stage's irradiance and support masks;
// moments, identities and normals are the temporal output's.
//
// Every tap of a pixel lies on the pixel's lattice x = px + step u,
// y = py + step v, so a block takes 16 x 16 pixels of one lattice phase
// (px, py) and stages the lattice points they read (20 x 20 with the two-point
// halo) in shared memory once; each pixel then evaluates its taps in the same
// order and arithmetic as a direct read would.  Points outside the image are
// staged with zero irradiance support (w = 0), which skips them as the bounds
// test does.
constexpr int kDenoiseTile = 16, kDenoiseSpan = kDenoiseTile + 4;
__global__ void __launch_bounds__(256) denoise_kernel(ScreenParams P, Input in, History T, const float4 *src,
                                                      const float *src_mask, float4 *dst, float *dst_mask) {
    __shared__ float4 s_value[kDenoiseSpan * kDenoiseSpan], s_meta[kDenoiseSpan * kDenoiseSpan];
    __shared__ float4 s_nrm[kDenoiseSpan * kDenoiseSpan], s_pos[kDenoiseSpan * kDenoiseSpan];
    __shared__ uint2 s_id[kDenoiseSpan * kDenoiseSpan];
    __shared__ float s_mask[kDenoiseSpan * kDenoiseSpan];
    const int step = (int)P.step;
    const int px = (int)blockIdx.x % step, py = (int)blockIdx.y % step;  // lattice phase
    const int u0 = ((int)blockIdx.x / step) * kDenoiseTile, v0 = ((int)blockIdx.y / step) * kDenoiseTile;
    const int tid = threadIdx.y * kDenoiseTile + threadIdx.x;
    for (int k = tid; k < kDenoiseSpan * kDenoiseSpan; k += kDenoiseTile * kDenoiseTile) {
        int qx = px + step * (u0 - 2 + k % kDenoiseSpan), qy = py + step * (v0 - 2 + k / kDenoiseSpan);
        if (qx < 0 || qy < 0 || qx >= (int)P.width || qy >= (int)P.height) {
            s_value[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            continue;
        }
        size_t q = (size_t)qy * P.width + qx;
        s_value[k] = src[q];
        s_meta[k] = T.meta[q];
        s_nrm[k] = T.nrm[q];
        s_pos[k] = in.pos[q];
        s_id[k] = T.id[q];
        s_mask[k] = src_mask[q];
    }
    __syncthreads();
    const int x = px + step * (u0 + (int)threadIdx.x), y = py + step * (v0 + (int)threadIdx.y);
    if (x >= (int)P.width || y >= (int)P.height) return;
    const size_t p = (size_t)y * P.width + x;
    const int c = ((int)threadIdx.y + 2) * kDenoiseSpan + ((int)threadIdx.x + 2);
    float4 center = s_value[c];
    bool has_light = center.w > 0.0f && isfinite(center.w) && finite3(center);
    float4 position = s_pos[c];
    float depth = has_light ? center.w : position.w;
    if (depth <= 0.0f || !isfinite(depth)) {
        dst[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        dst_mask[p] = 0.0f;
        return;
    }
    const float4 tm = s_meta[c];
    const bool surface = tm.w > 0.0f;
    const uint2 id = s_id[c];
    const float4 gn = s_nrm[c];
    const uint32_t center_mask = (uint32_t)s_mask[c];
    const bool center_supported = tm.x > 0.0f;
    const float variance = fmaxf(tm.y, 0.0f);
    const float cl = luminance(make_float3(center.x, center.y, center.z));
    const float kernel[5] = {1.0f, 4.0f, 6.0f, 4.0f, 1.0f};
    float sx = 0.0f, sy = 0.0f, sz = 0.0f, total = 0.0f;
    for (int dy = -2; dy <= 2; ++dy) {
        int xr = abs(dy) == 2 ? 1 : 2;
        for (int dx = -xr; dx <= xr; ++dx) {
            const int q = c + dy * kDenoiseSpan + dx;
            float4 value = s_value[q];
            if (value.w <= 0.0f) continue;
            float4 om = s_meta[q];
            if (om.x <= 0.0f) continue;
            float4 on = s_nrm[q];
            if (!compatible(surface, id, gn, om.w > 0.0f, s_id[q], on)) continue;
            uint32_t other_mask = (uint32_t)s_mask[q];
            if (center_mask != 0u && other_mask != center_mask) continue;
            if (center_mask == 0u && other_mask == 0u) continue;
            float4 op = s_pos[q];
            if (dot3(gn, on) < 0.95f) continue;
            float4 delta = make_float4(op.x - position.x, op.y - position.y, op.z - position.z, 0.0f);
            float pd = plane_distance(delta, gn, on);
            if (pd > P.tolerance) continue;
            float cs = fmaxf(0.0f, dot3(gn, on));
            float c2 = cs * cs, c4 = c2 * c2, c8 = c4 * c4, c16 = c8 * c8, c32 = c16 * c16;
            float weight = ((kernel[dx + 2] * kernel[dy + 2]) * c32) * expf(-pd / P.plane_scale);
            if (center_supported) {
                float scale = fmaxf(0.02f, 2.0f * sqrtf(fmaxf(variance + om.y, 0.0f)));
                weight *= expf(-fabsf(luminance(make_float3(value.x, value.y, value.z)) - cl) / scale);
            }
            sx += value.x * weight;
            sy += value.y * weight;
            sz += value.z * weight;
            total += weight;
        }
    }
    bool filtered = total > 0.00001f;
    float4 out = filtered ? make_float4(sx / total, sy / total, sz / total, 0.0f) : center;
    float out_depth = has_light || center_supported || filtered ? depth : 0.0f;
    out.w = out_depth;
    dst[p] = out;
    dst_mask[p] = out_depth > 0.0f ? 1.0f : 0.0f;
}

__global__ void mask_kernel(uint32_t n, const float4 *meta, float *mask) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) mask[i] = meta[i].z;
}

}  // namespace

struct LuxScreen {
    LuxContext *ctx = nullptr;
    uint32_t width = 0, height = 0;
    History h[2] = {};
    int cur = 0;          // h[cur] holds the last temporal output
    bool valid = false;   // screen history exists
    float4 *ping = nullptr, *pong = nullptr;
    float *mask_ping = nullptr, *mask_pong = nullptr;
};

static void screen_free(LuxScreen *s) {
    for (int i = 0; i < 2; ++i) {
        void *p[] = {s->h[i].irr, s->h[i].meta, s->h[i].pos, s->h[i].nrm, s->h[i].id};
        for (void *q : p)
            if (q) cudaFree(q);
    }
    void *p[] = {s->ping, s->pong, s->mask_ping, s->mask_pong};
    for (void *q : p)
        if (q) cudaFree(q);
}

extern "C" lux_status lux_screen_create(LuxContext *ctx, uint32_t width, uint32_t height, LuxScreen **out) {
    if (!ctx || !out || width == 0 || height == 0) return LUX_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if ((uint64_t)width * height > (1ull << 28))
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "screen: more than 2^28 pixels");
    cudaSetDevice(ctx->device);
    LuxScreen *s = new LuxScreen();
    s->ctx = ctx;
    s->width = width;
    s->height = height;
    size_t n = (size_t)width * height;
    bool ok = true;
    for (int i = 0; i < 2 && ok; ++i)
        ok = cudaMalloc((void **)&s->h[i].irr, n * 16) == cudaSuccess &&
             cudaMalloc((void **)&s->h[i].meta, n * 16) == cudaSuccess &&
             cudaMalloc((void **)&s->h[i].pos, n * 16) == cudaSuccess &&
             cudaMalloc((void **)&s->h[i].nrm, n * 16) == cudaSuccess &&
             cudaMalloc((void **)&s->h[i].id, n * 8) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&s->ping, n * 16) == cudaSuccess &&
         cudaMalloc((void **)&s->pong, n * 16) == cudaSuccess &&
         cudaMalloc((void **)&s->mask_ping, n * 4) == cudaSuccess &&
         cudaMalloc((void **)&s->mask_pong, n * 4) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        screen_free(s);
        delete s;
        return lux_fail(ctx, LUX_ERR_OUT_OF_MEMORY, "screen: device allocation failed");
    }
    *out = s;
    return LUX_OK;
}

extern "C" lux_status lux_screen_destroy(LuxScreen *s) {
    if (!s) return LUX_OK;
    cudaSetDevice(s->ctx->device);
    screen_free(s);
    delete s;
    return LUX_OK;
}

extern "C" lux_status lux_screen_reset(LuxScreen *s) {
    if (!s) return LUX_ERR_INVALID_ARGUMENT;
    s->valid = false;
    return LUX_OK;
}

extern "C" lux_status lux_screen_filter(LuxScreen *s, const LuxSettings *settings, const LuxScreenFrame *f,
                                        float *out) {
    if (!s || !settings || !f || !out || !f->irradiance || !f->position || !f->normal || !f->identity)
        return LUX_ERR_INVALID_ARGUMENT;
    LuxContext *ctx = s->ctx;
    if (f->spatial_filter_steps > 4)
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "screen: spatial_filter_steps above 4");
    LuxSettings st = *settings;
    lux_settings_sanitize(&st);
    cudaSetDevice(ctx->device);
    ScreenParams P;
    std::memset(&P, 0, sizeof P);
    P.width = s->width;
    P.height = s->height;
    P.temporal_blend = st.temporal_blend;
    P.capacity = (float)st.history_frames;
    P.tolerance = fmaxf(st.normal_bias * 2.0f, st.probe_spacing * 0.02f);
    P.plane_scale = fmaxf(st.normal_bias * 2.0f, st.probe_spacing * 0.05f);
    P.history_valid = s->valid ? 1u : 0u;
    P.scene_changed = f->scene_changed ? 1u : 0u;
    P.dirty = f->dirty ? 1u : 0u;
    for (int a = 0; a < 3; ++a) {
        P.dirty_lo[a] = f->dirty_lo[a];
        P.dirty_hi[a] = f->dirty_hi[a];
    }
    std::memcpy(P.prev, f->previous_clip_from_world, sizeof P.prev);
    Input in{(const float4 *)f->irradiance, (const float4 *)f->position, (const float4 *)f->normal,
             (const uint2 *)f->identity};
    cudaStream_t stream = ctx->stream;
    dim3 block(16, 16), grid((s->width + 15) / 16, (s->height + 15) / 16);
    History &prev = s->h[s->cur], &next = s->h[1 - s->cur];
    temporal_kernel<<<grid, block, 0, stream>>>(P, in, prev, next);
    s->cur = 1 - s->cur;
    s->valid = true;
    const History &T = s->h[s->cur];
    const size_t n = (size_t)s->width * s->height;
    if (f->spatial_filter_steps == 0) {
        cudaMemcpyAsync(out, T.irr, n * 16, cudaMemcpyDeviceToDevice, stream);
        return lux_cuda_check(ctx, (int)cudaGetLastError(), "screen temporal");
    }
    // Pass 0 reads the temporal output; later passes ping-pong; the last
    // pass writes `out`.
    mask_kernel<<<(uint32_t)((n + 255) / 256), 256, 0, stream>>>((uint32_t)n, T.meta, s->mask_ping);
    const float4 *src = T.irr;
    const float *src_mask = s->mask_ping;
    for (uint32_t level = 0; level < f->spatial_filter_steps; ++level) {
        P.step = level == 0 ? 1u : (1u << level);
        bool last = level + 1 == f->spatial_filter_steps;
        float4 *dst = last ? (float4 *)out : (level % 2 == 0 ? s->ping : s->pong);
        float *dst_mask = src_mask == s->mask_ping ? s->mask_pong : s->mask_ping;
        // Blocks of 16 x 16 pixels of one lattice phase, step x step phases.
        const uint32_t lu = (s->width + P.step - 1) / P.step, lv = (s->height + P.step - 1) / P.step;
        dim3 lattice(P.step * ((lu + kDenoiseTile - 1) / kDenoiseTile), P.step * ((lv + kDenoiseTile - 1) / kDenoiseTile));
        denoise_kernel<<<lattice, block, 0, stream>>>(P, in, T, src, src_mask, dst, dst_mask);
        src = dst;
        src_mask = dst_mask;
    }
    return lux_cuda_check(ctx, (int)cudaGetLastError(), "screen filter");
}

extern "C" lux_status lux_screen_read_history(LuxScreen *s, float *irradiance, float *metadata) {
    if (!s) return LUX_ERR_INVALID_ARGUMENT;
    LuxContext *ctx = s->ctx;
    cudaSetDevice(ctx->device);
    size_t n = (size_t)s->width * s->height;
    lux_status st = lux_cuda_check(ctx, (int)cudaStreamSynchronize(ctx->stream), "screen read");
    if (st != LUX_OK) return st;
    const History &T = s->h[s->cur];
    if (irradiance && cudaMemcpy(irradiance, T.irr, n * 16, cudaMemcpyDeviceToHost) != cudaSuccess)
        return lux_cuda_check(ctx, (int)cudaGetLastError(), "screen read irradiance");
    if (metadata && cudaMemcpy(metadata, T.meta, n * 16, cudaMemcpyDeviceToHost) != cudaSuccess)
        return lux_cuda_check(ctx, (int)cudaGetLastError(), "screen read metadata");
    return LUX_OK;
}
