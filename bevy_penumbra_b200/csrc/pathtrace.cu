// pathtrace.cu - FP64-accumulated path-traced reference irradiance.
//
// The quality oracle of the error reports: the reference project's offline
// path tracer (trace_sample, examples/pathtrace_reference.rs:724-833) run from
// the cascades' receivers.  At every diffuse vertex one emissive-triangle
// next-event sample (light CDF, area pdf converted to solid angle) weighted
// against the cosine proposal by the power heuristic, then a cosine-proposed
// continuation whose emitter hits carry the complementary weight; the last
// vertex takes the next-event sample alone (no competing BSDF ray is traced
// there); Russian roulette from the fourth vertex on.  The receiver vertex is
// Lambertian with unit albedo, so the estimate is irradiance / pi before the
// receiver's albedo, the cascades' raw output; later vertices scatter with
// the hit's diffuse colour and disneyDiffuseMultiplier (the hit shading of
// the cascade rays).  Rays are traced in FP32 by the library's traversal;
// every sample's radiance is summed per point in FP64.  Samples whose traces
// are unsupported (step budget) are left out of the mean.
#include <cuda_runtime.h>

#include <algorithm>

#include "lux_internal.h"
#include "lux_math.cuh"
#include "shade.cuh"
#include "traverse.cuh"

namespace {

using lux::f3;

constexpr uint32_t kPathChunk = 32;  // samples one thread sums before its FP64 atomics
constexpr uint32_t kDimsPerVertex = 6;

struct PathParams {
    lux::ShadeParams shade;  // exposure, normal bias, environment
    uint32_t spp, bounces, seed;
};

// A scattering vertex: position, shading normal, geometric normal facing the
// incoming ray, direction back along it, diffuse colour and roughness.  The
// receiver vertex is Lambertian with unit albedo.
struct Vertex {
    f3 position, normal, gnormal, view, diffuse;
    float roughness;
    bool lambert;
};

__device__ __forceinline__ float power_heuristic(float a, float b) {
    float aa = a * a;
    return aa / fmaxf(aa + b * b, 1e-30f);
}

// BSDF value without the cosine: 1 / pi at the receiver, diffuse x
// disneyDiffuseMultiplier / pi elsewhere.
__device__ __forceinline__ f3 response(const Vertex &v, f3 l) {
    if (v.lambert) return f3{1.0f / lux::kPi, 1.0f / lux::kPi, 1.0f / lux::kPi};
    float factor = lux::disney_multiplier(v.normal, l, v.view, v.roughness) / lux::kPi;
    return f3{v.diffuse.x * factor, v.diffuse.y * factor, v.diffuse.z * factor};
}

// Index (among the emissive records) of the record of triangle `tri` of
// instance slot `inst`, or kEmpty: the records are ordered by (slot, triangle).
__device__ uint32_t light_of(const SceneView &S, uint32_t inst, uint32_t tri) {
    const LuxLight *L = S.lights + S.conventional_lights;
    uint32_t lo = 0, hi = S.emissive_lights;
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2u;
        uint32_t a = __ldg(&L[mid].source[0]), b = __ldg(&L[mid].source[1]);
        if (a < inst || (a == inst && b < tri))
            lo = mid + 1u;
        else
            hi = mid;
    }
    if (lo < S.emissive_lights && __ldg(&L[lo].source[0]) == inst && __ldg(&L[lo].source[1]) == tri) return lo;
    return lux::kEmpty;
}

// One next-event sample at `v` (selection u0, triangle point u1, u2); false
// when its visibility query is unsupported.
__device__ bool next_event(const SceneView &S, const PathParams &P, const Vertex &v, float u0, float u1, float u2,
                           bool competitor, f3 &out, lux::TraceCounters &cn) {
    out = f3{0.0f, 0.0f, 0.0f};
    const uint32_t emissive = S.emissive_lights;
    if (emissive == 0u) return true;
    const LuxLight *lights = S.lights + S.conventional_lights;
    uint32_t low = 0, high = emissive - 1u;
    while (low < high) {
        uint32_t middle = (low + high) / 2u;
        if (__ldg(&lights[middle].direction[3]) < u0)
            low = middle + 1u;
        else
            high = middle;
    }
    const LuxLight *L = lights + low;
    const float bias = P.shade.normal_bias;
    f3 lp{__ldg(&L->position[0]), __ldg(&L->position[1]), __ldg(&L->position[2])};
    float lpw = __ldg(&L->position[3]);
    f3 ldir{__ldg(&L->direction[0]), __ldg(&L->direction[1]), __ldg(&L->direction[2])};
    f3 e1{__ldg(&L->edge1[0]), __ldg(&L->edge1[1]), __ldg(&L->edge1[2])};
    float prob = __ldg(&L->edge1[3]);
    f3 e2{__ldg(&L->edge2[0]), __ldg(&L->edge2[1]), __ldg(&L->edge2[2])};
    float area = __ldg(&L->color[3]);
    f3 rel = v.position - lp;
    if (prob <= 0.0f || (lpw != -2.0f && lux::dot(ldir, rel) <= 0.0f)) return true;
    float root = sqrtf(u1);
    float w1 = root * (1.0f - u2), w2 = root * u2;
    f3 target{(lp.x + e1.x * w1) + e2.x * w2, (lp.y + e1.y * w1) + e2.y * w2, (lp.z + e1.z * w1) + e2.z * w2};
    f3 to_light = target - v.position;
    float light_distance = lux::length(to_light);
    if (light_distance <= bias * 0.25f) return true;
    f3 ld = to_light / light_distance;
    float cosine = fmaxf(0.0f, lux::dot(v.normal, ld));
    float c_emit = lux::dot(ldir, -ld);
    if (lpw == -2.0f) c_emit = fabsf(c_emit);
    float emitter_cosine = fmaxf(0.0f, c_emit);
    if (cosine <= 0.0f || emitter_cosine <= 0.0f || lux::dot(v.gnormal, ld) <= 0.0f) return true;
    lux::Surface es = lux::surface_at(S, P.shade, __ldg(&L->source[0]), __ldg(&L->source[1]), 1.0f - root, w1, w2);
    f3 emission{fmaxf(es.emission.x, 0.0f), fmaxf(es.emission.y, 0.0f), fmaxf(es.emission.z, 0.0f)};
    if (!(emission.x > 0.0f || emission.y > 0.0f || emission.z > 0.0f)) return true;
    float pdf = ((prob * light_distance) * light_distance) / (area * emitter_cosine);
    float plane = fabsf(lux::dot(ldir, rel));
    f3 origin = lux::ray_offset(v.position, v.gnormal, fminf(bias, plane * 0.25f));
    f3 delta = target - origin;
    float distance = lux::length(delta);
    if (distance <= bias * 0.25f) return true;
    lux::Hit sh;
    lux::trace<true>(S, origin, delta / distance, 0.0f, distance - fminf(bias * 0.25f, distance * 0.001f), sh, cn);
    if (sh.tri != lux::kEmpty) return true;                       // blocked
    if ((sh.errors & lux::kQueryUnsupported) != 0u) return false;  // step budget exhausted
    f3 f = response(v, ld);
    float mis = competitor ? power_heuristic(pdf, cosine / lux::kPi) : 1.0f;
    float p = fmaxf(pdf, 1e-20f);
    out = f3{emission.x * (((f.x * cosine) / p) * mis), emission.y * (((f.y * cosine) / p) * mis),
             emission.z * (((f.z * cosine) / p) * mis)};
    return true;
}

// The vertex at a closest hit (hitAttributes / materialNormal as the
// cascades' hit shading, shaders/traversal.slang:258-282,
// shaders/material.slang:171-177).  emission: the hit's own emission (>= 0);
// returns whether the surface scatters light on.
__device__ bool hit_vertex(const SceneView &S, const PathParams &P, f3 origin, f3 direction, const lux::Hit &hit,
                           Vertex &v, f3 &emission) {
    float b0 = (1.0f - hit.b1) - hit.b2;
    lux::Surface sf = lux::surface_at(S, P.shade, hit.inst, hit.tri, b0, hit.b1, hit.b2);
    emission = f3{fmaxf(sf.emission.x, 0.0f), fmaxf(sf.emission.y, 0.0f), fmaxf(sf.emission.z, 0.0f)};
    if (!lux::finite3(emission)) emission = f3{0.0f, 0.0f, 0.0f};
    if ((sf.flags & 16u) != 0u) return false;  // unlit: emits its base colour, scatters nothing
    uint32_t ibase = lux::instance_base(S, hit.inst);
    uint4 header = lux::gword(S, 0);
    uint4 t = lux::gword(S, header.x + hit.tri);
    uint32_t idx[3] = {t.x, t.y, t.z};
    f3 A = lux::f3w(lux::gword(S, header.y + idx[0] * header.z));
    f3 B = lux::f3w(lux::gword(S, header.y + idx[1] * header.z));
    f3 C = lux::f3w(lux::gword(S, header.y + idx[2] * header.z));
    f3 position{origin.x + direction.x * hit.t, origin.y + direction.y * hit.t, origin.z + direction.z * hit.t};
    f3 gn = lux::unit_vector(lux::transform_direction_t(S, ibase, lux::cross(B - A, C - A)), f3{0.0f, 1.0f, 0.0f});
    gn = gn * ((sf.flags & 4u) != 0u ? -1.0f : 1.0f);
    float bary[3] = {b0, hit.b1, hit.b2};
    f3 world_normal{0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        uint32_t vb = header.y + idx[i] * header.z;
        f3 nrm = gn;
        if ((lux::gword(S, vb).w & 1u) != 0u)
            nrm = lux::unit_vector(lux::transform_direction_t(S, ibase, lux::f3w(lux::gword(S, vb + 1))), gn);
        world_normal = f3{world_normal.x + nrm.x * bary[i], world_normal.y + nrm.y * bary[i],
                          world_normal.z + nrm.z * bary[i]};
    }
    f3 normal = lux::unit_vector(world_normal, gn);
    if (lux::dot(gn, direction) > 0.0f && (sf.flags & 8u) != 0u) normal = -normal;
    f3 flipped = lux::dot(gn, direction) > 0.0f ? -gn : gn;
    f3 neg = -direction;
    if (lux::dot(normal, neg) <= 0.0f || lux::dot(normal, flipped) <= 0.0f) return false;
    float nl = lux::length(neg);
    float metallic = lux::saturate(sf.metallic);
    float roughness = lux::saturate(sf.roughness);
    if (!isfinite(roughness)) roughness = 1.0f;
    bool bf = lux::finite3(sf.base_color);
    v.position = position;
    v.normal = normal;
    v.gnormal = flipped;
    v.view = neg / nl;
    v.diffuse = f3{(bf ? lux::saturate(sf.base_color.x) : 0.0f) * (1.0f - metallic),
                   (bf ? lux::saturate(sf.base_color.y) : 0.0f) * (1.0f - metallic),
                   (bf ? lux::saturate(sf.base_color.z) : 0.0f) * (1.0f - metallic)};
    v.roughness = roughness;
    v.lambert = false;
    return lux::finite3(position) && (v.diffuse.x > 0.0f || v.diffuse.y > 0.0f || v.diffuse.z > 0.0f);
}

// One path from receiver p (sample s); false when a trace was unsupported.
__device__ bool path_sample(const SceneView &S, const PathParams &P, uint32_t p, f3 pos, f3 nrm, uint32_t s,
                            f3 &radiance, lux::TraceCounters &cn) {
    radiance = f3{0.0f, 0.0f, 0.0f};
    f3 throughput{1.0f, 1.0f, 1.0f};
    Vertex v;
    v.position = pos;
    v.normal = nrm;
    v.gnormal = nrm;
    v.view = nrm;
    v.diffuse = f3{1.0f, 1.0f, 1.0f};
    v.roughness = 1.0f;
    v.lambert = true;
    const float bias = P.shade.normal_bias;
    for (uint32_t bounce = 0; bounce < P.bounces; ++bounce) {
        const uint32_t dim = bounce * kDimsPerVertex;
        const bool competitor = bounce + 1u < P.bounces;
        f3 c;
        if (!next_event(S, P, v, lux::path_random(p, s, P.seed, dim), lux::path_random(p, s, P.seed, dim + 1u),
                        lux::path_random(p, s, P.seed, dim + 2u), competitor, c, cn))
            return false;
        radiance = radiance + throughput * c;
        if (!competitor) break;
        f3 d = lux::cosine_direction(v.normal, lux::path_random(p, s, P.seed, dim + 3u),
                                     lux::path_random(p, s, P.seed, dim + 4u));
        float cosine = lux::dot(v.normal, d);
        if (!(cosine > 0.0f) || lux::dot(v.gnormal, d) <= 0.0f) break;
        float pdf = cosine / lux::kPi;
        f3 f = response(v, d);
        throughput = f3{throughput.x * ((f.x * cosine) / pdf), throughput.y * ((f.y * cosine) / pdf),
                        throughput.z * ((f.z * cosine) / pdf)};
        if (bounce >= 3u) {
            float survival = fminf(fmaxf(fmaxf(throughput.x, fmaxf(throughput.y, throughput.z)), 0.05f), 0.95f);
            if (lux::path_random(p, s, P.seed, dim + 5u) >= survival) break;
            throughput = throughput / survival;
        }
        f3 origin = lux::ray_offset(v.position, v.gnormal, bias);
        lux::Hit hit;
        lux::trace<false>(S, origin, d, 0.0f, 1e20f, hit, cn);
        if ((hit.errors & lux::kQueryUnsupported) != 0u) return false;
        if (hit.tri == lux::kEmpty) {
            radiance = radiance + throughput * P.shade.environment;
            break;
        }
        Vertex next;
        f3 emission;
        bool scatters = hit_vertex(S, P, origin, d, hit, next, emission);
        if (emission.x > 0.0f || emission.y > 0.0f || emission.z > 0.0f) {
            // The emitter's next-event pdf of this direction for the weight.
            float mis = 1.0f;
            uint32_t li = light_of(S, hit.inst, hit.tri);
            if (li != lux::kEmpty) {
                const LuxLight *L = S.lights + S.conventional_lights + li;
                f3 ldir{__ldg(&L->direction[0]), __ldg(&L->direction[1]), __ldg(&L->direction[2])};
                float c_emit = lux::dot(ldir, -d);
                if (__ldg(&L->position[3]) == -2.0f) c_emit = fabsf(c_emit);
                float area = __ldg(&L->color[3]), prob = __ldg(&L->edge1[3]);
                if (c_emit > 0.0f && area > 0.0f && prob > 0.0f)
                    mis = power_heuristic(pdf, ((prob * hit.t) * hit.t) / (area * c_emit));
            }
            radiance = radiance + (throughput * emission) * mis;
        }
        if (!scatters) break;
        v = next;
    }
    if (!lux::finite3(radiance)) radiance = f3{0.0f, 0.0f, 0.0f};
    return true;
}

__global__ void __launch_bounds__(128) path_kernel(SceneView S, PathParams P, const float4 *__restrict__ pos,
                                                   const float4 *__restrict__ nrm, uint32_t count,
                                                   double *__restrict__ acc) {
    const uint32_t chunks = (P.spp + kPathChunk - 1u) / kPathChunk;
    const unsigned long long total = (unsigned long long)count * chunks;
    lux::TraceCounters cn{0, 0, 0};
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < total;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        uint32_t p = (uint32_t)(i / chunks), c = (uint32_t)(i % chunks);
        float4 p4 = pos[p], n4 = nrm[p];
        f3 P0{p4.x, p4.y, p4.z}, N0{n4.x, n4.y, n4.z};
        double sx = 0.0, sy = 0.0, sz = 0.0, n = 0.0;
        const uint32_t s_end = min(P.spp, (c + 1u) * kPathChunk);
        for (uint32_t s = c * kPathChunk; s < s_end; ++s) {
            f3 r;
            if (!path_sample(S, P, p, P0, N0, s, r, cn)) continue;
            sx += (double)r.x;
            sy += (double)r.y;
            sz += (double)r.z;
            n += 1.0;
        }
        atomicAdd(acc + 4 * (size_t)p + 0, sx);
        atomicAdd(acc + 4 * (size_t)p + 1, sy);
        atomicAdd(acc + 4 * (size_t)p + 2, sz);
        atomicAdd(acc + 4 * (size_t)p + 3, n);
    }
}

__global__ void path_finish_kernel(double4 *__restrict__ acc, uint32_t count) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    double4 a = acc[p];
    acc[p] = a.w > 0.0 ? make_double4(a.x / a.w, a.y / a.w, a.z / a.w, a.w) : make_double4(0.0, 0.0, 0.0, 0.0);
}

}  // namespace

extern "C" lux_status lux_path_reference(LuxContext *ctx, const LuxScene *scene, const LuxSettings *settings,
                                         const float *position, const float *normal, uint32_t count, uint32_t spp,
                                         uint32_t bounces, uint32_t seed, double *out) {
    if (!ctx || !scene || !settings || (count && (!position || !normal || !out))) return LUX_ERR_INVALID_ARGUMENT;
    if (count == 0) return LUX_OK;
    if (spp == 0 || bounces == 0 || bounces > 16)
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "path reference: spp must be positive, bounces 1..16");
    LuxSettings s = *settings;
    lux_settings_sanitize(&s);
    PathParams P{};
    P.shade.normal_bias = s.normal_bias;
    P.shade.exposure = s.exposure;
    P.shade.environment = f3{s.environment[0], s.environment[1], s.environment[2]};
    P.spp = spp;
    P.bounces = bounces;
    P.seed = seed;
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    lux_status rc = lux_cuda_check(ctx, (int)cudaMemsetAsync(out, 0, (size_t)count * 4 * sizeof(double), st),
                                   "path reference: clear");
    if (rc != LUX_OK) return rc;
    const unsigned long long total = (unsigned long long)count * ((spp + kPathChunk - 1u) / kPathChunk);
    const unsigned long long blocks = std::min<unsigned long long>((total + 127ull) / 128ull, (unsigned long long)ctx->sm_count * 64ull);
    path_kernel<<<(uint32_t)blocks, 128, 0, st>>>(scene->view, P, (const float4 *)position, (const float4 *)normal,
                                                  count, out);
    path_finish_kernel<<<(count + 127) / 128, 128, 0, st>>>((double4 *)out, count);
    return lux_cuda_check(ctx, (int)cudaGetLastError(), "path reference launch");
}
