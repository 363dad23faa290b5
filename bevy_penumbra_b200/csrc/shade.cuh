// shade.cuh - interval radiance at a hit: outgoingTransportRadianceTracked
// (shaders/cascades.slang:196-268) with emissive next-event estimation
// (emissiveResponseTracked, shaders/cascades.slang:57-134).
//
// Synthetic-material subset, identical to the CPU oracle: untextured opaque
// materials (materialSample = 1); a constant environment (no environment
// map) with cosine-proposal visibility rays (environmentResponseTracked,
// shaders/environment.slang:154-230); conventional
// (point, spot, directional) lights with visibility rays
// (conventionalLightResponseTracked, shaders/cascades.slang:136-176).  With
// multi-bounce on, the secondary cache's
// irradiance of the previous frame adds diffuse bounce light (secondaryFeedback,
// shaders/world_resolve.slang:204-279), and the secondary cache's own hits
// leave out their emission (environmentScale.z).  All source groups are
// summed into one radiance.  The scattering response is the diffuse colour
// times disneyDiffuseMultiplier / pi (shaders/common.slang:298-314 and the
// non-full branch of scatteringResponse, shaders/environment.slang:2-6).
#pragma once
#include "traverse.cuh"

namespace lux {

// The secondary cache's cascade-0 probes of the previous frame: a directory
// of cell keys (open addressing, lux::hash_key with level 0) and the packed
// 6x6 irradiance table of each cell.
struct Feedback {
    const unsigned long long *keys;  // [capacity] packed cell keys (kEmptyCell: free)
    const uint32_t *ids;             // [capacity] table of each slot's cell
    const float4 *tables;            // [cells][36]
    uint32_t capacity;               // power of two
    float spacing;                   // the secondary cache's cascade-0 spacing
};

struct ShadeParams {
    float probe_spacing;
    float normal_bias;
    float exposure;
    uint32_t emissive_samples;
    uint32_t frame;
    uint32_t skip_emission;  // secondary cache: no first-hit emission (next-event estimation carries it)
    uint32_t feedback;       // 1: add diffuse x the secondary cache's irradiance at the hit
    Feedback fb;
    f3 environment;          // constant environment radiance (black: no environment samples)
    uint32_t cached_sky;     // cachedHitSky: escapes of the secondary cache carry the environment, and hits
                             // the feedback probes cover take no environment samples
};

// environmentResponseTracked returns early for a black constant environment.
__device__ __forceinline__ bool environment_on(const ShadeParams &P) {
    return P.environment.x > 0.0f || P.environment.y > 0.0f || P.environment.z > 0.0f;
}

__device__ __forceinline__ uint4 sword(const SceneView &S, uint32_t i) {
    i = i < S.scene_word_count ? i : S.scene_word_count - 1u;
    return __ldg(S.scene_words + i);
}
__device__ __forceinline__ uint4 gword(const SceneView &S, uint32_t i) {
    i = i < S.geometry_word_count ? i : S.geometry_word_count - 1u;
    return __ldg(S.geometry_words + i);
}
__device__ __forceinline__ f3 f3w(uint4 w) { return f3{as_float(w.x), as_float(w.y), as_float(w.z)}; }

// unitVector, shaders/traversal.slang:183-190.
__device__ __forceinline__ f3 unit_vector(f3 v, f3 fallback) {
    float scale = fmaxf(fabsf(v.x), fmaxf(fabsf(v.y), fabsf(v.z)));
    if (scale == 0.0f || !isfinite(scale)) return fallback;
    float div = fmaxf(scale * 0.25f, 1.17549435e-38f);
    f3 w{v.x / div, v.y / div, v.z / div};
    float l = length(w);
    return f3{w.x / l, w.y / l, w.z / l};
}

// transformDirection, shaders/traversal.slang:229-244 (transpose form).
__device__ __forceinline__ f3 transform_direction_t(const SceneView &S, uint32_t base, f3 value) {
    f3 a = f3w(sword(S, base)), b = f3w(sword(S, base + 1)), c = f3w(sword(S, base + 2));
    f3 mag{fmaxf(fabsf(a.x), fmaxf(fabsf(b.x), fabsf(c.x))), fmaxf(fabsf(a.y), fmaxf(fabsf(b.y), fabsf(c.y))),
           fmaxf(fabsf(a.z), fmaxf(fabsf(b.z), fabsf(c.z)))};
    float scale = fmaxf(mag.x, fmaxf(mag.y, mag.z));
    if (scale == 0.0f) return f3{0.0f, 0.0f, 0.0f};
    scale = fmaxf(scale * 0.25f, 1.17549435e-38f);
    a = a / scale;
    b = b / scale;
    c = c / scale;
    f3 v = unit_vector(value, f3{0.0f, 0.0f, 0.0f});
    return f3{(a.x * v.x + b.x * v.y) + c.x * v.z, (a.y * v.x + b.y * v.y) + c.y * v.z,
              (a.z * v.x + b.z * v.y) + c.z * v.z};
}

struct Surface {
    f3 base_color;
    f3 emission;
    float metallic, roughness;
    uint32_t flags;
};

__device__ __forceinline__ uint32_t instance_base(const SceneView &S, uint32_t inst) {
    uint4 h = sword(S, 0);
    return h.y + inst * h.w;
}

// materialBaseColor / hitEmission (shaders/material.slang:139-141,
// shaders/traversal.slang:287-300), untextured.
__device__ __forceinline__ Surface surface_at(const SceneView &S, const ShadeParams &P, uint32_t inst, uint32_t tri,
                                              float b0, float b1, float b2) {
    uint32_t base = instance_base(S, inst);
    uint32_t flags = sword(S, base + 6).w;
    uint32_t material = sword(S, base + 7).w;
    uint4 m0 = sword(S, material), m1 = sword(S, material + 1), m2 = sword(S, material + 2);
    uint4 header = gword(S, 0);
    uint4 t = gword(S, header.x + tri);
    uint4 c0 = gword(S, header.y + t.x * header.z + 4);
    uint4 c1 = gword(S, header.y + t.y * header.z + 4);
    uint4 c2 = gword(S, header.y + t.z * header.z + 4);
    f3 color{(as_float(c0.x) * b0 + as_float(c1.x) * b1) + as_float(c2.x) * b2,
             (as_float(c0.y) * b0 + as_float(c1.y) * b1) + as_float(c2.y) * b2,
             (as_float(c0.z) * b0 + as_float(c1.z) * b1) + as_float(c2.z) * b2};
    Surface sf;
    sf.base_color = f3{as_float(m0.x) * color.x, as_float(m0.y) * color.y, as_float(m0.z) * color.z};
    sf.emission = (flags & 16u) != 0u ? sf.base_color : f3{as_float(m1.x), as_float(m1.y), as_float(m1.z)};
    float weight = (flags & 16u) != 0u ? 0.0f : as_float(m2.w);
    float exposure = fmaxf(P.exposure, 1e-20f);
    float inv = 1.0f / exposure;
    float factor = inv + weight * (1.0f - inv);
    sf.emission = sf.emission * factor;
    sf.metallic = as_float(m2.x);
    sf.roughness = as_float(m2.y);
    sf.flags = flags;
    return sf;
}

// disneyDiffuseMultiplier, shaders/common.slang:298-314.
__device__ __forceinline__ float disney_multiplier(f3 n, f3 l, f3 v, float pr) {
    float ndl = saturate(dot(n, l));
    float ndv = saturate(dot(n, v));
    f3 h = l + v;
    float hl2 = dot(h, h);
    if (ndl <= 0.0f || ndv <= 0.0f || hl2 <= 1e-20f) return 0.0f;
    float hl = sqrtf(hl2);
    f3 hv{h.x / hl, h.y / hl, h.z / hl};
    float rough = fmaxf(saturate(pr), 0.089f);
    rough = rough * rough;
    float ldh = saturate(dot(l, hv));
    float f90 = 0.5f + ((2.0f * rough) * ldh) * ldh;
    float a = 1.0f - ndl, b = 1.0f - ndv;
    float a2 = a * a, bb = b * b;
    float ls = 1.0f + (f90 - 1.0f) * ((a2 * a2) * a);
    float vs = 1.0f + (f90 - 1.0f) * ((bb * bb) * b);
    return ls * vs;
}

// irradianceLookup + diffuseProbePage (shaders/world_resolve.slang:27-89)
// on one packed table: rgb and coverage.
__device__ __forceinline__ float4 probe_irradiance(const float4 *__restrict__ table, f3 normal) {
    float ex, ey;
    encode_normal(normal, ex, ey);
    float gx = ex * 6.0f - 0.5f, gy = ey * 6.0f - 0.5f;
    float bxf = floorf(gx), byf = floorf(gy);
    float fx = gx - bxf, fy = gy - byf;
    float cx = 1.0f - fx, cy = 1.0f - fy;
    float weight[4] = {cx * cy, fx * cy, cx * fy, fx * fy};
    int32_t ix = (int32_t)bxf, iy = (int32_t)byf;
    uint32_t texel[4] = {texel_index(ix, iy), texel_index(ix + 1, iy), texel_index(ix, iy + 1),
                         texel_index(ix + 1, iy + 1)};
    float px = 0.0f, py = 0.0f, pz = 0.0f, obs = 0.0f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float bw = weight[c];
        if (!(bw > 0.0f)) continue;
        float4 t = __ldg(table + texel[c]);
        if (!(t.w > 0.0f) || !(isfinite(t.x) && isfinite(t.y) && isfinite(t.z) && isfinite(t.w))) continue;
        float w = bw * saturate(t.w);
        px = px + t.x * w;
        py = py + t.y * w;
        pz = pz + t.z * w;
        obs += w;
    }
    return obs > 0.0f ? make_float4(px / obs, py / obs, pz / obs, saturate(obs)) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// secondaryFeedback (shaders/world_resolve.slang:204-279) at one LOD: the
// previous frame's secondary probe of the cell holding `position`, looked up
// with the shading normal; resolveLodSource with a zero LOD blend gives
// (rgb * coverage) / coverage, and zero without coverage.
__device__ __forceinline__ f3 feedback_irradiance(const Feedback &fb, f3 position, f3 normal, float &coverage) {
    coverage = 0.0f;
    const float s = fb.spacing;
    int32_t x = (int32_t)floorf(position.x / s), y = (int32_t)floorf(position.y / s), z = (int32_t)floorf(position.z / s);
    if (!finite3(position) || !cell_in_range(x, y, z)) return f3{0.0f, 0.0f, 0.0f};
    unsigned long long key = pack_cell(x, y, z);
    uint32_t slot = hash_key(x, y, z, 0, fb.capacity);
    for (uint32_t attempt = 0; attempt < fb.capacity; ++attempt) {
        unsigned long long k = __ldg(fb.keys + slot);
        if (k == key) {
            uint32_t id = __ldg(fb.ids + slot);
            if (id == kEmpty) break;
            float4 e = probe_irradiance(fb.tables + (size_t)id * 36, normal);
            if (!(e.w > 0.0f)) break;
            coverage = e.w;
            return f3{(e.x * e.w) / e.w, (e.y * e.w) / e.w, (e.z * e.w) / e.w};
        }
        if (k == kEmptyCell) break;
        slot = (slot + 1u) & (fb.capacity - 1u);
    }
    return f3{0.0f, 0.0f, 0.0f};
}

// The surface a multi-bounce secondary receiver takes from an interval-ray
// hit (the primary trace's hit record, shaders/split.slang:1199-1211).
struct SurfaceRecord {
    f3 position, normal;  // hit position, geometric normal facing the ray origin
    bool valid;
};

// Next-event slots of one hit: max(1, emissive_samples / 2) emissive samples,
// as many environment samples with a non-black environment, one per
// conventional light.
constexpr uint32_t kMaxNeeSamples = 16u;

enum NeeGroup : uint32_t { kNeeEmissive = 0u, kNeeEnvironment = 1u, kNeeConventional = 2u };

// One next-event sample of emissiveResponseTracked whose visibility query is
// still to be traced: the query ray and the sample's contribution if visible.
struct NeeQuery {
    f3 origin, direction;
    float limit;
    f3 contribution;
    uint32_t light;  // emitter record index (coherence sort key)
    NeeGroup group;  // emissive and environment samples are averaged per group, conventional lights summed
};

// emissiveResponseTracked, shaders/cascades.slang:57-134, up to (but not
// including) the visibility trace: every sample that survives the geometric
// tests becomes a query with its contribution emission * (response * cos / pdf).
// Samples are emitted in sample order; `count` is the estimator's divisor.
template <typename Emit>
__device__ void emissive_queries(const SceneView &S, const ShadeParams &P, f3 position, f3 normal, f3 gnormal,
                                 f3 view, float roughness, f3 diffuse, uint32_t &count, Emit &&emit) {
    uint32_t emissive = S.emissive_lights;
    count = P.emissive_samples / 2u;
    count = count < 1u ? 1u : count;
    if (emissive == 0u) return;
    float cell = P.probe_spacing * 0.05f;
    uint32_t seed = hash_key((int32_t)floorf(position.x / cell), (int32_t)floorf(position.y / cell),
                             (int32_t)floorf(position.z / cell), 0, 16777216u);
    float rot_x, rot_y;
    r2(seed, rot_x, rot_y);
    float s0 = P.probe_spacing * 1.0f;
    uint32_t selection_seed = hash_key((int32_t)floorf(position.x / s0), (int32_t)floorf(position.y / s0),
                                       (int32_t)floorf(position.z / s0), 0, 65536u);
    uint32_t sample_frame = P.frame ^ 0xE11E0001u;
    float ax, ay, bx, by;
    r2(sample_frame, ax, ay);
    r2(selection_seed, bx, by);
    float phase = fracf(ax + bx);
    const float bias = P.normal_bias;
    const LuxLight *lights = S.lights + S.conventional_lights;
    for (uint32_t sample = 0; sample < count; ++sample) {
        float rx, ry;
        r2(sample + sample_frame * count + 1u, rx, ry);
        float ux = fracf(rx + rot_x), uy = fracf(ry + rot_y);
        float selection = fracf(((float)sample + 0.5f) / (float)count + phase);
        uint32_t low = 0, high = emissive - 1u;
        while (low < high) {
            uint32_t middle = (low + high) / 2u;
            if (__ldg(&lights[middle].direction[3]) < selection)
                low = middle + 1u;
            else
                high = middle;
        }
        const LuxLight *L = lights + low;
        f3 lp{__ldg(&L->position[0]), __ldg(&L->position[1]), __ldg(&L->position[2])};
        float lpw = __ldg(&L->position[3]);
        f3 ldir{__ldg(&L->direction[0]), __ldg(&L->direction[1]), __ldg(&L->direction[2])};
        f3 e1{__ldg(&L->edge1[0]), __ldg(&L->edge1[1]), __ldg(&L->edge1[2])};
        float e1w = __ldg(&L->edge1[3]);
        f3 e2{__ldg(&L->edge2[0]), __ldg(&L->edge2[1]), __ldg(&L->edge2[2])};
        float area = __ldg(&L->color[3]);
        f3 rel = position - lp;
        if (e1w <= 0.0f || (lpw != -2.0f && dot(ldir, rel) <= 0.0f)) continue;
        float root = sqrtf(ux);
        float w1 = root * (1.0f - uy), w2 = root * uy;
        f3 target{(lp.x + e1.x * w1) + e2.x * w2, (lp.y + e1.y * w1) + e2.y * w2, (lp.z + e1.z * w1) + e2.z * w2};
        f3 to_light = target - position;
        float light_distance = length(to_light);
        if (light_distance <= bias * 0.25f) continue;
        f3 ld = to_light / light_distance;
        float cosine = fmaxf(0.0f, dot(normal, ld));
        float c_emit = dot(ldir, -ld);
        if (lpw == -2.0f) c_emit = fabsf(c_emit);
        float emitter_cosine = fmaxf(0.0f, c_emit);
        if (cosine <= 0.0f || emitter_cosine <= 0.0f || dot(gnormal, ld) <= 0.0f) continue;
        Surface es = surface_at(S, P, __ldg(&L->source[0]), __ldg(&L->source[1]), 1.0f - root, w1, w2);
        f3 emission{fmaxf(es.emission.x, 0.0f), fmaxf(es.emission.y, 0.0f), fmaxf(es.emission.z, 0.0f)};
        if (!(emission.x > 0.0f || emission.y > 0.0f || emission.z > 0.0f)) continue;
        float pdf = ((e1w * light_distance) * light_distance) / (area * emitter_cosine);
        float plane = fabsf(dot(ldir, rel));
        f3 origin = ray_offset(position, gnormal, fminf(bias, plane * 0.25f));
        f3 delta = target - origin;
        float distance = length(delta);
        if (distance <= bias * 0.25f) continue;
        NeeQuery q;
        q.origin = origin;
        q.direction = delta / distance;
        q.limit = distance - fminf(bias * 0.25f, distance * 0.001f);
        float factor = disney_multiplier(normal, ld, view, roughness) / kPi;
        float p = fmaxf(pdf, 1e-20f);
        q.contribution = f3{emission.x * (((diffuse.x * factor) * cosine) / p),
                            emission.y * (((diffuse.y * factor) * cosine) / p),
                            emission.z * (((diffuse.z * factor) * cosine) / p)};
        q.light = low;
        q.group = kNeeEmissive;
        emit(sample, q);
    }
}

// conventionalLightResponseTracked (shaders/cascades.slang:136-176) up to the
// visibility traces: one query per conventional light that faces the
// surface, from the biased hit point to the light (finite lights: range fade
// (1 - (d/range)^4)^2 / d^2, spot cone squared; directional lights: the
// direction in position.xyz at distance 1e20), contribution color x
// (attenuation x cos x response).  Light i takes slot first_slot + i.
// (d/range)^4 is (x^2)^2 here and in the oracle.
template <typename Emit>
__device__ void conventional_queries(const SceneView &S, const ShadeParams &P, f3 position, f3 normal, f3 gnormal,
                                     f3 view, float roughness, f3 diffuse, uint32_t first_slot, Emit &&emit) {
    const uint32_t n = S.conventional_lights;
    if (n == 0u) return;
    const float bias = P.normal_bias;
    const f3 offset = ray_offset(position, gnormal, bias);
    for (uint32_t i = 0; i < n; ++i) {
        const LuxLight *L = S.lights + i;
        f3 lp{__ldg(&L->position[0]), __ldg(&L->position[1]), __ldg(&L->position[2])};
        float range = __ldg(&L->position[3]);
        const bool finite = range > 0.0f;
        f3 to_light = lp;
        float distance = 1e20f, attenuation = 1.0f;
        if (finite) {
            to_light = lp - position;
            distance = length(to_light);
            if (distance >= range || distance < bias) continue;
            to_light = to_light / distance;
            float x = distance / range;
            float x2 = x * x;
            float fade = saturate(1.0f - x2 * x2);
            attenuation = (fade * fade) / fmaxf(distance * distance, 0.0001f);
            float spot = __ldg(&L->direction[3]);
            if (spot > 0.0f) {
                f3 ldir{__ldg(&L->direction[0]), __ldg(&L->direction[1]), __ldg(&L->direction[2])};
                float cone = saturate(dot(ldir, -to_light) * spot + __ldg(&L->color[3]));
                attenuation *= cone * cone;
            }
        }
        float cosine = fmaxf(0.0f, dot(normal, to_light));
        if (!(cosine > 0.0f && dot(gnormal, to_light) > 0.0f && attenuation > 0.0f)) continue;
        NeeQuery q;
        q.origin = offset;
        q.direction = to_light;
        q.limit = distance - bias;
        float factor = disney_multiplier(normal, to_light, view, roughness) / kPi;
        float scale = attenuation * cosine;
        q.contribution = f3{__ldg(&L->color[0]) * (scale * (diffuse.x * factor)),
                            __ldg(&L->color[1]) * (scale * (diffuse.y * factor)),
                            __ldg(&L->color[2]) * (scale * (diffuse.z * factor))};
        q.light = i;
        q.group = kNeeConventional;
        emit(first_slot + i, q);
    }
}

// environmentResponseTracked (shaders/environment.slang:154-230) for a
// constant environment, up to the visibility traces: `count` cosine
// proposals (no alias samples without an environment map, so pdf = cos / pi),
// direction cosineDirection(normal, transportRandom lanes 0 and 1) of the
// seed transportHash(seed ^ transportHash(sequence + 0x85ebca6b)),
// sequence = sample + (frame ^ 0xE17A0002) x count, seed = hashKey of the
// hit's cell of 0.05 probe spacings with w = 37; each a query from the biased
// hit point to distance 1e20 with contribution environment x (response x
// cos / pdf).  Sample i takes slot first_slot + i.
template <typename Emit>
__device__ void environment_queries(const ShadeParams &P, f3 position, f3 normal, f3 gnormal, f3 view,
                                    float roughness, f3 diffuse, uint32_t count, uint32_t first_slot, Emit &&emit) {
    if (!environment_on(P)) return;
    const f3 env = P.environment;
    float cell = P.probe_spacing * 0.05f;
    uint32_t seed = hash_key((int32_t)floorf(position.x / cell), (int32_t)floorf(position.y / cell),
                             (int32_t)floorf(position.z / cell), 37, 16777216u);
    uint32_t sample_frame = P.frame ^ 0xE17A0002u;
    const f3 offset = ray_offset(position, gnormal, P.normal_bias);
    for (uint32_t sample = 0; sample < count; ++sample) {
        uint32_t sequence = sample + sample_frame * count;
        uint32_t sample_seed = transport_hash(seed ^ transport_hash(sequence + 0x85ebca6bu));
        f3 d = cosine_direction_frame(normal, transport_random(sample_seed, 0u), transport_random(sample_seed, 1u));
        float cosine = fmaxf(0.0f, dot(normal, d));
        if (cosine <= 0.0f || dot(gnormal, d) <= 0.0f) continue;
        float pdf = cosine / kPi;
        if (!(pdf > 0.0f) || !isfinite(pdf)) continue;
        NeeQuery q;
        q.origin = offset;
        q.direction = d;
        q.limit = 1e20f;
        float factor = disney_multiplier(normal, d, view, roughness) / kPi;
        q.contribution = f3{env.x * (((diffuse.x * factor) * cosine) / pdf),
                            env.y * (((diffuse.y * factor) * cosine) / pdf),
                            env.z * (((diffuse.z * factor) * cosine) / pdf)};
        q.light = 63u;
        q.group = kNeeEnvironment;
        emit(first_slot + sample, q);
    }
}

// outgoingTransportRadianceTracked, shaders/cascades.slang:196-268, up to the
// visibility traces.  Writes the hit's own emission to `base`, the
// multi-bounce term (diffuse x secondary-cache irradiance) to `extra`, the
// surface a secondary receiver would take to `rec`, and emits the next-event
// queries; returns false when the query is unsupported (no deposit).
// `count` = 0 when no next-event estimate applies; `sky` is set when the
// hit takes environment samples (slots count .. 2 count - 1).
template <typename Emit>
__device__ bool outgoing_record(const SceneView &S, const ShadeParams &P, f3 origin, f3 direction, const Hit &hit,
                                f3 &base, f3 &extra, SurfaceRecord &rec, uint32_t &count, bool &sky, Emit &&emit) {
    base = f3{0.0f, 0.0f, 0.0f};
    extra = f3{0.0f, 0.0f, 0.0f};
    rec.valid = false;
    count = 0;
    sky = false;
    if ((hit.errors & kQueryUnsupported) != 0u) return false;
    if (hit.tri == kEmpty) {
        // outgoingEnvironmentEscape (shaders/environment.slang:145-152): the
        // secondary cache's escapes carry the environment with cached hit sky.
        if (P.skip_emission && P.cached_sky) base = P.environment;
        return true;
    }
    float b0 = (1.0f - hit.b1) - hit.b2;
    Surface sf = surface_at(S, P, hit.inst, hit.tri, b0, hit.b1, hit.b2);
    if (!P.skip_emission) base = sf.emission;
    if ((sf.flags & 16u) != 0u) return true;
    uint32_t ibase = instance_base(S, hit.inst);
    uint4 header = gword(S, 0);
    uint4 t = gword(S, header.x + hit.tri);
    uint32_t idx[3] = {t.x, t.y, t.z};
    f3 A = f3w(gword(S, header.y + idx[0] * header.z));
    f3 B = f3w(gword(S, header.y + idx[1] * header.z));
    f3 C = f3w(gword(S, header.y + idx[2] * header.z));
    f3 position{origin.x + direction.x * hit.t, origin.y + direction.y * hit.t, origin.z + direction.z * hit.t};
    f3 gn = unit_vector(transform_direction_t(S, ibase, cross(B - A, C - A)), f3{0.0f, 1.0f, 0.0f});
    float sign = (sf.flags & 4u) != 0u ? -1.0f : 1.0f;
    gn = gn * sign;
    // hitAttributes world normal, shaders/traversal.slang:258-282.
    float bary[3] = {b0, hit.b1, hit.b2};
    f3 world_normal{0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        uint32_t vb = header.y + idx[i] * header.z;
        f3 nrm = gn;
        if ((gword(S, vb).w & 1u) != 0u) nrm = unit_vector(transform_direction_t(S, ibase, f3w(gword(S, vb + 1))), gn);
        world_normal = f3{world_normal.x + nrm.x * bary[i], world_normal.y + nrm.y * bary[i],
                          world_normal.z + nrm.z * bary[i]};
    }
    // materialNormal without a normal texture, shaders/material.slang:171-177.
    f3 normal = unit_vector(world_normal, gn);
    bool back = dot(gn, direction) > 0.0f;
    if (back && (sf.flags & 8u) != 0u) normal = -normal;
    f3 flipped = dot(gn, direction) > 0.0f ? -gn : gn;
    f3 neg = -direction;
    if (dot(normal, neg) <= 0.0f || dot(normal, flipped) <= 0.0f) return true;
    float nl = length(neg);
    f3 view = neg / nl;
    float metallic = saturate(sf.metallic);
    float roughness = saturate(sf.roughness);
    if (!isfinite(roughness)) roughness = 1.0f;
    bool bf = finite3(sf.base_color);
    f3 diffuse{(bf ? saturate(sf.base_color.x) : 0.0f) * (1.0f - metallic),
               (bf ? saturate(sf.base_color.y) : 0.0f) * (1.0f - metallic),
               (bf ? saturate(sf.base_color.z) : 0.0f) * (1.0f - metallic)};
    rec.position = position;
    rec.normal = flipped;
    rec.valid = finite3(position) && finite3(flipped) && finite3(normal) && dot(flipped, flipped) > 0.01f;
    float coverage = 0.0f;
    if (P.feedback) {
        f3 e = feedback_irradiance(P.fb, position, normal, coverage);
        extra = f3{e.x * diffuse.x, e.y * diffuse.y, e.z * diffuse.z};
    }
    // skyFromCache (shaders/cascades.slang:242): a covered hit takes its sky
    // light from the secondary cache's probe instead of environment samples.
    sky = environment_on(P) && !(P.cached_sky && coverage > 0.0f);
    emissive_queries(S, P, position, normal, flipped, view, roughness, diffuse, count, emit);
    if (sky) environment_queries(P, position, normal, flipped, view, roughness, diffuse, count, count, emit);
    conventional_queries(S, P, position, normal, flipped, view, roughness, diffuse, sky ? 2u * count : count, emit);
    return true;
}

template <typename Emit>
__device__ bool outgoing_record(const SceneView &S, const ShadeParams &P, f3 origin, f3 direction, const Hit &hit,
                                f3 &base, uint32_t &count, Emit &&emit) {
    f3 extra;
    SurfaceRecord rec;
    bool sky;
    return outgoing_record(S, P, origin, direction, hit, base, extra, rec, count, sky, emit);
}

// clampOutgoingTransportRadiance, shaders/cascades.slang:179-188, after the
// next-event sums: radiance = base + sum / count + environment / count
// + conventional + extra.
__device__ __forceinline__ f3 finish_radiance(f3 base, f3 sum, uint32_t count, const f3 *environment = nullptr,
                                              const f3 *conventional = nullptr, const f3 *extra = nullptr) {
    f3 radiance = base;
    if (count) radiance = radiance + f3{sum.x / (float)count, sum.y / (float)count, sum.z / (float)count};
    if (count && environment)  // the environment samples, averaged over the same count
        radiance = radiance + f3{environment->x / (float)count, environment->y / (float)count,
                                 environment->z / (float)count};
    if (conventional) radiance = radiance + *conventional;  // conventional lights' visible contributions
    if (extra) radiance = radiance + *extra;  // secondaryFeedback's diffuse term, added last
    if (!finite3(radiance)) return f3{0.0f, 0.0f, 0.0f};
    return f3{fmaxf(radiance.x, 0.0f), fmaxf(radiance.y, 0.0f), fmaxf(radiance.z, 0.0f)};
}

}  // namespace lux
