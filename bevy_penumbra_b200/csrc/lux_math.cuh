// lux_math.cuh - device math of the Split transport path.
//
// Evaluation contract: every expression is IEEE binary32, evaluated in the
// order written, without fused multiply-add contraction (the library is
// compiled with --fmad=false) and with IEEE division and square root.  The
// reference computes these on its GPU; the formulas and the order of
// operations follow the Slang sources cited at each function.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define LUX_HD __host__ __device__ __forceinline__
#else
#define LUX_HD inline
#endif

namespace lux {

constexpr uint32_t kEmpty = 0xffffffffu;
constexpr uint32_t kQueryUnsupported = 4u;  // shaders/traversal.slang:16
constexpr float kPi = 3.14159265358979323846f;

struct f3 {
    float x, y, z;
};
LUX_HD f3 make3(float x, float y, float z) { return f3{x, y, z}; }
LUX_HD f3 operator+(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
LUX_HD f3 operator-(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
LUX_HD f3 operator-(f3 a) { return f3{-a.x, -a.y, -a.z}; }
LUX_HD f3 operator*(f3 a, float s) { return f3{a.x * s, a.y * s, a.z * s}; }
LUX_HD f3 operator*(f3 a, f3 b) { return f3{a.x * b.x, a.y * b.y, a.z * b.z}; }
LUX_HD f3 operator/(f3 a, float s) { return f3{a.x / s, a.y / s, a.z / s}; }
LUX_HD float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
LUX_HD f3 cross(f3 a, f3 b) {
    return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
LUX_HD float comp(f3 v, uint32_t i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
LUX_HD float saturate(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }
LUX_HD float fracf(float x) { return x - floorf(x); }
LUX_HD bool finite3(f3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }
LUX_HD float length(f3 v) { return sqrtf(dot(v, v)); }

LUX_HD float as_float(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    __builtin_memcpy(&f, &u, 4);
    return f;
#endif
}
LUX_HD uint32_t as_uint(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u;
    __builtin_memcpy(&u, &f, 4);
    return u;
#endif
}

// cos and sin of 2*pi*turns, evaluated identically on host and device:
// exact reduction to the nearest quarter turn, then the Taylor series of
// sin(2 pi r) (degree 11) and cos(2 pi r) (degree 10) for |r| <= 1/8
// (truncation below 3e-8).  Replaces the GPU cos/sin of decodeDirection
// (shaders/common.slang:376-382).
LUX_HD void sincos_turns(float turns, float &c, float &s) {
    float k = floorf(turns * 4.0f + 0.5f);
    float r = turns - k * 0.25f;
    int q = ((int)k) & 3;
    float r2 = r * r;
    float sp = 42.058693f - r2 * 15.094643f;
    sp = 76.70586f - r2 * sp;
    sp = 81.60525f - r2 * sp;
    sp = 41.3417f - r2 * sp;
    sp = 6.2831855f - r2 * sp;
    float sn = r * sp;
    float cp = 60.24464f - r2 * 26.426256f;
    cp = 85.45682f - r2 * cp;
    cp = 64.93939f - r2 * cp;
    cp = 19.739208f - r2 * cp;
    float cs = 1.0f - r2 * cp;
    if (q == 0) {
        c = cs;
        s = sn;
    } else if (q == 1) {
        c = -sn;
        s = cs;
    } else if (q == 2) {
        c = -cs;
        s = -sn;
    } else {
        c = sn;
        s = -cs;
    }
}

// decodeDirection, shaders/common.slang:376-382.
LUX_HD f3 decode_direction(float u, float v) {
    float y = v * 2.0f - 1.0f;
    float r = sqrtf(fmaxf(0.0f, 1.0f - y * y));
    float c, s;
    sincos_turns(u, c, s);
    return f3{r * c, y, r * s};
}

// binDirection, shaders/common.slang:395-400 (columns x rows grid).
LUX_HD f3 bin_direction(uint32_t index, uint32_t columns, uint32_t rows) {
    float u = ((float)(index % columns) + 0.5f) / (float)columns;
    float v = ((float)(index / columns) + 0.5f) / (float)rows;
    return decode_direction(u, v);
}

// directionIndex, shaders/common.slang:388-394, on the (u, v) of a decoded
// direction (encodeDirection inverts decodeDirection).
LUX_HD uint32_t direction_index_uv(float u, float v, uint32_t columns, uint32_t rows) {
    uint32_t x = (uint32_t)(u * (float)columns);
    uint32_t y = (uint32_t)(v * (float)rows);
    x = x > columns - 1u ? columns - 1u : x;
    y = y > rows - 1u ? rows - 1u : y;
    return x + y * columns;
}

// r2, shaders/common.slang:401-406.
LUX_HD void r2(uint32_t index, float &x, float &y) {
    uint32_t px = index * 3242174889u;
    uint32_t py = index * 2447445414u;
    x = (float)(px >> 8) / 16777216.0f;
    y = (float)(py >> 8) / 16777216.0f;
}

// transportHash, shaders/common.slang:281-289.
LUX_HD uint32_t transport_hash(uint32_t value) {
    value ^= value >> 16;
    value *= 0x7feb352du;
    value ^= value >> 15;
    value *= 0x846ca68bu;
    value ^= value >> 16;
    return value;
}

// Sample (u1, u2) in [0, 1)^2 of hemisphere sample `s` at reference point
// `p` (the FP64 reference irradiance; no reference counterpart): two chained
// transportHash values, 24 bits each.
LUX_HD void reference_sample(uint32_t p, uint32_t s, uint32_t seed, float &u1, float &u2) {
    uint32_t h1 = transport_hash(p ^ transport_hash(s ^ transport_hash(seed + 0x2545f491u)));
    uint32_t h2 = transport_hash(h1 ^ 0x68bc21ebu);
    u1 = (float)(h1 >> 8) / 16777216.0f;
    u2 = (float)(h2 >> 8) / 16777216.0f;
}

// Uniform number in [0, 1) of the path-traced reference: dimension `dim` of
// sample `s` at point `p` (an independent hash stream per point and sample).
LUX_HD float path_random(uint32_t p, uint32_t s, uint32_t seed, uint32_t dim) {
    uint32_t h = transport_hash(p ^ transport_hash(s ^ transport_hash(seed + 0x7f4a7c15u + dim * 0x9e3779b9u)));
    return (float)(h >> 8) / 16777216.0f;
}

// hashKey, shaders/common.slang:423-429.
LUX_HD uint32_t hash_key(int32_t kx, int32_t ky, int32_t kz, int32_t kw, uint32_t buckets) {
    uint32_t h = (uint32_t)kx * 0x8da6b343u ^ (uint32_t)ky * 0xd8163841u ^ (uint32_t)kz * 0xcb1ab31fu ^
                 (uint32_t)kw * 0x165667b1u;
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    return h & (buckets - 1u);
}

// rayOffset, shaders/common.slang:343-359, one axis.
LUX_HD float ray_offset_axis(float position, float normal, float bias) {
    float origin = position + normal * bias;
    int32_t step = (int32_t)(normal * 256.0f);
    int32_t bits = (int32_t)as_uint(origin);
    float integer_offset = as_float((uint32_t)(bits + (origin < 0.0f ? -step : step)));
    float shifted = fabsf(origin) < 0.03125f ? origin + normal / 65536.0f : integer_offset;
    return isfinite(shifted) ? shifted : position;
}
LUX_HD f3 ray_offset(f3 p, f3 n, float bias) {
    return f3{ray_offset_axis(p.x, n.x, bias), ray_offset_axis(p.y, n.y, bias), ray_offset_axis(p.z, n.z, bias)};
}

// encodeNormal, shaders/common.slang:360-366.
LUX_HD void encode_normal(f3 n, float &ox, float &oy) {
    float d = (fabsf(n.x) + fabsf(n.y)) + fabsf(n.z);
    n = f3{n.x / d, n.y / d, n.z / d};
    float px = n.x, py = n.y;
    if (n.z < 0.0f) {
        float qx = (1.0f - fabsf(n.y)) * (px >= 0.0f ? 1.0f : -1.0f);
        float qy = (1.0f - fabsf(n.x)) * (py >= 0.0f ? 1.0f : -1.0f);
        px = qx;
        py = qy;
    }
    ox = px * 0.5f + 0.5f;
    oy = py * 0.5f + 0.5f;
}

// decodeNormal, shaders/common.slang:367-374 (normalize as v / length(v)).
LUX_HD f3 decode_normal(float ux, float uy) {
    float px = ux * 2.0f - 1.0f, py = uy * 2.0f - 1.0f;
    f3 n{px, py, (1.0f - fabsf(px)) - fabsf(py)};
    float t = saturate(-n.z);
    n.x = n.x + (n.x >= 0.0f ? -t : t);
    n.y = n.y + (n.y >= 0.0f ? -t : t);
    float l = length(n);
    return f3{n.x / l, n.y / l, n.z / l};
}

// wrapIrradianceTexel + irradianceTexelIndex, shaders/world_resolve.slang:1-11.
LUX_HD uint32_t texel_index(int32_t x, int32_t y) {
    if (x < 0) {
        int32_t nx = -x - 1, ny = 5 - y;
        x = nx;
        y = ny;
    } else if (x >= 6) {
        int32_t nx = 11 - x, ny = 5 - y;
        x = nx;
        y = ny;
    }
    if (y < 0) {
        int32_t nx = 5 - x, ny = -y - 1;
        x = nx;
        y = ny;
    } else if (y >= 6) {
        int32_t nx = 5 - x, ny = 11 - y;
        x = nx;
        y = ny;
    }
    return (uint32_t)(y * 6 + x);
}

// Cell keys of the world grid: 19 bits per axis biased by 2^18, and the
// probe LOD in bits 57-61 (cacheKey's lod field, shaders/common.slang:418-422).
LUX_HD uint64_t pack_cell(int32_t x, int32_t y, int32_t z, uint32_t lod = 0u) {
    return ((uint64_t)((uint32_t)(x + (1 << 18)) & 0x7ffffu)) |
           ((uint64_t)((uint32_t)(y + (1 << 18)) & 0x7ffffu) << 19) |
           ((uint64_t)((uint32_t)(z + (1 << 18)) & 0x7ffffu) << 38) | ((uint64_t)(lod & 31u) << 57);
}
LUX_HD void unpack_cell(uint64_t key, int32_t &x, int32_t &y, int32_t &z, uint32_t &lod) {
    x = (int32_t)(key & 0x7ffffull) - (1 << 18);
    y = (int32_t)((key >> 19) & 0x7ffffull) - (1 << 18);
    z = (int32_t)((key >> 38) & 0x7ffffull) - (1 << 18);
    lod = (uint32_t)(key >> 57) & 31u;
}
LUX_HD bool cell_in_range(int32_t x, int32_t y, int32_t z) {
    const int32_t lim = 1 << 18;
    return x >= -lim && x < lim && y >= -lim && y < lim && z >= -lim && z < lim;
}

// Distance LODs (MAX_PROBE_LOD, shaders/common.slang:16).
constexpr uint32_t kMaxLod = 24u;
// 2^lod exactly (lod <= kMaxLod): spacing and interval ends scale by it.
LUX_HD float lod_scale(uint32_t lod) { return as_float((127u + lod) << 23); }
// The LOD field of a cell key's w (level << 12 | lod << 18).
LUX_HD uint32_t key_lod(int32_t w) { return ((uint32_t)w >> 18) & 31u; }

// splitLodBlendForParameters (shaders/common.slang:431-461) with the
// camera terms precomputed per frame: perspective cameras scale by the
// Chebyshev distance from the camera over `base` (max(focal pixels x
// spacing / target pixels, spacing)); orthographic cameras use the fixed
// `ortho_scale` (target pixels / projected spacing).  floor(log2(x)) for
// x >= 1 is the float's exponent (exact), and the next boundary 2^(low+1) is
// an exact power of two.
LUX_HD void lod_blend(bool perspective, float cx, float cy, float cz, float base, float ortho_scale, f3 p,
                      uint32_t &low, uint32_t &high, float &blend) {
    float scale;
    if (perspective) {
        float ox = fabsf(p.x - cx), oy = fabsf(p.y - cy), oz = fabsf(p.z - cz);
        scale = fmaxf(ox, fmaxf(oy, oz)) / base;
    } else {
        scale = ortho_scale;
    }
    float s1 = fmaxf(scale, 1.0f);
    uint32_t e = s1 < INFINITY ? (as_uint(s1) >> 23) - 127u : kMaxLod;
    low = e < kMaxLod ? e : kMaxLod;
    high = low;
    blend = 0.0f;
    if (low < kMaxLod) {
        float next = lod_scale(low + 1u);
        float overlap = 0.9f * next;
        if (scale >= overlap && scale < next) {
            high = low + 1u;
            blend = saturate((scale - overlap) / (next - overlap));
        }
    }
}

// The seeded variant of a receiver in an LOD overlap: temporal
// low-discrepancy selection of the high LOD with probability `blend`
// (seed, shaders/split.slang:747-752).
LUX_HD bool lod_selects_high(uint32_t sample, uint32_t frame, float blend) {
    uint32_t bits = transport_hash(sample ^ (frame * 0x9e3779b9u));
    float phase = (float)(bits >> 8) * (1.0f / 16777216.0f);
    return phase < blend;
}
constexpr uint64_t kEmptyCell = 0xffffffffffffffffull;

// transportRandom (shaders/common.slang:292-295): a decorrelated uniform in
// (0, 1) from a seed and a lane.
LUX_HD float transport_random(uint32_t seed, uint32_t lane) {
    uint32_t bits = transport_hash(seed + 0x9e3779b9u * (lane + 1u));
    return ((float)(bits >> 8) + 0.5f) * (1.0f / 16777216.0f);
}

// cosineDirection (shaders/common.slang:407-412): tangent frame from the
// normal and the y axis (the x axis near the poles), radius sqrt(u1) at u2
// turns, height sqrt(1 - u1); cos/sin of the turn as sincos_turns.
LUX_HD f3 cosine_direction_frame(f3 n, float u1, float u2) {
    f3 axis = fabsf(n.y) < 0.99f ? f3{0.0f, 1.0f, 0.0f} : f3{1.0f, 0.0f, 0.0f};
    f3 t = cross(axis, n);
    float tl = sqrtf(dot(t, t));
    t = f3{t.x / tl, t.y / tl, t.z / tl};
    f3 b = cross(n, t);
    float c, s;
    sincos_turns(u2, c, s);
    float r = sqrtf(u1), h = sqrtf(1.0f - u1);
    float rc = r * c, rs = r * s;
    return f3{(t.x * rc + b.x * rs) + n.x * h, (t.y * rc + b.y * rs) + n.y * h, (t.z * rc + b.z * rs) + n.z * h};
}

// Cosine-weighted direction about the unit normal n: radius sqrt(u1) at
// u2 turns in the tangent plane, height sqrt(1 - u1), in the orthonormal
// frame of Duff et al., "Building an Orthonormal Basis, Revisited" (2017).
LUX_HD f3 cosine_direction(f3 n, float u1, float u2) {
    float sign = n.z >= 0.0f ? 1.0f : -1.0f;
    float a = -1.0f / (sign + n.z);
    float b = n.x * n.y * a;
    f3 t{1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x};
    f3 bt{b, sign + n.y * n.y * a, -n.y};
    float c, s;
    sincos_turns(u2, c, s);
    float r = sqrtf(u1);
    float z = sqrtf(fmaxf(1.0f - u1, 0.0f));
    float x = r * c, y = r * s;
    return f3{(t.x * x + bt.x * y) + n.x * z, (t.y * x + bt.y * y) + n.y * z, (t.z * x + bt.z * y) + n.z * z};
}

}  // namespace lux
