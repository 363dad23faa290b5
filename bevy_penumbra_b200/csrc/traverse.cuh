// traverse.cuh - closest-hit and any-hit traversal of the two-level BVH4.
//
// Restates traceRayTracked / traceInstance / traceTriangle /
// intersectTriangle (shaders/traversal.slang:349-811) and traceOccluded /
// occludedInstance / occludedTriangle (shaders/traversal.slang:826-1046) on
// a 4-wide BVH whose child boxes are the reference's binary node boxes.
// Hit distances, triangles and instances are produced by the same watertight
// triangle test as the reference; equal distances resolve to the smaller
// (instance, triangle), which makes the answer independent of tree shape.
#pragma once
#include "lux_internal.h"
#include "lux_math.cuh"

namespace lux {

constexpr uint32_t kMaxSteps = 4096u;  // MAX_TRAVERSAL_STEPS, shaders/traversal.slang:8
constexpr int kStack = 64;  // default traversal stack depth (entries)

struct Hit {
    float t;
    uint32_t tri, inst, errors;
    float b1, b2;
};

struct TraceCounters {
    uint32_t nodes, triangles, instances;
};

// boxRayInterval, shaders/traversal.slang:349-369, for one box.
__device__ __forceinline__ bool box_interval(f3 o, f3 d, float lx, float ly, float lz, float hx, float hy,
                                             float hz, float limit, float &entry, float &exit) {
    float near_t = 0.0f, far_t = limit;
    float lo[3] = {lx, ly, lz}, hi[3] = {hx, hy, hz};
    float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (dd[a] == 0.0f) {
            if (oo[a] < lo[a] || oo[a] > hi[a]) {
                entry = 0.0f;
                exit = 0.0f;
                return false;
            }
        } else {
            float ta = (lo[a] - oo[a]) / dd[a];
            float tb = (hi[a] - oo[a]) / dd[a];
            float ax = fmaxf(ta, tb);
            near_t = fmaxf(near_t, fminf(ta, tb));
            far_t = fminf(far_t, ax + fabsf(ax) * 3.5762791e-7f);
        }
    }
    entry = near_t;
    exit = far_t;
    return near_t <= far_t;
}

// Per-ray slab constants for the BVH4 child tests.  The reference divides
// by the direction for every slab (shaders/traversal.slang:360-361); the
// child tests here multiply by the correctly rounded reciprocal and widen the
// interval so the test stays conservative: t = (plane - o) * inv carries
// under 2 ulp of relative error, and the interval grows by 7.2e-7 (about 6
// ulp) relative on both ends.  Culling only decides which triangles are
// tested; hit distances come from the exact triangle test.
//
// The sign of each reciprocal picks the near and far plane of every axis
// once per ray (s = 1 selects the high plane as near), so a child costs two
// subtracts, two multiplies and no min/max per axis.  A zero direction
// component gives an infinite reciprocal: planes on either side of the
// origin give -inf/+inf (no constraint), a box wholly on one side gives an
// infinite near or -inf far (miss), and a plane through the origin gives
// NaN, which fmaxf/fminf ignore -- the reference's inside test for a zero
// component.
#ifndef LUX_NODE_EMPTY_CHECK
#define LUX_NODE_EMPTY_CHECK 0
#endif

struct SlabRay {
    float ox, oy, oz;
    float ix, iy, iz;     // 1 / d, correctly rounded (+-inf on zero axes)
    uint32_t sx, sy, sz;  // sign bits of ix, iy, iz
};

__device__ __forceinline__ SlabRay slab_ray(f3 o, f3 d) {
    SlabRay r;
    r.ox = o.x;
    r.oy = o.y;
    r.oz = o.z;
    r.ix = __frcp_rn(d.x);
    r.iy = __frcp_rn(d.y);
    r.iz = __frcp_rn(d.z);
    r.sx = as_uint(r.ix) >> 31;
    r.sy = as_uint(r.iy) >> 31;
    r.sz = as_uint(r.iz) >> 31;
    return r;
}

// Child tests of one BVH4 node.  Returns the hit mask and conservative entry
// distances; children that end before tmin or start after `limit` are culled.
__device__ __forceinline__ uint32_t node_test(const Bvh4Node *__restrict__ nodes, uint32_t index, const SlabRay &r,
                                              float limit, float tmin, float entry[4], uint32_t child[4]) {
    // Node rows: lo_x, hi_x, lo_y, hi_y, lo_z, hi_z, child.
    const float4 *p = reinterpret_cast<const float4 *>(nodes + index);
    float4 nx = __ldg(p + r.sx), fx = __ldg(p + (1u - r.sx));
    float4 ny = __ldg(p + 2u + r.sy), fy = __ldg(p + (3u - r.sy));
    float4 nz = __ldg(p + 4u + r.sz), fz = __ldg(p + (5u - r.sz));
    uint4 ch = __ldg(reinterpret_cast<const uint4 *>(p + 6));
    child[0] = ch.x;
    child[1] = ch.y;
    child[2] = ch.z;
    child[3] = ch.w;
    float NX[4] = {nx.x, nx.y, nx.z, nx.w}, FX[4] = {fx.x, fx.y, fx.z, fx.w};
    float NY[4] = {ny.x, ny.y, ny.z, ny.w}, FY[4] = {fy.x, fy.y, fy.z, fy.w};
    float NZ[4] = {nz.x, nz.y, nz.z, nz.w}, FZ[4] = {fz.x, fz.y, fz.z, fz.w};
    uint32_t mask = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float ax = (NX[i] - r.ox) * r.ix, bx = (FX[i] - r.ox) * r.ix;
        float ay = (NY[i] - r.oy) * r.iy, by = (FY[i] - r.oy) * r.iy;
        float az = (NZ[i] - r.oz) * r.iz, bz = (FZ[i] - r.oz) * r.iz;
        float near_t = fmaxf(fmaxf(ax, ay), fmaxf(az, 0.0f));
        float far_t = fminf(fminf(bx, by), bz);
        near_t = near_t - fabsf(near_t) * 7.2e-7f;
        far_t = far_t + fabsf(far_t) * 7.2e-7f;
#if LUX_NODE_EMPTY_CHECK
        bool h = child[i] != kEmpty && near_t <= far_t && near_t <= limit && far_t >= tmin;
#else
        // An empty slot's box is inverted infinities: its near and far come
        // out NaN after the padding, and every comparison with NaN fails.
        bool h = near_t <= far_t && near_t <= limit && far_t >= tmin;
#endif
        entry[i] = h ? near_t : 0.0f;
        mask |= h ? (1u << i) : 0u;
    }
    return mask;
}

struct TriRay {
    uint32_t kx, ky, kz;
    float sx, sy;
    bool valid;
};

// triangleRay, shaders/traversal.slang:399-413.
__device__ __forceinline__ TriRay triangle_ray(f3 d) {
    TriRay r{0, 0, 0, 0.0f, 0.0f, false};
    float mx = fabsf(d.x), my = fabsf(d.y), mz = fabsf(d.z);
    r.kz = mx > my ? (mx > mz ? 0u : 2u) : (my > mz ? 1u : 2u);
    float dz = comp(d, r.kz);
    r.valid = dz != 0.0f;
    if (!r.valid) return r;
    r.kx = (r.kz + 1u) % 3u;
    r.ky = (r.kx + 1u) % 3u;
    if (dz < 0.0f) {
        uint32_t t = r.kx;
        r.kx = r.ky;
        r.ky = t;
    }
    r.sx = comp(d, r.kx) / dz;
    r.sy = comp(d, r.ky) / dz;
    return r;
}

// orientedEdge, shaders/traversal.slang:379-392.
__device__ __forceinline__ float oriented_edge(float ax, float ay, float bx, float by) {
    bool reverse = ax > bx || (ax == bx && ay > by);
    float fx = reverse ? bx : ax, fy = reverse ? by : ay;
    float sx = reverse ? ax : bx, sy = reverse ? ay : by;
    float pa = fx * sy;
    float pb = fy * sx;
    float edge = pa - pb;
    float error = (fabsf(pa) + fabsf(pb)) * 2.3841858e-7f;
    if (fabsf(edge) <= error) edge = 0.0f;
    return reverse ? -edge : edge;
}

// intersectTriangle, shaders/traversal.slang:415-443.  Returns distance or -1.
__device__ __forceinline__ float intersect_triangle(f3 o, f3 d, const TriRay &ray, f3 A, f3 B, f3 C, float &w1,
                                                    float &w2) {
    if (!ray.valid) return -1.0f;
    f3 a = A - o, b = B - o, c = C - o;
    float akz = comp(a, ray.kz), bkz = comp(b, ray.kz), ckz = comp(c, ray.kz);
    float pax = comp(a, ray.kx) - ray.sx * akz, pay = comp(a, ray.ky) - ray.sy * akz;
    float pbx = comp(b, ray.kx) - ray.sx * bkz, pby = comp(b, ray.ky) - ray.sy * bkz;
    float pcx = comp(c, ray.kx) - ray.sx * ckz, pcy = comp(c, ray.ky) - ray.sy * ckz;
    float largest = fmaxf(fmaxf(fmaxf(fabsf(pax), fabsf(pay)), fmaxf(fabsf(pbx), fabsf(pby))),
                          fmaxf(fabsf(pcx), fabsf(pcy)));
    if (largest == 0.0f || !isfinite(largest)) return -1.0f;
    uint32_t exponent = (as_uint(largest) >> 23) & 255u;
    exponent = exponent < 1u ? 1u : (exponent > 253u ? 253u : exponent);
    float scale = as_float((254u - exponent) << 23);
    pax *= scale;
    pay *= scale;
    pbx *= scale;
    pby *= scale;
    pcx *= scale;
    pcy *= scale;
    float e0 = oriented_edge(pbx, pby, pcx, pcy);
    float e1 = oriented_edge(pcx, pcy, pax, pay);
    float e2 = oriented_edge(pax, pay, pbx, pby);
    bool any_neg = e0 < 0.0f || e1 < 0.0f || e2 < 0.0f;
    bool any_pos = e0 > 0.0f || e1 > 0.0f || e2 > 0.0f;
    if (any_neg && any_pos) return -1.0f;
    float det = (e0 + e1) + e2;
    if (det == 0.0f || !isfinite(det)) return -1.0f;
    float wx = e0 / det, wy = e1 / det, wz = e2 / det;
    float dist = ((wx * akz + wy * bkz) + wz * ckz) / comp(d, ray.kz);
    if (!isfinite(dist)) return -1.0f;
    w1 = wy;
    w2 = wz;
    return dist;
}

__device__ __forceinline__ bool hit_better(float t, uint32_t inst, uint32_t tri, const Hit &h) {
    if (t < h.t) return true;
    if (t > h.t || h.tri == kEmpty) return false;
    if (inst != h.inst) return inst < h.inst;
    return tri < h.tri;
}

// Face culling of traceTriangle / occludedTriangle (shaders/traversal.slang:449-453).
__device__ __forceinline__ bool cull_reject(uint32_t flags, f3 A, f3 B, f3 C, f3 d) {
    if ((flags & 3u) == 0u) return false;
    float facing = dot(cross(B - A, C - A), d) * ((flags & 4u) != 0u ? -1.0f : 1.0f);
    return ((flags & 1u) != 0u && facing >= 0.0f) || ((flags & 2u) != 0u && facing <= 0.0f);
}

__device__ __forceinline__ void load_triangle(const float4 *__restrict__ tris, uint32_t t, f3 &A, f3 &B, f3 &C) {
    float4 a = __ldg(tris + 3 * (size_t)t), b = __ldg(tris + 3 * (size_t)t + 1), c = __ldg(tris + 3 * (size_t)t + 2);
    A = f3{a.x, a.y, a.z};
    B = f3{b.x, b.y, b.z};
    C = f3{c.x, c.y, c.z};
}

// Local ray, shaders/traversal.slang:481-488.
__device__ __forceinline__ void local_ray(const DeviceInstance &I, f3 o, f3 d, f3 &lo, f3 &ld) {
    float r[3][4];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int c = 0; c < 4; ++c) r[k][c] = I.row[k][c];
    lo = f3{((r[0][0] * o.x + r[0][1] * o.y) + r[0][2] * o.z) + r[0][3] * 1.0f,
            ((r[1][0] * o.x + r[1][1] * o.y) + r[1][2] * o.z) + r[1][3] * 1.0f,
            ((r[2][0] * o.x + r[2][1] * o.y) + r[2][2] * o.z) + r[2][3] * 1.0f};
    ld = f3{((r[0][0] * d.x + r[0][1] * d.y) + r[0][2] * d.z) + r[0][3] * 0.0f,
            ((r[1][0] * d.x + r[1][1] * d.y) + r[1][2] * d.z) + r[1][3] * 0.0f,
            ((r[2][0] * d.x + r[2][1] * d.y) + r[2][2] * d.z) + r[2][3] * 0.0f};
}

__device__ __forceinline__ DeviceInstance load_instance(const DeviceInstance *__restrict__ inst, uint32_t i) {
    const float4 *p = reinterpret_cast<const float4 *>(inst + i);
    float4 r0 = __ldg(p), r1 = __ldg(p + 1), r2 = __ldg(p + 2);
    uint4 w = __ldg(reinterpret_cast<const uint4 *>(p + 3));
    DeviceInstance I;
    I.row[0][0] = r0.x; I.row[0][1] = r0.y; I.row[0][2] = r0.z; I.row[0][3] = r0.w;
    I.row[1][0] = r1.x; I.row[1][1] = r1.y; I.row[1][2] = r1.z; I.row[1][3] = r1.w;
    I.row[2][0] = r2.x; I.row[2][1] = r2.y; I.row[2][2] = r2.z; I.row[2][3] = r2.w;
    I.root = w.x;
    I.first = w.y;
    I.count = w.z;
    I.flags = w.w;
    return I;
}

// Child ordering keys: the entry distance's bits (entries are >= 0, so the
// bits order like the values) with the low two bits replaced by the child
// slot; missed children get ~0 and sort last.  Truncating two mantissa bits
// only lowers a stored entry, which keeps the closest-hit pop test
// (skip when entry > best distance) conservative.
__device__ __forceinline__ uint32_t child_key(uint32_t mask, const float entry[4], int i) {
    return (mask & (1u << i)) ? ((as_uint(entry[i]) & ~3u) | (uint32_t)i) : 0xffffffffu;
}

__device__ __forceinline__ void key_swap(uint32_t &a, uint32_t &b) {
    uint32_t lo = min(a, b), hi = max(a, b);
    a = lo;
    b = hi;
}

__device__ __forceinline__ uint32_t key_child(uint32_t key, const uint32_t child[4]) {
    uint32_t s = key & 3u;
    return s == 0u ? child[0] : (s == 1u ? child[1] : (s == 2u ? child[2] : child[3]));
}

__device__ __forceinline__ float key_entry(uint32_t key) { return as_float(key & ~3u); }

// traceRayTracked + traceInstance (kAnyHit = false) and traceOccluded +
// occludedInstance (kAnyHit = true) as one resumable walk over one stack.  A
// TLAS leaf enters its first instance (the rest of the leaf is pushed back);
// the BLAS walk runs on the same stack above `blas_base` in the instance's
// local space and returns to world space when the stack drops back to it.
// Each step traverses inner nodes until a leaf is reached, then processes
// that leaf (the while-while order), so the lanes of a warp stay in step and
// a lane whose ray finished can take a new ray between steps.
//
// Error bits follow the reference: 4 when a walk exceeds MAX_TRAVERSAL_STEPS
// (per TLAS walk and per instance walk), 2 / 1 when the stack is exhausted in
// the TLAS / a BLAS, after which the walk continues over every instance / every
// triangle of the instance in order (shaders/traversal.slang:498-517, :729-745).
// One warp's scratch for the cooperative leaf pass (shared memory).  Only
// the owning lane writes its own slots.
struct LeafScratch {
    float ox[32], oy[32], oz[32], dx[32], dy[32], dz[32], sx[32], sy[32], lower[32], limit[32];
    uint32_t axes[32], flags[32], first[32], pre[32];
    unsigned long long best[32];
};

template <bool kAnyHit, int kDepth = kStack>
struct Walker {
    Hit hit;
    f3 o, d, lo, ld;
    float tmin, lower;
    SlabRay r;       // slab constants of the current space's ray
    TriRay tri_ray;  // world ray's constants in the TLAS; the local ray's inside an instance
    bool rotated;    // the current instance changed the direction (r, tri_ray are local)
    uint32_t inst, inst_flags, inst_first, inst_count;
    int blas_base;        // stack depth at instance entry; -1 = TLAS space
    uint32_t tlas_next;   // TLAS fallback: next instance to scan in order
    uint32_t blas_next;   // BLAS fallback: next triangle to scan in order
    uint32_t tlas_steps, blas_steps;
    int sp;  // depth of the caller's stack: kDepth entries of (payload, entry distance bits)
    uint32_t cur;
    float cur_t;
    bool have;

    // Returns false when the query is already complete (no instances, or the
    // ray misses the TLAS root box: traceRayTracked's early exits).
    __device__ __forceinline__ bool start(const SceneView &S, f3 origin, f3 direction, float t_min, float limit) {
        hit.t = limit;
        hit.tri = kEmpty;
        hit.inst = kEmpty;
        hit.errors = 0;
        hit.b1 = 0.0f;
        hit.b2 = 0.0f;
        if (S.instance_count == 0) return false;
        // The TLAS root box is read from the live scene words (node 0), so a
        // device-side refit takes effect without a host round trip.
        float re, rx;
        uint4 ra = __ldg(S.scene_words + 1), rb = __ldg(S.scene_words + 2);
        if (!box_interval(origin, direction, as_float(ra.x), as_float(ra.y), as_float(ra.z), as_float(rb.x),
                          as_float(rb.y), as_float(rb.z), limit, re, rx))
            return false;
        o = origin;
        d = direction;
        tmin = t_min;
        lower = fmaxf(t_min, 0.000025f);
        r = slab_ray(o, d);
        tri_ray = triangle_ray(d);
        rotated = false;
        lo = o;
        ld = d;
        inst = kEmpty;
        inst_flags = inst_first = inst_count = 0;
        blas_base = -1;
        tlas_next = blas_next = kEmpty;
        tlas_steps = blas_steps = 0;
        sp = 0;
        cur = S.tlas_root;
        cur_t = 0.0f;
        have = true;
        return true;
    }

    // One step: inner nodes down to a leaf, that leaf, then the next pending
    // entry.  Returns true when the query is complete.
    // The stack lives outside the walker so the walker's fields stay in
    // registers; only the stack itself is addressed dynamically.
    // One inner node of the descent: its child tests, the farther hit
    // children pushed, the nearest taken.  Clears `have` at a dead end, an
    // instance's step budget or a stack overflow (the ordered-scan
    // fallback); returns true when the whole query is abandoned (the TLAS
    // step budget).
    __device__ __forceinline__ bool node_step(const SceneView &S, uint2 *stack, TraceCounters &cn) {
        bool in_tlas = blas_base < 0;
        uint32_t steps = (in_tlas ? tlas_steps : blas_steps) + 1u;
        if (in_tlas)
            tlas_steps = steps;
        else
            blas_steps = steps;
        if (steps > kMaxSteps) {
            hit.errors |= kQueryUnsupported;
            if (in_tlas) return true;  // abandon the whole query
            sp = blas_base;            // abandon this instance
            have = false;
            return false;
        }
        float entry[4];
        uint32_t child[4];
        cn.nodes++;
        uint32_t mask = node_test(S.nodes, cur, r, hit.t, tmin, entry, child);
        if (mask == 0u) {
            have = false;
            return false;
        }
        if (kAnyHit) {
            // Visibility needs a blocker, not the nearest one: the hit
            // children are taken in slot order without sorting (1.6% less
            // trace time at the bench frame than nearest first).
            const int n = __popc(mask);
            if (sp + n - 1 > kDepth) {
                if (in_tlas) {
                    hit.errors |= 2u;
                    sp = 0;
                    tlas_next = 0;
                } else {
                    hit.errors |= 1u;
                    sp = blas_base;
                    blas_next = inst_first;
                }
                have = false;
                return false;
            }
            const int first = __ffs(mask) - 1;
#pragma unroll
            for (int i = 3; i >= 1; --i)
                if (((mask >> i) & 1u) && i != first) stack[sp++] = make_uint2(child[i], 0u);
            cur = first == 0 ? child[0] : (first == 1 ? child[1] : (first == 2 ? child[2] : child[3]));
            cur_t = 0.0f;
            return false;
        }
        uint32_t k0 = child_key(mask, entry, 0), k1 = child_key(mask, entry, 1);
        uint32_t k2 = child_key(mask, entry, 2), k3 = child_key(mask, entry, 3);
        key_swap(k0, k1);
        key_swap(k2, k3);
        key_swap(k0, k2);
        key_swap(k1, k3);
        key_swap(k1, k2);
        int n = __popc(mask);
        if (sp + n - 1 > kDepth) {
            if (in_tlas) {
                hit.errors |= 2u;
                sp = 0;
                tlas_next = 0;
            } else {
                hit.errors |= 1u;
                sp = blas_base;
                blas_next = inst_first;
            }
            have = false;
            return false;
        }
        if (n > 3) stack[sp++] = make_uint2(key_child(k3, child), k3 & ~3u);
        if (n > 2) stack[sp++] = make_uint2(key_child(k2, child), k2 & ~3u);
        if (n > 1) stack[sp++] = make_uint2(key_child(k1, child), k1 & ~3u);
        cur = key_child(k0, child);
        cur_t = key_entry(k0);
        return false;
    }

    // A TLAS leaf (first, count): enter its first instance (the rest of the
    // leaf waits on the stack).
    __device__ __forceinline__ void enter_instance(const SceneView &S, uint2 *stack, TraceCounters &cn, uint32_t first,
                                                   uint32_t count) {
        // TLAS leaf: enter its first instance; the rest waits on the stack.
        if (count > 1u) {
            if (sp < kDepth) {
                stack[sp++] = make_uint2(kLeafBit | ((first + 1u) & kLeafFirstMask) | ((count - 2u) << 27),
                                         as_uint(cur_t));
            } else {
                // Stack exhausted: after this instance, scan every instance.
                hit.errors |= 2u;
                sp = 0;
                tlas_next = 0;
            }
        }
        DeviceInstance I = load_instance(S.instances, first);
        local_ray(I, o, d, lo, ld);
        cn.instances++;
        // A local direction bit-identical to the world direction
        // (translation-only instances) keeps the world constants;
        // only the origin moves.
        rotated = !(as_uint(ld.x) == as_uint(d.x) && as_uint(ld.y) == as_uint(d.y) &&
                    as_uint(ld.z) == as_uint(d.z));
        if (rotated) {
            r = slab_ray(lo, ld);
            tri_ray = triangle_ray(ld);
        } else {
            r.ox = lo.x;
            r.oy = lo.y;
            r.oz = lo.z;
        }
        inst = first;
        inst_flags = I.flags;
        inst_first = I.first;
        inst_count = I.count;
        blas_base = sp;
        blas_steps = 0;
        cur = I.root;
        cur_t = 0.0f;
        have = true;
    }

    // Inner nodes down to a leaf and that leaf's kind: a TLAS leaf enters its
    // first instance; a BLAS leaf within the step budget is returned as
    // (first, count) for its triangle tests (count 0: none).  Returns true
    // when the query is complete.
    __device__ __forceinline__ bool descend(const SceneView &S, uint2 *stack, TraceCounters &cn, uint32_t &leaf_first,
                                            uint32_t &leaf_count) {
        leaf_first = 0;
        leaf_count = 0;
        while (have && (cur & kLeafBit) == 0u)
            if (node_step(S, stack, cn)) return true;
        if (have) {
            uint32_t first = cur & kLeafFirstMask;
            uint32_t count = ((cur >> 27) & 15u) + 1u;
            have = false;
            if (blas_base < 0) {
                enter_instance(S, stack, cn, first, count);
                return false;
            }
            // BLAS leaf (traceTriangle / occludedTriangle).
            if (++blas_steps > kMaxSteps) {
                hit.errors |= kQueryUnsupported;
                sp = blas_base;
            } else {
                leaf_first = first;
                leaf_count = count;
            }
        }
        return false;
    }

    // The triangles of one BLAS leaf in order; true when an any-hit query is
    // complete.
    __device__ __forceinline__ bool test_leaf(const SceneView &S, uint32_t first, uint32_t count, TraceCounters &cn) {
        {
            {
                for (uint32_t t = first; t < first + count; ++t) {
                    f3 A, B, C;
                    load_triangle(S.triangles, t, A, B, C);
                    cn.triangles++;
                    if (cull_reject(inst_flags, A, B, C, ld)) continue;
                    float w1 = 0.0f, w2 = 0.0f;
                    float dist = intersect_triangle(lo, ld, tri_ray, A, B, C, w1, w2);
                    if (kAnyHit) {
                        if (dist > 0.000025f && dist < hit.t) {
                            // Any accepted blocker is a complete proof
                            // (shaders/traversal.slang:786-792, :1035-1040).
                            hit.tri = t;
                            hit.inst = inst;
                            hit.errors &= ~kQueryUnsupported;
                            return true;
                        }
                    } else if (dist > lower && hit_better(dist, inst, t, hit)) {
                        hit.t = dist;
                        hit.tri = t;
                        hit.inst = inst;
                        hit.b1 = w1;
                        hit.b2 = w2;
                    }
                }
            }
        }
        return false;
    }

    // The next pending entry, leaving instances and fallbacks as needed; true
    // when the query is complete.
    __device__ __forceinline__ bool next(const SceneView &S, uint2 *stack) {
        while (!have) {
            if (blas_base >= 0 && sp == blas_base) {
                if (blas_next != kEmpty && blas_next < inst_first + inst_count) {
                    uint32_t c = min(kLeafMaxCount, inst_first + inst_count - blas_next);
                    cur = kLeafBit | (blas_next & kLeafFirstMask) | ((c - 1u) << 27);
                    blas_next += c;
                    have = true;
                    break;
                }
                blas_next = kEmpty;
                blas_base = -1;
                if (rotated) {
                    r = slab_ray(o, d);
                    tri_ray = triangle_ray(d);
                    rotated = false;
                } else {
                    r.ox = o.x;
                    r.oy = o.y;
                    r.oz = o.z;
                }
                inst = kEmpty;
                continue;
            }
            if (sp == 0) {
                if (tlas_next != kEmpty && tlas_next < S.instance_count) {
                    cur = kLeafBit | (tlas_next & kLeafFirstMask);
                    ++tlas_next;
                    have = true;
                    break;
                }
                return true;
            }
            uint2 top = stack[--sp];
            if (!kAnyHit && as_float(top.y) > hit.t) continue;
            cur = top.x;
            cur_t = as_float(top.y);
            have = true;
        }
        return false;
    }

    // One step: inner nodes down to a leaf, that leaf, then the next pending
    // entry.  Returns true when the query is complete.
    // The stack lives outside the walker so the walker's fields stay in
    // registers; only the stack itself is addressed dynamically.
    __device__ __forceinline__ bool step(const SceneView &S, uint2 *stack, TraceCounters &cn) {
        uint32_t first, count;
        if (descend(S, stack, cn, first, count)) return true;
        if (count && test_leaf(S, first, count, cn)) return true;
        return next(S, stack);
    }

    // The BLAS leaves that the lanes of the warp reached in this step, tested
    // by the whole warp: lane l owns a leaf of count(l) triangles (0: none),
    // the warp's sum(count) (ray, triangle) pairs are dealt out to its lanes
    // in turn, and each owner then takes the best of its candidates.  The
    // closest candidate is the minimum of (distance bits, triangle index)
    // over triangles of one instance, which is the order hit_better applies,
    // so the hit is the one the in-order loop of test_leaf keeps, and the
    // owner re-evaluates the winner for its barycentrics.  For any hit the
    // lowest blocking triangle index is the one the in-order loop stops at,
    // and the owner counts the triangles that loop would have tested.
    // Returns true when the lane's any-hit query is complete.
    __device__ bool leaf_pass(const SceneView &S, LeafScratch *L, uint32_t first, uint32_t count, TraceCounters &cn) {
        const unsigned group = 0xffffffffu;  // every lane of the warp takes part
        const uint32_t lane = threadIdx.x & 31u;
        const unsigned below = (1u << lane) - 1u;
        uint32_t pre = 0, total = 0;
#pragma unroll
        for (int b = 0; b < 5; ++b) {  // leaf counts are at most 16
            const unsigned v = __ballot_sync(group, (count >> b) & 1u);
            pre += (uint32_t)__popc(v & below) << b;
            total += (uint32_t)__popc(v) << b;
        }
        if (total == 0u) return false;
        // Every lane publishes its prefix (non-decreasing in lane order),
        // owners their ray.
        L->pre[lane] = pre;
        if (count) {
            L->ox[lane] = lo.x;
            L->oy[lane] = lo.y;
            L->oz[lane] = lo.z;
            L->dx[lane] = ld.x;
            L->dy[lane] = ld.y;
            L->dz[lane] = ld.z;
            L->sx[lane] = tri_ray.sx;
            L->sy[lane] = tri_ray.sy;
            L->axes[lane] = tri_ray.kx | (tri_ray.ky << 2) | (tri_ray.kz << 4) | (tri_ray.valid ? 64u : 0u);
            L->flags[lane] = inst_flags;
            L->first[lane] = first;
            L->lower[lane] = lower;
            L->limit[lane] = hit.t;
            L->best[lane] = ~0ull;
        }
        __syncwarp(group);
        const uint32_t workers = 32u, me = lane;
        for (uint32_t p = me; p < total; p += workers) {
            // The pair's owner: the highest lane whose prefix is <= p (a lane
            // without a leaf shares its prefix with the next lane, so the
            // highest such lane owns triangles).
            uint32_t o = 0;
#pragma unroll
            for (uint32_t half = 16; half >= 1u; half >>= 1)
                if (o + half < 32u && L->pre[o + half] <= p) o += half;
            const uint32_t t = L->first[o] + (p - L->pre[o]);
            f3 A, B, C;
            load_triangle(S.triangles, t, A, B, C);
            const f3 rd{L->dx[o], L->dy[o], L->dz[o]};
            if (cull_reject(L->flags[o], A, B, C, rd)) continue;
            TriRay tr;
            const uint32_t ax = L->axes[o];
            tr.kx = ax & 3u;
            tr.ky = (ax >> 2) & 3u;
            tr.kz = (ax >> 4) & 3u;
            tr.valid = (ax & 64u) != 0u;
            tr.sx = L->sx[o];
            tr.sy = L->sy[o];
            float w1 = 0.0f, w2 = 0.0f;
            const float dist = intersect_triangle(f3{L->ox[o], L->oy[o], L->oz[o]}, rd, tr, A, B, C, w1, w2);
            if (kAnyHit) {
                if (dist > 0.000025f && dist < L->limit[o]) atomicMin(&L->best[o], (unsigned long long)t);
            } else if (dist > L->lower[o]) {
                atomicMin(&L->best[o], ((unsigned long long)as_uint(dist) << 32) | t);
            }
        }
        __syncwarp(group);
        bool done = false;
        if (count) {
            const unsigned long long b = L->best[lane];
            if (kAnyHit) {
                if (b != ~0ull) {
                    const uint32_t t = (uint32_t)b;
                    cn.triangles += t - first + 1u;
                    hit.tri = t;
                    hit.inst = inst;
                    hit.errors &= ~kQueryUnsupported;
                    done = true;
                } else {
                    cn.triangles += count;
                }
            } else {
                cn.triangles += count;
                if (b != ~0ull) {
                    const float dist = as_float((uint32_t)(b >> 32));
                    const uint32_t t = (uint32_t)b;
                    if (hit_better(dist, inst, t, hit)) {
                        f3 A, B, C;
                        load_triangle(S.triangles, t, A, B, C);
                        float w1 = 0.0f, w2 = 0.0f;
                        intersect_triangle(lo, ld, tri_ray, A, B, C, w1, w2);
                        hit.t = dist;
                        hit.tri = t;
                        hit.inst = inst;
                        hit.b1 = w1;
                        hit.b2 = w2;
                    }
                }
            }
        }
        __syncwarp(group);  // the scratch is rewritten by the next pass
        return done;
    }

    // step() for walks of a whole warp: every lane calls it in every round
    // (alive = the lane still has a query), so the leaf pass runs over the
    // full warp.  Returns true when the lane's query is complete (or it has
    // none).
    __device__ __forceinline__ bool step_warp(const SceneView &S, uint2 *stack, TraceCounters &cn, LeafScratch *L,
                                              bool alive) {
        uint32_t first = 0, count = 0;
        bool complete = !alive;
        if (alive) complete = descend(S, stack, cn, first, count);
        if (complete) count = 0;
        if (leaf_pass(S, L, first, count, cn)) complete = true;
        if (complete) return true;
        return next(S, stack);
    }
};

// Closest hit (kAnyHit = false) or any hit of one ray.  kDepth is the stack
// depth: a shallower stack uses less local memory per thread, and a walk that
// overflows it continues with the reference's ordered scan (same answers).
template <bool kAnyHit, int kDepth = kStack>
__device__ void trace(const SceneView &S, f3 o, f3 d, float tmin, float limit, Hit &hit, TraceCounters &cn) {
    Walker<kAnyHit, kDepth> w;
    uint2 stack[kDepth];
    if (w.start(S, o, d, tmin, limit))
        while (!w.step(S, stack, cn)) {
        }
    hit = w.hit;
}

// trace() for a whole warp: every lane of the warp calls it (active: the
// lane has a query), and the BLAS leaves reached in each round are tested
// by the whole warp (Walker::leaf_pass).  A lane without a query returns no
// hit.
template <bool kAnyHit, int kDepth = kStack>
__device__ void trace_warp(const SceneView &S, bool active, f3 o, f3 d, float tmin, float limit, Hit &hit,
                           TraceCounters &cn, LeafScratch *L) {
    Walker<kAnyHit, kDepth> w;
    w.hit = Hit{limit, kEmpty, kEmpty, 0u, 0.0f, 0.0f};
    uint2 stack[kDepth];
    bool alive = active && w.start(S, o, d, tmin, limit);
    while (__any_sync(0xffffffffu, alive)) {
        const bool complete = w.step_warp(S, stack, cn, L, alive);
        alive = alive && !complete;
    }
    hit = w.hit;
}

// Persistent warp loop with per-lane refill: whenever lanes are idle, the
// warp takes that many new rays from `counter` (one atomic per refill) and
// keeps stepping until the counter passes `n` and every lane is done.
// gen(id, o, d, tmin, limit) produces ray `id`; done(id, hit) consumes it.
// With a leaf scratch (L), the warp's walks step together and the leaves of
// each round are tested by the whole warp (Walker::step_warp).
template <bool kAnyHit, typename Gen, typename Done>
__device__ void trace_persistent(const SceneView &S, uint32_t *counter, uint32_t n, Gen &&gen, Done &&done,
                                 TraceCounters &cn, LeafScratch *L = nullptr) {
    const uint32_t lane = threadIdx.x & 31u;
    Walker<kAnyHit> w;
    uint2 stack[kStack];
    bool active = false;
    bool exhausted = false;  // the counter passed n: no further rays for this warp
    uint32_t id = 0;
    while (true) {
        uint32_t need = __ballot_sync(0xffffffffu, !active && !exhausted);
        if (need) {
            uint32_t leader = __ffs(need) - 1u;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(need));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base + (uint32_t)__popc(need) > n) exhausted = true;  // uniform across the warp
            if (!active && (need & (1u << lane))) {
                id = base + (uint32_t)__popc(need & ((1u << lane) - 1u));
                if (id < n) {
                    f3 o, d;
                    float tmin, limit;
                    gen(id, o, d, tmin, limit);
                    active = w.start(S, o, d, tmin, limit);
                    if (!active) done(id, w.hit);
                }
            }
        }
        if (!__any_sync(0xffffffffu, active)) {
            if (exhausted) break;
            continue;
        }
        const bool complete = L ? w.step_warp(S, stack, cn, L, active) : (active && w.step(S, stack, cn));
        if (active && complete) {
            done(id, w.hit);
            active = false;
        }
    }
}

}  // namespace lux
