// scene.cu - scene upload (reference words -> device BVH4) and the
// traversal harness entry point lux_trace_rays.
//
// Upload validates the reference's word streams (src/scene.rs:2096-2117,
// :809-823), collapses every binary BVH built by build_tree
// (src/scene.rs:2398-2554) into a 4-wide BVH whose child boxes are the binary
// nodes' boxes, gathers triangle positions into leaf order (3 x 16 bytes per
// triangle), and keeps the verbatim words on the device for hit shading.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "lux_internal.h"
#include "lux_math.cuh"
#include "traverse.cuh"

namespace {

struct BinNode {
    float mn[3], mx[3];
    uint32_t first, count;
};

inline float fword(const uint32_t *w, size_t i) {
    float f;
    std::memcpy(&f, &w[i], 4);
    return f;
}

struct Collapser {
    const std::vector<BinNode> &bin;
    std::vector<Bvh4Node> &out;
    std::string error;
    uint32_t leaf_limit;  // elements addressable by a leaf (triangles or instances)
    // Per-element world boxes (TLAS only): a leaf of 2-4 instances becomes a
    // node whose children are single instances with their own boxes, so an
    // instance is entered (ray transform, BLAS root test) only when the ray
    // meets that instance's box rather than the whole leaf's.
    const std::vector<BinNode> *element_box = nullptr;
    // Where each child slot's box comes from (TLAS only, for refit):
    // (binary node, instance) -- the instance is kEmpty unless the slot is a
    // single-instance child cut from binary leaf `x`.
    std::vector<uint2> *sources = nullptr;
    // Binary nodes already taken into the BVH4, shared by the TLAS and every
    // BLAS collapse of one upload: build_tree (src/scene.rs:2398-2554) emits
    // trees, so a node reached a second time means the words hold a cycle or
    // a shared subtree.  Rejecting it keeps the collapse linear in the node
    // count (a shared subtree repeated at every level would otherwise double
    // the work per level).
    std::vector<uint8_t> *seen = nullptr;

    bool visit(uint32_t index) {
        if ((*seen)[index]) {
            error = "BVH node reached twice (the node words do not form a tree)";
            return false;
        }
        (*seen)[index] = 1;
        return true;
    }

    static double area(const BinNode &n) {
        double sx = (double)n.mx[0] - n.mn[0], sy = (double)n.mx[1] - n.mn[1], sz = (double)n.mx[2] - n.mn[2];
        return 2.0 * (sx * sy + sy * sz + sz * sx);
    }

    uint32_t new_node() {
        Bvh4Node n;
        for (int i = 0; i < 4; ++i) {
            n.lo_x[i] = n.lo_y[i] = n.lo_z[i] = INFINITY;
            n.hi_x[i] = n.hi_y[i] = n.hi_z[i] = -INFINITY;
            n.child[i] = lux::kEmpty;
            n.pad[i] = 0;
        }
        out.push_back(n);
        if (sources)
            for (int i = 0; i < 4; ++i) sources->push_back(make_uint2(lux::kEmpty, lux::kEmpty));
        return (uint32_t)out.size() - 1;
    }

    void set_child(uint32_t node, int slot, const float mn[3], const float mx[3], uint32_t payload,
                   uint32_t bin_index, uint32_t instance = lux::kEmpty) {
        if (sources) (*sources)[4 * (size_t)node + slot] = make_uint2(bin_index, instance);
        Bvh4Node &n = out[node];
        n.lo_x[slot] = mn[0];
        n.lo_y[slot] = mn[1];
        n.lo_z[slot] = mn[2];
        n.hi_x[slot] = mx[0];
        n.hi_y[slot] = mx[1];
        n.hi_z[slot] = mx[2];
        n.child[slot] = payload;
    }

    // A leaf of `count` elements as one payload; ranges above 16 elements
    // become a small subtree of 16-element leaves with the leaf's box.
    uint32_t leaf_payload(uint32_t first, uint32_t count, const float mn[3], const float mx[3], uint32_t bin_index) {
        if (count <= kLeafMaxCount) return kLeafBit | (first & kLeafFirstMask) | ((count - 1u) << 27);
        uint32_t per = (count + 3u) / 4u;
        uint32_t node = new_node();
        int slot = 0;
        for (uint32_t start = 0; start < count && slot < 4; start += per, ++slot) {
            uint32_t c = std::min(per, count - start);
            uint32_t p = leaf_payload(first + start, c, mn, mx, bin_index);
            set_child(node, slot, mn, mx, p, bin_index);
        }
        return node;
    }

    // Payload of binary subtree `index`.
    uint32_t collapse(uint32_t index, int depth) {
        if (index >= bin.size() || depth > 96) {
            error = "BVH node index out of range or cyclic";
            return lux::kEmpty;
        }
        if (!visit(index)) return lux::kEmpty;
        const BinNode &b = bin[index];
        if (b.count > 0) {
            if ((uint64_t)b.first + b.count > leaf_limit || b.first + b.count > kLeafFirstMask) {
                error = "BVH leaf range exceeds the element array";
                return lux::kEmpty;
            }
            if (b.count > 256u) {
                error = "BVH leaf holds more than 256 elements";
                return lux::kEmpty;
            }
            if (element_box && b.count >= 2u && b.count <= 4u) {
                uint32_t node = new_node();
                for (uint32_t k = 0; k < b.count; ++k) {
                    const BinNode &e = (*element_box)[b.first + k];
                    float mn[3], mx[3];
                    for (int a = 0; a < 3; ++a) {
                        mn[a] = std::max(e.mn[a], b.mn[a]);
                        mx[a] = std::min(e.mx[a], b.mx[a]);
                    }
                    set_child(node, (int)k, mn, mx, kLeafBit | ((b.first + k) & kLeafFirstMask), index, b.first + k);
                }
                return node;
            }
            return leaf_payload(b.first, b.count, b.mn, b.mx, index);
        }
        if ((size_t)b.first + 1 >= bin.size()) {
            error = "BVH child index out of range";
            return lux::kEmpty;
        }
        std::vector<uint32_t> kids = {b.first, b.first + 1};
        while (kids.size() < 4) {
            int best = -1;
            double best_area = -1.0;
            for (size_t k = 0; k < kids.size(); ++k) {
                const BinNode &c = bin[kids[k]];
                if (c.count == 0 && (size_t)c.first + 1 < bin.size()) {
                    double a = area(c);
                    if (a > best_area) {
                        best_area = a;
                        best = (int)k;
                    }
                }
            }
            if (best < 0) break;
            uint32_t c = kids[best];
            if (!visit(c)) return lux::kEmpty;
            kids.erase(kids.begin() + best);
            kids.push_back(bin[c].first);
            kids.push_back(bin[c].first + 1);
        }
        uint32_t node = new_node();
        for (size_t k = 0; k < kids.size(); ++k) {
            uint32_t p = collapse(kids[k], depth + 1);
            if (!error.empty()) return lux::kEmpty;
            set_child(node, (int)k, bin[kids[k]].mn, bin[kids[k]].mx, p, kids[k]);
        }
        return node;
    }

    // Payload usable as a traversal start: a node index.
    uint32_t root(uint32_t index) {
        uint32_t p = collapse(index, 0);
        if (!error.empty()) return lux::kEmpty;
        if ((p & kLeafBit) == 0u) return p;
        uint32_t node = new_node();
        set_child(node, 0, bin[index].mn, bin[index].mx, p, index);
        return node;
    }
};

// 128 threads per block; every lane of a warp walks together (whole-warp
// leaf tests), lanes past `count` without a query.
__global__ void __launch_bounds__(128) trace_rays_kernel(SceneView S, const LuxRay *__restrict__ rays, uint32_t count,
                                                         uint32_t any_hit, LuxHit *__restrict__ hits,
                                                         unsigned long long *__restrict__ counters) {
    __shared__ lux::LeafScratch scratch[4];
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    lux::TraceCounters cn{0, 0, 0};
    const bool active = i < count;
    LuxRay r{};
    if (active) r = rays[i];
    lux::f3 o{r.origin[0], r.origin[1], r.origin[2]};
    lux::f3 d{r.direction[0], r.direction[1], r.direction[2]};
    lux::Hit h;
    lux::LeafScratch *L = &scratch[threadIdx.x >> 5];
    if (any_hit)
        lux::trace_warp<true>(S, active, o, d, 0.0f, r.limit, h, cn, L);
    else
        lux::trace_warp<false>(S, active, o, d, r.tmin, r.limit, h, cn, L);
    if (active) {
        LuxHit out;
        out.distance = h.t;
        out.triangle = h.tri;
        out.instance = h.inst;
        out.errors = h.errors;
        out.barycentric[0] = (1.0f - h.b1) - h.b2;
        out.barycentric[1] = h.b1;
        out.barycentric[2] = h.b2;
        out.visited = cn.nodes;
        hits[i] = out;
    }
    if (counters) {
        unsigned long long n = cn.nodes, t = cn.triangles, in = cn.instances;
        for (int off = 16; off > 0; off >>= 1) {
            n += __shfl_down_sync(0xffffffffu, n, off);
            t += __shfl_down_sync(0xffffffffu, t, off);
            in += __shfl_down_sync(0xffffffffu, in, off);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&counters[0], n);
            atomicAdd(&counters[1], t);
            atomicAdd(&counters[2], in);
        }
    }
}

__device__ __forceinline__ float4 word_f4(const uint4 w) {
    return make_float4(lux::as_float(w.x), lux::as_float(w.y), lux::as_float(w.z), lux::as_float(w.w));
}

// Conservative world box of one instance (refitTlas's leaf loop,
// shaders/acceleration.slang:73-84), its error term scaled by `pad`: the
// BLAS root box's centre and half extent through world_from_local (rows
// 3-5), widened by (|t| + |M| max(|lo|, |hi|)) * 9.536743164e-7 * pad.
__device__ void instance_world_box(const uint4 *__restrict__ sw, uint32_t inst_base, uint32_t instance, float pad,
                                   float mn[3], float mx[3]) {
    uint32_t base = inst_base + instance * 9u;
    uint32_t root = sw[base + 8].x;
    uint4 la = sw[1 + root * 2], ub = sw[2 + root * 2];
    float a[3] = {lux::as_float(la.x), lux::as_float(la.y), lux::as_float(la.z)};
    float b[3] = {lux::as_float(ub.x), lux::as_float(ub.y), lux::as_float(ub.z)};
    float center[3], extent[3], absolute[3];
    for (int k = 0; k < 3; ++k) {
        center[k] = a[k] * 0.5f + b[k] * 0.5f;
        extent[k] = b[k] * 0.5f - a[k] * 0.5f;
        absolute[k] = fmaxf(fabsf(a[k]), fabsf(b[k]));
    }
    for (int r = 0; r < 3; ++r) {
        float4 row = word_f4(sw[base + 3 + r]);
        float wc = ((row.x * center[0] + row.y * center[1]) + row.z * center[2]) + row.w * 1.0f;
        float we = (fabsf(row.x) * extent[0] + fabsf(row.y) * extent[1]) + fabsf(row.z) * extent[2];
        float err = (fabsf(row.w) + ((fabsf(row.x) * absolute[0] + fabsf(row.y) * absolute[1]) +
                                     fabsf(row.z) * absolute[2])) * 9.536743164e-7f;
        err = err * pad;
        mn[r] = (wc - we) - err;
        mx[r] = (wc + we) + err;
    }
}

// refitTlas (shaders/acceleration.slang:61-88) for every depth in one block:
// `order` lists the binary TLAS nodes deepest depth first, so each pass
// reads children written by the previous one (a block barrier between
// depths).  Then every TLAS BVH4 child slot takes the refit box of the
// binary node it was collapsed from; single-instance slots take the
// instance's own box (error term x8, so it contains refitTlas's) cut by the
// refit leaf box.
__global__ void __launch_bounds__(1024) refit_kernel(uint4 *__restrict__ sw, uint32_t inst_base,
                                                     const uint32_t *__restrict__ order,
                                                     const uint32_t *__restrict__ depth_start, uint32_t depths,
                                                     Bvh4Node *__restrict__ nodes, const uint2 *__restrict__ source,
                                                     uint32_t slots) {
    for (uint32_t d = 0; d < depths; ++d) {
        for (uint32_t k = depth_start[d] + threadIdx.x; k < depth_start[d + 1]; k += blockDim.x) {
            uint32_t node = order[k];
            uint4 lower = sw[1 + node * 2], upper = sw[2 + node * 2];
            float mn[3] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
            float mx[3] = {-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f};
            if (upper.w == 0u) {
                uint32_t child = lower.w;
                uint4 a0 = sw[1 + child * 2], a1 = sw[1 + (child + 1) * 2];
                uint4 b0 = sw[2 + child * 2], b1 = sw[2 + (child + 1) * 2];
                mn[0] = fminf(lux::as_float(a0.x), lux::as_float(a1.x));
                mn[1] = fminf(lux::as_float(a0.y), lux::as_float(a1.y));
                mn[2] = fminf(lux::as_float(a0.z), lux::as_float(a1.z));
                mx[0] = fmaxf(lux::as_float(b0.x), lux::as_float(b1.x));
                mx[1] = fmaxf(lux::as_float(b0.y), lux::as_float(b1.y));
                mx[2] = fmaxf(lux::as_float(b0.z), lux::as_float(b1.z));
            } else {
                for (uint32_t i = lower.w; i < lower.w + upper.w; ++i) {
                    float a[3], b[3];
                    instance_world_box(sw, inst_base, i, 1.0f, a, b);
                    for (int r = 0; r < 3; ++r) {
                        mn[r] = fminf(mn[r], a[r]);
                        mx[r] = fmaxf(mx[r], b[r]);
                    }
                }
            }
            sw[1 + node * 2] = make_uint4(lux::as_uint(mn[0]), lux::as_uint(mn[1]), lux::as_uint(mn[2]), lower.w);
            sw[2 + node * 2] = make_uint4(lux::as_uint(mx[0]), lux::as_uint(mx[1]), lux::as_uint(mx[2]), upper.w);
        }
        __syncthreads();
    }
    for (uint32_t slot = threadIdx.x; slot < slots; slot += blockDim.x) {
        uint2 src = source[slot];
        if (src.x == lux::kEmpty) continue;
        uint4 la = sw[1 + src.x * 2], ub = sw[2 + src.x * 2];
        float mn[3] = {lux::as_float(la.x), lux::as_float(la.y), lux::as_float(la.z)};
        float mx[3] = {lux::as_float(ub.x), lux::as_float(ub.y), lux::as_float(ub.z)};
        if (src.y != lux::kEmpty) {
            float a[3], b[3];
            instance_world_box(sw, inst_base, src.y, 8.0f, a, b);
            for (int r = 0; r < 3; ++r) {
                mn[r] = fmaxf(mn[r], a[r]);
                mx[r] = fminf(mx[r], b[r]);
            }
        }
        Bvh4Node &n = nodes[slot / 4];
        uint32_t c = slot % 4;
        n.lo_x[c] = mn[0];
        n.lo_y[c] = mn[1];
        n.lo_z[c] = mn[2];
        n.hi_x[c] = mx[0];
        n.hi_y[c] = mx[1];
        n.hi_z[c] = mx[2];
    }
}

}  // namespace

// Host half of an upload: validation of the reference word streams, the
// BVH4 collapse of the TLAS and every distinct BLAS, and the leaf-ordered
// triangle positions.  Needs no device.
struct HostScene {
    std::vector<Bvh4Node> nodes;
    std::vector<float4> tris;
    std::vector<DeviceInstance> inst;
    std::vector<uint2> slot_source;
    std::vector<uint32_t> refit_order, depth_start;
    uint32_t tlas_root = lux::kEmpty, inst_base = 0, inst_count = 0, tri_count = 0, tlas_slots = 0;
    float root_lo[3] = {0, 0, 0}, root_hi[3] = {0, 0, 0};
};

static lux_status prepare_scene(const uint32_t *sw, size_t sn, const uint32_t *gw, size_t gn, const LuxLight *lights,
                                uint32_t light_count, uint32_t conventional, HostScene &H, std::string &message) {
    auto fail = [&](lux_status status, const std::string &text) {
        message = text;
        return status;
    };
    std::vector<Bvh4Node> &nodes = H.nodes;
    std::vector<uint2> &slot_source = H.slot_source;
    std::vector<uint32_t> &refit_order = H.refit_order, &depth_start = H.depth_start;
    if (!sw || sn < 1 || !gw || gn < 1 || (light_count && !lights) || conventional > light_count)
        return fail(LUX_ERR_INVALID_ARGUMENT, "scene upload: missing words or lights");
    if (conventional >= 16u)
        return fail(LUX_ERR_CAPACITY,
                        "scene upload: at most 15 conventional lights (a hit's next-event slots are shared with the "
                        "emissive samples)");
    for (uint32_t l = 0; l < conventional; ++l) {
        const LuxLight &L = lights[l];
        for (int c = 0; c < 4; ++c)
            if (!std::isfinite(L.position[c]) || !std::isfinite(L.color[c]) || !std::isfinite(L.direction[c]))
                return fail(LUX_ERR_MALFORMED_SCENE, "scene upload: conventional light with non-finite fields");
    }
    if (sn > 0xffffffffu || gn > 0xffffffffu)
        return fail(LUX_ERR_MALFORMED_SCENE, "scene upload: word stream exceeds 2^32 words");
    // Header (src/scene.rs:2103-2110): material end, instance base, count, stride.
    uint32_t inst_base = sw[1], inst_count = sw[2], stride = sw[3];
    if (stride != 9u || (uint64_t)inst_base + (uint64_t)inst_count * 9u > sn)
        return fail(LUX_ERR_MALFORMED_SCENE, "scene upload: instance records outside the scene words");
    if (inst_count > kLeafFirstMask)
        return fail(LUX_ERR_MALFORMED_SCENE, "scene upload: too many instances");
    uint32_t node_words = inst_base - 1u;
    uint32_t node_count = node_words / 2u;
    std::vector<BinNode> bin(node_count);
    for (uint32_t i = 0; i < node_count; ++i) {
        const uint32_t *a = sw + 4 * (size_t)(1 + 2 * i), *b = sw + 4 * (size_t)(2 + 2 * i);
        for (int k = 0; k < 3; ++k) {
            std::memcpy(&bin[i].mn[k], &a[k], 4);
            std::memcpy(&bin[i].mx[k], &b[k], 4);
        }
        bin[i].first = a[3];
        bin[i].count = b[3];
    }
    // Geometry header (src/scene.rs:809-823).
    uint32_t tri_word = gw[0], vertex_base = gw[1], vertex_stride = gw[2], vertex_count = gw[3];
    if (tri_word != 1u || vertex_stride != 5u || vertex_base < 1u || (uint64_t)vertex_base + (uint64_t)vertex_count * 5u > gn)
        return fail(LUX_ERR_MALFORMED_SCENE, "scene upload: malformed geometry header");
    uint32_t tri_capacity = vertex_base - 1u;
    std::vector<DeviceInstance> &inst = H.inst;
    inst.assign(inst_count, DeviceInstance{});
    uint32_t tri_count = 0;
    for (uint32_t i = 0; i < inst_count; ++i) {
        const uint32_t *w = sw + 4 * (size_t)(inst_base + 9 * i);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 4; ++c) inst[i].row[r][c] = fword(w, 4 * r + c);
        inst[i].flags = w[4 * 6 + 3];
        uint32_t material = w[4 * 7 + 3];
        inst[i].first = w[4 * 8 + 1];
        inst[i].count = w[4 * 8 + 2];
        inst[i].root = w[4 * 8 + 0];
        if ((uint64_t)inst[i].first + inst[i].count > tri_capacity)
            return fail(LUX_ERR_MALFORMED_SCENE, "scene upload: instance triangle range outside geometry");
        if (inst[i].root >= node_count)
            return fail(LUX_ERR_MALFORMED_SCENE, "scene upload: instance BLAS root outside the node words");
        if ((uint64_t)material + 8 > sn)
            return fail(LUX_ERR_MALFORMED_SCENE, "scene upload: material record outside the scene words");
        const uint32_t *m = sw + 4 * (size_t)material;
        float cutoff;
        std::memcpy(&cutoff, &m[7], 4);
        if (cutoff != -1.0f)
            return fail(LUX_ERR_MALFORMED_SCENE,
                            "scene upload: alpha-tested materials are not supported by this build");
        const uint32_t *tex = m + 4 * 6;
        if (tex[0] != lux::kEmpty || tex[1] != lux::kEmpty || tex[2] != lux::kEmpty || tex[3] != lux::kEmpty ||
            m[4 * 7] != lux::kEmpty)
            return fail(LUX_ERR_MALFORMED_SCENE,
                            "scene upload: textured materials are not supported by this build");
        tri_count = std::max(tri_count, inst[i].first + inst[i].count);
    }
    // World box of every instance: the eight corners of its BLAS root box
    // through world_from_local (instance rows 3-5) in f64, padded by 2^-17
    // of the coordinate magnitude plus the box extent.  The reference's
    // instance box (src/scene.rs:1911-1924) is the same transformed box padded
    // by 8 f32 epsilons of the magnitudes, so this box contains it, and the
    // child box (this box cut by the TLAS leaf's box, which is a union of
    // reference instance boxes) never culls more than the reference's own
    // box for that instance would.
    std::vector<BinNode> inst_box(inst_count);
    for (uint32_t i = 0; i < inst_count; ++i) {
        const uint32_t *w = sw + 4 * (size_t)(inst_base + 9 * i);
        double m[3][4];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 4; ++c) m[r][c] = (double)fword(w, 12 + 4 * r + c);
        const BinNode &rb = bin[inst[i].root];
        double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int corner = 0; corner < 8; ++corner) {
            double q[3] = {(corner & 1) ? rb.mx[0] : rb.mn[0], (corner & 2) ? rb.mx[1] : rb.mn[1],
                           (corner & 4) ? rb.mx[2] : rb.mn[2]};
            for (int r = 0; r < 3; ++r) {
                double v = m[r][0] * q[0] + m[r][1] * q[1] + m[r][2] * q[2] + m[r][3];
                mn[r] = std::min(mn[r], v);
                mx[r] = std::max(mx[r], v);
            }
        }
        BinNode &b = inst_box[i];
        for (int r = 0; r < 3; ++r) {
            double pad = (std::max(std::fabs(mn[r]), std::fabs(mx[r])) + (mx[r] - mn[r])) * 7.62939453125e-6 + 1e-30;
            bool finite = std::isfinite(mn[r]) && std::isfinite(mx[r]);
            b.mn[r] = finite ? (float)(mn[r] - pad) : -INFINITY;
            b.mx[r] = finite ? (float)(mx[r] + pad) : INFINITY;
        }
        b.first = i;
        b.count = 1;
    }
    // Collapse: TLAS from node 0, every distinct BLAS root once.
    std::vector<uint8_t> seen(node_count, 0);
    nodes.reserve(node_count / 2 + 16);
    uint32_t &tlas_root = H.tlas_root;
    float *root_lo = H.root_lo, *root_hi = H.root_hi;
    if (inst_count > 0) {
        if (node_count == 0) return fail(LUX_ERR_MALFORMED_SCENE, "scene upload: no TLAS nodes");
        Collapser tl{bin, nodes, {}, inst_count, &inst_box, &slot_source, &seen};
        tlas_root = tl.root(0);
        if (!tl.error.empty()) return fail(LUX_ERR_MALFORMED_SCENE, "scene upload (TLAS): " + tl.error);
        for (int k = 0; k < 3; ++k) {
            root_lo[k] = bin[0].mn[k];
            root_hi[k] = bin[0].mx[k];
        }
        // Binary TLAS nodes grouped by depth, deepest first: the pass order
        // of refitTlas (shaders/acceleration.slang:61), where each depth's
        // children are final before their parents read them.
        std::vector<std::vector<uint32_t>> by_depth;
        std::vector<std::pair<uint32_t, uint32_t>> todo = {{0u, 0u}};
        while (!todo.empty()) {
            auto [index, depth] = todo.back();
            todo.pop_back();
            if (by_depth.size() <= depth) by_depth.resize(depth + 1);
            by_depth[depth].push_back(index);
            if (bin[index].count == 0) {
                todo.push_back({bin[index].first, depth + 1});
                todo.push_back({bin[index].first + 1, depth + 1});
            }
        }
        for (size_t d = by_depth.size(); d-- > 0;) {
            depth_start.push_back((uint32_t)refit_order.size());
            refit_order.insert(refit_order.end(), by_depth[d].begin(), by_depth[d].end());
        }
        depth_start.push_back((uint32_t)refit_order.size());
    }
    uint32_t tlas_slots = (uint32_t)slot_source.size();
    std::unordered_map<uint32_t, uint32_t> blas_root;
    for (uint32_t i = 0; i < inst_count; ++i) {
        auto it = blas_root.find(inst[i].root);
        if (it == blas_root.end()) {
            Collapser bl{bin, nodes, {}, tri_count, nullptr, nullptr, &seen};
            uint32_t r = bl.root(inst[i].root);
            if (!bl.error.empty()) return fail(LUX_ERR_MALFORMED_SCENE, "scene upload (BLAS): " + bl.error);
            it = blas_root.emplace(inst[i].root, r).first;
        }
        inst[i].root = it->second;
    }
    // Triangle positions in packed (leaf) order.
    std::vector<float4> &tris = H.tris;
    tris.assign(3 * (size_t)std::max(tri_count, 1u), float4{});
    for (uint32_t t = 0; t < tri_count; ++t) {
        const uint32_t *idx = gw + 4 * (size_t)(1 + t);
        for (int v = 0; v < 3; ++v) {
            uint32_t vi = idx[v];
            if (vi >= vertex_count) return fail(LUX_ERR_MALFORMED_SCENE, "scene upload: vertex index out of range");
            const uint32_t *p = gw + 4 * ((size_t)vertex_base + (size_t)vi * 5u);
            float4 f;
            std::memcpy(&f.x, &p[0], 4);
            std::memcpy(&f.y, &p[1], 4);
            std::memcpy(&f.z, &p[2], 4);
            f.w = 0.0f;
            tris[3 * (size_t)t + v] = f;
        }
    }
    if (light_count > conventional) {
        for (uint32_t l = conventional; l < light_count; ++l)
            if (lights[l].source[0] >= inst_count || lights[l].source[1] >= tri_capacity)
                return fail(LUX_ERR_MALFORMED_SCENE, "scene upload: emitter record outside the scene");
    }
    H.inst_base = inst_base;
    H.inst_count = inst_count;
    H.tri_count = tri_count;
    H.tlas_slots = tlas_slots;
    return LUX_OK;
}

extern "C" lux_status lux_scene_validate(const uint32_t *sw, size_t sn, const uint32_t *gw, size_t gn,
                                         const LuxLight *lights, uint32_t light_count, uint32_t conventional,
                                         char *message, size_t message_size) {
    HostScene H;
    std::string text;
    lux_status status = prepare_scene(sw, sn, gw, gn, lights, light_count, conventional, H, text);
    if (message && message_size) {
        size_t n = std::min(text.size(), message_size - 1);
        std::memcpy(message, text.data(), n);
        message[n] = '\0';
    }
    return status;
}

extern "C" lux_status lux_scene_upload(LuxContext *ctx, const uint32_t *sw, size_t sn, const uint32_t *gw, size_t gn,
                                       const LuxLight *lights, uint32_t light_count, uint32_t conventional,
                                       LuxScene **out) {
    if (!ctx || !out) return LUX_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    HostScene H;
    std::string message;
    lux_status prep = prepare_scene(sw, sn, gw, gn, lights, light_count, conventional, H, message);
    if (prep != LUX_OK) return lux_fail(ctx, prep, message);
    const std::vector<Bvh4Node> &nodes = H.nodes;
    const std::vector<float4> &tris = H.tris;
    const std::vector<DeviceInstance> &inst = H.inst;
    const std::vector<uint2> &slot_source = H.slot_source;
    const std::vector<uint32_t> &refit_order = H.refit_order, &depth_start = H.depth_start;
    const uint32_t tlas_root = H.tlas_root, inst_base = H.inst_base, inst_count = H.inst_count;
    const uint32_t tri_count = H.tri_count, tlas_slots = H.tlas_slots;
    const float *root_lo = H.root_lo, *root_hi = H.root_hi;
    LuxScene *S = new LuxScene();
    S->ctx = ctx;
    auto alloc_copy = [&](void **dst, const void *src, size_t bytes) -> bool {
        if (bytes == 0) {
            bytes = 16;
            src = nullptr;
        }
        if (cudaMalloc(dst, bytes) != cudaSuccess) return false;
        if (src && cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return false;
        return true;
    };
    bool ok = alloc_copy(&S->d_nodes, nodes.data(), nodes.size() * sizeof(Bvh4Node)) &&
              alloc_copy(&S->d_tris, tris.data(), tris.size() * sizeof(float4)) &&
              alloc_copy(&S->d_inst, inst.data(), inst.size() * sizeof(DeviceInstance)) &&
              alloc_copy(&S->d_sw, sw, sn * 16) && alloc_copy(&S->d_gw, gw, gn * 16) &&
              alloc_copy(&S->d_lights, lights, (size_t)light_count * sizeof(LuxLight)) &&
              alloc_copy((void **)&S->d_refit_order, refit_order.data(), refit_order.size() * 4) &&
              alloc_copy((void **)&S->d_depth_start, depth_start.data(), depth_start.size() * 4) &&
              alloc_copy((void **)&S->d_slot_source, slot_source.data(), slot_source.size() * sizeof(uint2));
    if (!ok) {
        cudaGetLastError();
        lux_scene_destroy(S);
        return lux_fail(ctx, LUX_ERR_OUT_OF_MEMORY, "scene upload: device allocation failed");
    }
    SceneView &V = S->view;
    V.nodes = (const Bvh4Node *)S->d_nodes;
    V.triangles = (const float4 *)S->d_tris;
    V.instances = (const DeviceInstance *)S->d_inst;
    V.scene_words = (const uint4 *)S->d_sw;
    V.geometry_words = (const uint4 *)S->d_gw;
    V.lights = (const LuxLight *)S->d_lights;
    V.tlas_root = tlas_root;
    V.instance_count = inst_count;
    V.triangle_count = tri_count;
    V.scene_word_count = (uint32_t)sn;
    V.geometry_word_count = (uint32_t)gn;
    V.conventional_lights = conventional;
    V.emissive_lights = light_count - conventional;
    for (int k = 0; k < 3; ++k) {
        V.root_lo[k] = root_lo[k];
        V.root_hi[k] = root_hi[k];
    }
    S->node_count = (uint32_t)nodes.size();
    S->instance_base = inst_base;
    S->instance_words.assign(sw + 4 * (size_t)inst_base, sw + 4 * ((size_t)inst_base + 9 * (size_t)inst_count));
    S->instances = inst;
    S->depth_start = depth_start;
    S->slot_count = tlas_slots;
    S->light_count = light_count;
    *out = S;
    return LUX_OK;
}

extern "C" lux_status lux_scene_destroy(LuxScene *S) {
    if (!S) return LUX_OK;
    cudaFree(S->d_nodes);
    cudaFree(S->d_tris);
    cudaFree(S->d_inst);
    cudaFree(S->d_sw);
    cudaFree(S->d_gw);
    cudaFree(S->d_lights);
    cudaFree(S->d_refit_order);
    cudaFree(S->d_depth_start);
    cudaFree(S->d_slot_source);
    delete S;
    return LUX_OK;
}

extern "C" lux_status lux_scene_layout(const LuxScene *S, uint32_t *nodes, uint32_t *node_bytes, uint32_t *triangles,
                                       uint32_t *triangle_bytes, uint32_t *instances) {
    if (!S) return LUX_ERR_INVALID_ARGUMENT;
    if (nodes) *nodes = S->node_count;
    if (node_bytes) *node_bytes = (uint32_t)sizeof(Bvh4Node);
    if (triangles) *triangles = S->view.triangle_count;
    if (triangle_bytes) *triangle_bytes = 48u;
    if (instances) *instances = S->view.instance_count;
    return LUX_OK;
}

extern "C" lux_status lux_scene_refit(LuxScene *S, const float *wfl, uint32_t count, const LuxLight *lights,
                                      uint32_t light_count) {
    if (!S) return LUX_ERR_INVALID_ARGUMENT;
    LuxContext *ctx = S->ctx;
    uint32_t n = S->view.instance_count;
    if (count != n || (n && !wfl))
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "scene refit: need one world_from_local per instance");
    if (lights && light_count != S->light_count)
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "scene refit: light count differs from the upload");
    if (lights)
        for (uint32_t l = S->view.conventional_lights; l < light_count; ++l)
            if (lights[l].source[0] >= n)
                return lux_fail(ctx, LUX_ERR_MALFORMED_SCENE, "scene refit: emitter record outside the scene");
    if (n == 0 && !lights) return LUX_OK;
    // Host half: instance rows 0-5 and the device instances' local_from_world.
    std::vector<uint32_t> words = S->instance_words;
    std::vector<DeviceInstance> inst = S->instances;
    for (uint32_t i = 0; i < n; ++i) {
        const float *m = wfl + 12 * (size_t)i;
        for (int k = 0; k < 12; ++k)
            if (!std::isfinite(m[k]))
                return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "scene refit: non-finite transform");
        float lfw[12];
        if (!lux_affine_inverse(m, lfw))
            return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "scene refit: singular transform");
        uint32_t *w = words.data() + 36 * (size_t)i;
        for (int k = 0; k < 12; ++k) {
            std::memcpy(&w[k], &lfw[k], 4);
            std::memcpy(&w[12 + k], &m[k], 4);
        }
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 4; ++c) inst[i].row[r][c] = lfw[4 * r + c];
    }
    cudaStream_t st = ctx->stream;
    cudaSetDevice(ctx->device);
    uint4 *sw = (uint4 *)S->d_sw;
    lux_status rc = LUX_OK;
    if (n) {
        rc = lux_cuda_check(ctx, (int)cudaMemcpyAsync(sw + S->instance_base, words.data(), words.size() * 4,
                                                      cudaMemcpyHostToDevice, st),
                            "scene refit: instance words");
        if (rc == LUX_OK)
            rc = lux_cuda_check(ctx, (int)cudaMemcpyAsync(S->d_inst, inst.data(), inst.size() * sizeof(DeviceInstance),
                                                          cudaMemcpyHostToDevice, st),
                                "scene refit: instances");
    }
    if (rc == LUX_OK && lights)
        rc = lux_cuda_check(ctx, (int)cudaMemcpyAsync(S->d_lights, lights, (size_t)light_count * sizeof(LuxLight),
                                                      cudaMemcpyHostToDevice, st),
                            "scene refit: lights");
    if (rc != LUX_OK) return rc;
    if (n) {
        uint32_t depths = S->depth_start.empty() ? 0u : (uint32_t)S->depth_start.size() - 1u;
        refit_kernel<<<1, 1024, 0, st>>>(sw, S->instance_base, S->d_refit_order, S->d_depth_start, depths,
                                         (Bvh4Node *)S->d_nodes, S->d_slot_source, S->slot_count);
        rc = lux_cuda_check(ctx, (int)cudaGetLastError(), "scene refit: launch");
        if (rc != LUX_OK) return rc;
    }
    // The pageable copies above may return before the transfer completes;
    // keep the staging vectors alive until the stream has consumed them.
    rc = lux_cuda_check(ctx, (int)cudaStreamSynchronize(st), "scene refit");
    if (rc != LUX_OK) return rc;
    S->instance_words.swap(words);
    S->instances.swap(inst);
    return LUX_OK;
}

extern "C" lux_status lux_scene_read_words(const LuxScene *S, uint32_t *out, size_t word_count) {
    if (!S || !out) return LUX_ERR_INVALID_ARGUMENT;
    LuxContext *ctx = S->ctx;
    if (word_count != S->view.scene_word_count)
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "scene words: count differs from the upload");
    cudaSetDevice(ctx->device);
    lux_status rc = lux_cuda_check(ctx, (int)cudaMemcpyAsync(out, S->d_sw, word_count * 16, cudaMemcpyDeviceToHost,
                                                             ctx->stream),
                                   "scene words: copy");
    if (rc != LUX_OK) return rc;
    return lux_cuda_check(ctx, (int)cudaStreamSynchronize(ctx->stream), "scene words: synchronize");
}

lux_status lux_launch_trace_rays(LuxContext *ctx, const LuxScene *scene, const LuxRay *rays, uint32_t count,
                                 uint32_t any_hit, LuxHit *hits, unsigned long long *counters) {
    if (count == 0) return LUX_OK;
    uint32_t block = 128;
    uint32_t grid = (count + block - 1) / block;
    trace_rays_kernel<<<grid, block, 0, ctx->stream>>>(scene->view, rays, count, any_hit, hits, counters);
    return lux_cuda_check(ctx, (int)cudaGetLastError(), "trace_rays_kernel launch");
}

extern "C" lux_status lux_trace_rays(LuxContext *ctx, const LuxScene *scene, const LuxRay *rays, uint32_t count,
                                     uint32_t any_hit, LuxHit *hits) {
    if (!ctx || !scene || (count && (!rays || !hits))) return LUX_ERR_INVALID_ARGUMENT;
    return lux_launch_trace_rays(ctx, scene, rays, count, any_hit, hits, nullptr);
}
