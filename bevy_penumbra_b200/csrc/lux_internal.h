// lux_internal.h - host-side structures shared by the library's sources.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/lux.h"

#include <cuda_runtime.h>

// Device BVH4 node: child boxes in structure-of-arrays order so one warp lane
// reads the node with eight 128-bit loads.  child[i]:
//   kEmpty                   empty slot
//   bit 31 clear             inner node index
//   bit 31 set               leaf: bits 0..26 first element, bits 27..30 count-1
struct alignas(16) Bvh4Node {
    float lo_x[4], hi_x[4];
    float lo_y[4], hi_y[4];
    float lo_z[4], hi_z[4];
    uint32_t child[4];
    uint32_t pad[4];
};
static_assert(sizeof(Bvh4Node) == 128, "BVH4 node must be one 128-byte line");

constexpr uint32_t kLeafBit = 0x80000000u;
constexpr uint32_t kLeafFirstMask = (1u << 27) - 1u;
constexpr uint32_t kLeafMaxCount = 16u;

// Device instance record (64 bytes): local_from_world rows, BLAS root node,
// triangle range and flags (pack_instances rows 0-2 and word 8, word 6.w).
struct alignas(16) DeviceInstance {
    float row[3][4];
    uint32_t root;
    uint32_t first;
    uint32_t count;
    uint32_t flags;
};

// Scene data as the kernels see it (all device pointers).
struct SceneView {
    const Bvh4Node *nodes;
    const float4 *triangles;        // 3 float4 per triangle (local positions)
    const DeviceInstance *instances;
    const uint4 *scene_words;       // verbatim reference words (materials, transforms)
    const uint4 *geometry_words;    // verbatim reference words (indices, vertices)
    const LuxLight *lights;
    uint32_t tlas_root;             // BVH4 node index of the TLAS root
    uint32_t instance_count;
    uint32_t triangle_count;
    uint32_t scene_word_count;
    uint32_t geometry_word_count;
    uint32_t conventional_lights;
    uint32_t emissive_lights;
    float root_lo[3], root_hi[3];   // TLAS root box at upload (quantises coherence sort keys only)
};

// Wavefront trace scratch (the reference's deferred-trace slots and query
// list, shaders/common.slang:501-533): [rays] and [rays * 16] records.
struct TraceScratch {
    float4 *ray_o;          // origin, hit t
    float4 *ray_d;          // direction, barycentric 1
    uint4 *ray_h;           // triangle, instance, errors, barycentric 2 bits
    float4 *ray_base;       // hit emission, next-event count (kEmpty: unsupported)
    float4 *ray_extra;      // multi-bounce term of the hit (written when the frame has feedback)
    uint32_t *query_slot;   // compact query list: the (ray, sample) slot of query i
    float4 *slot_contrib;   // per (ray, sample): contribution if visible
    float4 *queue_o;        // per (ray, sample): query origin, limit
    float4 *queue_d;        // per (ray, sample): query direction, coherence sort key bits
    uint8_t *queue_result;  // per (ray, sample): 0 visible, 1 blocked, 2 unsupported
    uint32_t *queue_count;
    uint32_t *work_counter; // [2] persistent-warp ray fetch: closest, shadow
};

struct LuxContext {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool owns_stream = false;
    std::string last_error;
    int sm_count = 148;
    // Trace scratch of lux_interval_radiance, grown on demand.
    void *scratch_mem = nullptr;
    uint32_t scratch_rays = 0;
};

// Carves trace scratch for `rays` rays, plus an error word and 16 statistics
// counters, out of one 256-byte-aligned block of trace_scratch_bytes(rays) +
// 256 bytes.  Returns the end of the carved range.
inline unsigned char *carve_trace_scratch(unsigned char *base, uint32_t rays, TraceScratch &t, uint32_t *&error_flags,
                                          unsigned long long *&stats) {
    auto take = [&](size_t bytes) {
        unsigned char *p = base;
        base += (bytes + 255) & ~(size_t)255;
        return p;
    };
    size_t r = rays, q = (size_t)rays * 16u;
    t.ray_o = (float4 *)take(r * 16);
    t.ray_d = (float4 *)take(r * 16);
    t.ray_h = (uint4 *)take(r * 16);
    t.ray_base = (float4 *)take(r * 16);
    t.query_slot = (uint32_t *)take(q * 4);
    t.slot_contrib = (float4 *)take(q * 16);
    t.queue_o = (float4 *)take(q * 16);
    t.queue_d = (float4 *)take(q * 16);
    t.queue_result = (uint8_t *)take(q);
    t.queue_count = (uint32_t *)take(16);
    t.work_counter = (uint32_t *)take(16);
    error_flags = (uint32_t *)take(16);
    stats = (unsigned long long *)take(16 * 8);
    return base;
}

// Bytes carve_trace_scratch consumes for `rays` rays.
inline size_t carved_scratch_bytes(uint32_t rays) {
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t r = rays, q = (size_t)rays * 16u;
    return 4 * up(r * 16) + up(q * 4) + 3 * up(q * 16) + up(q) + 3 * up(16) + up(128);
}

struct LuxScene {
    LuxContext *ctx = nullptr;
    SceneView view{};
    void *d_nodes = nullptr, *d_tris = nullptr, *d_inst = nullptr, *d_sw = nullptr, *d_gw = nullptr,
         *d_lights = nullptr;
    uint32_t node_count = 0;
    // Refit state (lux_scene_refit): host copies of the instance records and
    // device instances, the TLAS binary nodes by depth, and where every TLAS
    // BVH4 child slot takes its box from.
    uint32_t instance_base = 0;                 // first instance word
    std::vector<uint32_t> instance_words;       // inst_count * 9 uint4 words
    std::vector<DeviceInstance> instances;
    std::vector<uint32_t> depth_start;          // refit order offsets, one per depth + 1
    uint32_t slot_count = 0;                    // TLAS BVH4 nodes * 4
    uint32_t *d_refit_order = nullptr;          // binary TLAS nodes, deepest depth first
    uint32_t *d_depth_start = nullptr;
    uint2 *d_slot_source = nullptr;             // (binary node, instance or kEmpty) per slot
    uint32_t light_count = 0;
};

// local_from_world of a 3x4 world_from_local (row-major), inverted in f64
// and rounded to f32; false when the linear part is singular or not finite.
// Shared by the packer and lux_scene_refit so a refit to a pose writes the
// same instance rows as packing the scene at that pose.
bool lux_affine_inverse(const float world_from_local[12], float local_from_world[12]);

// Cache query over a compacted list whose length is on the device
// (count <= max_count); ordered on the cache's context stream.
LuxContext *lux_cache_context(const LuxCache *cache);
lux_status lux_cache_query_device_count(LuxCache *cache, const LuxCacheSample *queries, const uint32_t *count,
                                        uint32_t max_count, float *out);

lux_status lux_fail(LuxContext *ctx, lux_status status, const std::string &message);
lux_status lux_cuda_check(LuxContext *ctx, int err, const char *what);
