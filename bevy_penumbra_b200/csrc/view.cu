// view.cu - one cascade frame of a view: the Split dispatch sequence of
// render() (src/render.rs:9553-9801) as CUDA kernels.
//
//   seed      world cells of every level that hold a receiver, in per-level
//             open-addressing directories (seed/rank/insertProbeDescriptor,
//             shaders/split.slang:292-319, :734-893) with dense cell ids
//   trace     closest hit + hit shading + deposit in one kernel
//             (traceTransport/finishTransportVariant/deposit,
//             shaders/split.slang:1056-1216); the per-key mean of reduce
//             (shaders/split.slang:1386-1476) is a sum + count per record
//   merge     levels L-1..0 (mergeEntry, shaders/split.slang:1624-1725)
//   pack      cascade-0 cells to 6x6 octahedral tables (packProbes,
//             shaders/split.slang:1786-1918)
//   resolve   worldResolve (shaders/world_resolve.slang:281-313)
//
// Records live in dense per-level arrays indexed [cell][direction] instead of
// the reference's hashed bucket chains; keys (cell, direction, level) are the
// reference's world-grid keys (cacheKey, shaders/common.slang:417-422).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_segmented_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "lux_internal.h"
#include "lux_math.cuh"
#include "shade.cuh"
#include "traverse.cuh"

// Resident 128-thread blocks per SM the trace kernels are compiled for: the
// register cap that trades walker state kept in registers against warps in
// flight (6 blocks = 80 registers per thread, 7 = 72).  The visibility walk
// keeps no child order, so it fits 7.
#ifndef LUX_CLOSEST_MIN_BLOCKS
#define LUX_CLOSEST_MIN_BLOCKS 6
#endif
#ifndef LUX_SHADOW_MIN_BLOCKS
#define LUX_SHADOW_MIN_BLOCKS 7
#endif
// The batched trace kernels keep a job's scene pointers per warp as well.
#ifndef LUX_BATCH_MIN_BLOCKS
#define LUX_BATCH_MIN_BLOCKS 6
#endif
// Merge launch shape: threads per block and the resident blocks the
// register budget is sized for.
#ifndef LUX_MERGE_THREADS
#define LUX_MERGE_THREADS 256
#endif
#ifndef LUX_MERGE_MIN_BLOCKS
#define LUX_MERGE_MIN_BLOCKS 4
#endif
// The own pass (every record of every level, no children): 256-thread
// blocks, register budget for this many resident per SM (6: 40 registers;
// at 8 the 32-register budget spills and the pass ran 5% longer).
#ifndef LUX_MERGE_OWN_MIN_BLOCKS
#define LUX_MERGE_OWN_MIN_BLOCKS 6
#endif
// The merge's own pass lists the records that pass light on, and the
// children pass of each level runs over that list only (full warps) instead
// of over every record of the level.
#ifndef LUX_MERGE_COMPACT
#define LUX_MERGE_COMPACT 1
#endif

// The merge preparation takes one thread per (cell, corner) instead of one
// per cell.
#ifndef LUX_MERGE_PREP_SPLIT
#define LUX_MERGE_PREP_SPLIT 1
#endif

#ifndef LUX_MERGE_CORNER_OUTER
#define LUX_MERGE_CORNER_OUTER 1
#endif
// The refill schedulers' register budget (resident 128-thread blocks per SM):
// 5 blocks (92 registers) measured faster than 96 registers or 80.
#ifndef LUX_REFILL_MIN_BLOCKS
#define LUX_REFILL_MIN_BLOCKS 5
#endif
// Hit shading's register budget (resident 128-thread blocks per SM): 80
// registers with a few spills measured faster than 112 without.
#ifndef LUX_SHADE_MIN_BLOCKS
#define LUX_SHADE_MIN_BLOCKS 6
#endif
// Whole-warp traversal in the persistent trace kernels: the BLAS leaves the
// lanes reach in a step are tested by the whole warp.
#ifndef LUX_WARP_LEAVES
#define LUX_WARP_LEAVES 1
#endif
// The fused batch trace kernel carries the shading phase's registers too.
#ifndef LUX_FUSED_MIN_BLOCKS
#define LUX_FUSED_MIN_BLOCKS 4
#endif

namespace {

using lux::f3;

constexpr int kMaxDirty = 8;  // invalidation boxes per frame (more are merged into their union)
constexpr uint32_t kRetainBins = 256;  // age classes of retained cells (older cells share the last)

// The previous frame's records: its cell directories, record offsets, and
// blended raw records with their masses (swapped with the current frame's
// buffers at the start of each frame).
struct HistoryDevice {
    const unsigned long long *dir_keys;
    const uint32_t *dir_ids;
    const unsigned long long *level_base;
    const uint32_t *cell_count;
    const float4 *raw;
    const float2 *mass;
    const uint32_t *cell_last;  // [levels][cell_capacity] frame of each cell's last receiver
    const int4 *cell_keys;      // [levels][cell_capacity]
};

struct FrameParams {
    uint32_t levels, layout, rays_per_receiver, receivers;
    uint32_t dir_capacity, cell_capacity, ray_capacity, queue_capacity;
    unsigned long long entry_capacity;
    float spacing[LUX_MAX_LEVELS];
    float start[LUX_MAX_LEVELS];
    float end[LUX_MAX_LEVELS];
    uint32_t columns[LUX_MAX_LEVELS];
    uint32_t rows[LUX_MAX_LEVELS];
    uint32_t dirs[LUX_MAX_LEVELS];
    lux::ShadeParams shade;
    // World history (mergeEntry, shaders/split.slang:1624-1725).
    float radiance_blend, transmittance_blend;  // 0 disables that quantity's history
    uint32_t history;                           // 1: the previous frame's records may be reused
    uint32_t dirty_count;                       // boxes whose records do not reuse history
    float dirty_lo[kMaxDirty][3], dirty_hi[kMaxDirty][3];
    // Multi-bounce: the secondary cache's receivers are the primary hits, one
    // slot per primary receiver, and a slot with position.w == 0 holds none.
    uint32_t sparse;       // receivers with position.w == 0 are absent
    uint32_t record_hits;  // write each receiver's hit surface (ray frame % R) to hit_pos / hit_nrm
    // Distance LODs (splitLodBlendForParameters, shaders/common.slang:431-461;
    // lod_enabled = 0: every receiver and resolve point uses LOD 0).
    uint32_t lod_enabled, lod_perspective;
    float lod_camera[3];
    float lod_base;         // perspective: max(focal pixels x spacing / target pixels, spacing)
    float lod_ortho_scale;  // orthographic: target pixels / max(focal pixels x spacing, 1e-20)
};

// Device state of a view (ViewBuffers, src/render.rs:5077-5160).
struct ViewDevice {
    unsigned long long *dir_keys;   // [levels][dir_capacity]
    uint32_t *dir_ids;              // [levels][dir_capacity]
    int4 *cell_keys;                // [levels][cell_capacity]
    uint32_t *cell_count;           // [levels]
    unsigned long long *level_base; // [levels]
    uint32_t *receiver_cell;        // [levels][max_receivers]
    uint32_t *receiver_lod;         // [max_receivers] the LOD each receiver's rays deposit into
    uint32_t *receiver_ordinal;     // [max_receivers] the receiver's place in the sample sequence
    unsigned long long *order_keys; // [2][max_receivers] sequence-order sort keys (in, out)
    uint32_t *order_vals;           // [2][max_receivers] receiver indices (in, out)
    void *order_temp;               // radix-sort scratch
    size_t order_temp_bytes;
    uint32_t *corner_ids;           // [levels][cell_capacity][8] (level+1 ids)
    float4 *corner_frac;            // [levels][cell_capacity]
    float4 *accum;                  // [entries] J sum rgb, non-terminating count
    uint32_t *count;                // [entries]
    float4 *merged;                 // [entries] I rgb, support
    float4 *raw;                    // [entries] J rgb, beta (history-blended)
    float2 *mass;                   // [entries] radiance mass, transmittance mass
    uint32_t *pass_list;            // [entries] per level (at its record base): records that pass light on
    uint32_t *pass_count;           // [levels] entries of pass_list per level
    uint32_t *hist_cell;            // [levels][cell_capacity] the previous frame's id of each cell, or kEmpty
    uint32_t *cell_last;            // [levels][cell_capacity] frame index of the cell's last receiver
    uint32_t *retain_hist;          // [levels][kRetainBins] retain candidates per age class
    uint32_t *retain_limit;         // [levels] age classes below this are retained
    float4 *hit_pos;                // [receivers] multi-bounce: hit position, 1 (0: no surface)
    float4 *hit_nrm;                // [receivers] multi-bounce: geometric normal facing the ray
    float4 *tables;                 // [cell_capacity][36]
    uint32_t *error_flags;
    unsigned long long *stats;      // 8 counters
    TraceScratch ts;                // wavefront trace state
    // Coherence ordering of rays / visibility queries (counting sort by bin).
    uint32_t *sort_keys;            // [max(rays, queries)]
    uint32_t *sort_perm;            // [max(rays, queries)] processing order -> item
    uint32_t *sort_hist;            // [kSortBins]
    uint32_t *sort_offs;            // [kSortBins] exclusive prefix of sort_hist, then scatter cursors
    void *scan_temp;                // device-wide scan scratch
    size_t scan_temp_bytes;
    const uint32_t *ray_order;      // closest-hit processing order (nullptr: identity)
    const uint32_t *query_order;    // visibility processing order (nullptr: identity)
};

// Rays per work-queue fetch of a tuning (0 means 32).
static inline uint32_t tile_of(const LuxTuning &t) { return t.tile_rays ? t.tile_rays : 32u; }

constexpr uint32_t kSortCells = 4096;           // 16^3 origin cells over the TLAS root box
constexpr uint32_t kQueryCells = 2097152;       // 128^3 origin cells of visibility queries
constexpr uint32_t kRaySortBins = 32 * kSortCells;  // 32 direction bins x 16^3 origin cells of interval rays
constexpr uint32_t kSortBins = 8 * kQueryCells; // 8 emitter buckets x 128^3 origin cells of queries,
                                                // or 32 direction bins x 16^3 cells of interval rays

// Morton index of a point's cell in a 128^3 grid over the scene box.
__device__ __forceinline__ uint32_t cell128(const SceneView &S, lux::f3 p) {
    float e[3] = {p.x, p.y, p.z};
    uint32_t c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float span = S.root_hi[a] - S.root_lo[a];
        float t = span > 0.0f ? (e[a] - S.root_lo[a]) / span : 0.0f;
        int q = (int)(t * 128.0f);
        c[a] = (uint32_t)(q < 0 ? 0 : (q > 127 ? 127 : q));
    }
    uint32_t m = 0;
#pragma unroll
    for (int b = 0; b < 7; ++b)
        m |= (((c[0] >> b) & 1u) << (3 * b)) | (((c[1] >> b) & 1u) << (3 * b + 1)) | (((c[2] >> b) & 1u) << (3 * b + 2));
    return m;
}

// Morton index of a point's cell in a 16^3 grid over the scene box.
__device__ __forceinline__ uint32_t cell16(const SceneView &S, lux::f3 p) {
    float e[3] = {p.x, p.y, p.z};
    uint32_t c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float span = S.root_hi[a] - S.root_lo[a];
        float t = span > 0.0f ? (e[a] - S.root_lo[a]) / span : 0.0f;
        int q = (int)(t * 16.0f);
        c[a] = (uint32_t)(q < 0 ? 0 : (q > 15 ? 15 : q));
    }
    uint32_t m = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b)
        m |= (((c[0] >> b) & 1u) << (3 * b)) | (((c[1] >> b) & 1u) << (3 * b + 1)) | (((c[2] >> b) & 1u) << (3 * b + 2));
    return m;
}

constexpr int kStatInterval = 0, kStatShadow = 1, kStatNodes = 2, kStatTris = 3, kStatInst = 4, kStatDeposits = 5,
              kStatUnsupported = 6, kStatShadowNodes = 7, kStatShadowTris = 8, kStatShadowInst = 9;
constexpr int kStats = 10;

__device__ __forceinline__ void add_stats(unsigned long long *stats, unsigned long long v[7],
                                          const unsigned long long *extra = nullptr) {
    unsigned long long w[kStats];
#pragma unroll
    for (int k = 0; k < kStats; ++k) w[k] = k < 7 ? v[k] : (extra ? extra[k - 7] : 0ull);
#pragma unroll
    for (int k = 0; k < kStats; ++k)
        for (int off = 16; off > 0; off >>= 1) w[k] += __shfl_down_sync(0xffffffffu, w[k], off);
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < kStats; ++k)
            if (w[k]) atomicAdd(&stats[k], w[k]);
    }
}

// Spacing of a level at an LOD (spacing, shaders/common.slang:414-416).
__device__ __forceinline__ float level_spacing(const FrameParams &F, uint32_t level, uint32_t lod) {
    return F.spacing[level] * lux::lod_scale(lod);
}

__device__ __forceinline__ void cell_of(const FrameParams &F, uint32_t level, f3 p, int32_t &x, int32_t &y,
                                        int32_t &z, uint32_t lod = 0u) {
    float s = level_spacing(F, level, lod);
    x = (int32_t)floorf(p.x / s);
    y = (int32_t)floorf(p.y / s);
    z = (int32_t)floorf(p.z / s);
}

// A point's LOD pair and blend (0, 0, 0 without distance LODs).
__device__ __forceinline__ void point_lod(const FrameParams &F, f3 p, uint32_t &low, uint32_t &high, float &blend) {
    low = high = 0u;
    blend = 0.0f;
    if (F.lod_enabled)
        lux::lod_blend(F.lod_perspective != 0u, F.lod_camera[0], F.lod_camera[1], F.lod_camera[2], F.lod_base,
                       F.lod_ortho_scale, p, low, high, blend);
}

// Probe of a level directory; returns the slot or kEmpty.
__device__ __forceinline__ uint32_t dir_find(const ViewDevice &V, const FrameParams &F, uint32_t level, int32_t x,
                                             int32_t y, int32_t z, uint32_t lod = 0u) {
    if (!lux::cell_in_range(x, y, z)) return lux::kEmpty;
    unsigned long long key = lux::pack_cell(x, y, z, lod);
    const unsigned long long *keys = V.dir_keys + (size_t)level * F.dir_capacity;
    uint32_t slot = lux::hash_key(x, y, z, (int32_t)(level | (lod << 18)), F.dir_capacity);
    for (uint32_t attempt = 0; attempt < F.dir_capacity; ++attempt) {
        unsigned long long k = keys[slot];
        if (k == key) return slot;
        if (k == lux::kEmptyCell) return lux::kEmpty;
        slot = (slot + 1u) & (F.dir_capacity - 1u);
    }
    return lux::kEmpty;
}

__device__ __forceinline__ uint32_t cell_id(const ViewDevice &V, const FrameParams &F, uint32_t level, int32_t x,
                                            int32_t y, int32_t z, uint32_t lod = 0u) {
    uint32_t slot = dir_find(V, F, level, x, y, z, lod);
    return slot == lux::kEmpty ? lux::kEmpty : V.dir_ids[(size_t)level * F.dir_capacity + slot];
}

// Item i of a frame's clear: directory slot i, and with the first items
// the per-level counters, statistics, error word and trace counters (the
// directory has at least 64 slots per level).
__device__ __forceinline__ void clear_item(const ViewDevice &V, const FrameParams &F, unsigned long long i) {
    if (i >= (unsigned long long)F.levels * F.dir_capacity) return;
    V.dir_keys[i] = lux::kEmptyCell;
    V.dir_ids[i] = lux::kEmpty;
    if (i < LUX_MAX_LEVELS) {
        V.cell_count[i] = 0;
        V.level_base[i] = 0;
    }
    if (i < 16) V.stats[i] = 0;
    if (i == 0) {
        *V.error_flags = 0;
        *V.ts.queue_count = 0;
        V.ts.work_counter[0] = 0;
        V.ts.work_counter[1] = 0;
    }
}

__global__ void clear_kernel(ViewDevice V, FrameParams F) {
    size_t n = (size_t)F.levels * F.dir_capacity;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        clear_item(V, F, i);
}

// seed: insert every receiver's cell of every level (insertProbeDescriptor,
// shaders/split.slang:292-319, with a 64-bit key compare-and-swap); in an
// LOD overlap both LOD variants' cells are seeded (seed,
// shaders/split.slang:758-786).
__device__ __forceinline__ void seed_cell(const ViewDevice &V, const FrameParams &F, uint32_t level, f3 p, uint32_t lod) {
    int32_t x, y, z;
    cell_of(F, level, p, x, y, z, lod);
    if (!lux::cell_in_range(x, y, z)) {
        atomicOr(V.error_flags, LUX_VIEW_ERR_CELL_CAPACITY);
        return;
    }
    unsigned long long key = lux::pack_cell(x, y, z, lod);
    unsigned long long *keys = V.dir_keys + (size_t)level * F.dir_capacity;
    uint32_t slot = lux::hash_key(x, y, z, (int32_t)(level | (lod << 18)), F.dir_capacity);
    for (uint32_t attempt = 0; attempt < F.dir_capacity; ++attempt) {
        unsigned long long prev = atomicCAS(&keys[slot], lux::kEmptyCell, key);
        if (prev == lux::kEmptyCell || prev == key) return;
        slot = (slot + 1u) & (F.dir_capacity - 1u);
    }
    atomicOr(V.error_flags, LUX_VIEW_ERR_CELL_CAPACITY);
}

// Item i = receiver x levels + level.
__device__ __forceinline__ void seed_insert_item(const ViewDevice &V, const FrameParams &F, const float4 *__restrict__ pos,
                                                 unsigned long long i) {
    if (i >= (unsigned long long)F.receivers * F.levels) return;
    uint32_t r = (uint32_t)(i / F.levels), level = (uint32_t)(i % F.levels);
    float4 p = pos[r];
    if (F.sparse && p.w == 0.0f) return;
    const f3 q{p.x, p.y, p.z};
    uint32_t low, high;
    float blend;
    point_lod(F, q, low, high, blend);
    seed_cell(V, F, level, q, low);
    if (high != low) seed_cell(V, F, level, q, high);
}

__global__ void seed_insert_kernel(ViewDevice V, FrameParams F, const float4 *__restrict__ pos) {
    size_t n = (size_t)F.receivers * F.levels;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        seed_insert_item(V, F, pos, i);
}

// rank: dense ids for occupied directory slots.
__device__ __forceinline__ void seed_assign_item(const ViewDevice &V, const FrameParams &F, unsigned long long i) {
    if (i >= (unsigned long long)F.levels * F.dir_capacity) return;
    unsigned long long key = V.dir_keys[i];
    if (key == lux::kEmptyCell) return;
    uint32_t level = (uint32_t)(i / F.dir_capacity);
    uint32_t id = atomicAdd(&V.cell_count[level], 1u);
    if (id >= F.cell_capacity) {
        atomicOr(V.error_flags, LUX_VIEW_ERR_CELL_CAPACITY);
        V.dir_ids[i] = lux::kEmpty;
        return;
    }
    V.dir_ids[i] = id;
    int32_t x, y, z;
    uint32_t lod;
    lux::unpack_cell(key, x, y, z, lod);
    V.cell_keys[(size_t)level * F.cell_capacity + id] = make_int4(x, y, z, (int32_t)((level << 12) | (lod << 18)));
    V.cell_last[(size_t)level * F.cell_capacity + id] = F.shade.frame;
}

__global__ void seed_assign_kernel(ViewDevice V, FrameParams F) {
    size_t n = (size_t)F.levels * F.dir_capacity;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        seed_assign_item(V, F, i);
}

// Sample sequence order (the reference's rank / parents / prefix passes,
// shaders/split.slang:788-963): the receivers of one cascade-0 cell take
// consecutive places and sibling cells of every coarser level adjacent runs,
// so each probe's rays are consecutive points of the R2 sequence.  The order
// is the LOD, then the Morton order of the cascade-0 cell (at every level
// the octant ordinal x + 2y + 4z, as `prefix` orders siblings), then the
// receiver index; the reference takes atomic arrival order where the index
// and the Morton order of the roots decide here.  Absent receivers sort last.
__device__ __forceinline__ unsigned long long sequence_key(int32_t x, int32_t y, int32_t z, uint32_t lod) {
    const uint32_t bx = (uint32_t)x + (1u << 18), by = (uint32_t)y + (1u << 18), bz = (uint32_t)z + (1u << 18);
    unsigned long long m = 0;
#pragma unroll
    for (int b = 0; b < 19; ++b)
        m |= ((unsigned long long)((bx >> b) & 1u) << (3 * b)) | ((unsigned long long)((by >> b) & 1u) << (3 * b + 1)) |
             ((unsigned long long)((bz >> b) & 1u) << (3 * b + 2));
    return ((unsigned long long)(lod & 31u) << 57) | m;
}

// sorted: the receiver indices in sequence order (the sort's output half).
__global__ void ordinal_kernel(ViewDevice V, const uint32_t *__restrict__ sorted, uint32_t receivers) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < receivers; j += gridDim.x * blockDim.x)
        V.receiver_ordinal[sorted[j]] = j;
}

// Item i = receiver x levels + level; the receiver's sequence key and index
// go to keys[r], vals[r].
__device__ __forceinline__ void seed_lookup_item(const ViewDevice &V, const FrameParams &F,
                                                 const float4 *__restrict__ pos, unsigned long long i,
                                                 unsigned long long *keys, uint32_t *vals) {
    if (i >= (unsigned long long)F.receivers * F.levels) return;
    uint32_t r = (uint32_t)(i / F.levels), level = (uint32_t)(i % F.levels);
    float4 p = pos[r];
    const f3 q{p.x, p.y, p.z};
    // The variant this receiver's rays deposit into (one trace per
    // receiver; in an LOD overlap the high LOD with probability blend).
    uint32_t low, high;
    float blend;
    point_lod(F, q, low, high, blend);
    uint32_t lod = high != low && lux::lod_selects_high(r, F.shade.frame, blend) ? high : low;
    if (level == 0u) V.receiver_lod[r] = lod;
    int32_t x, y, z;
    cell_of(F, level, q, x, y, z, lod);
    if (level == 0u) {
        keys[r] = F.sparse && p.w == 0.0f ? ~0ull : sequence_key(x, y, z, lod);
        vals[r] = r;
    }
    V.receiver_cell[(size_t)level * F.receivers + r] =
        F.sparse && p.w == 0.0f ? lux::kEmpty : cell_id(V, F, level, x, y, z, lod);
}

__global__ void seed_lookup_kernel(ViewDevice V, FrameParams F, const float4 *__restrict__ pos) {
    size_t n = (size_t)F.receivers * F.levels;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        seed_lookup_item(V, F, pos, i, V.order_keys, V.order_vals);
}

// Per-level record offsets; the entry capacity bounds the whole frame.
__device__ __forceinline__ void layout_view(const ViewDevice &V, const FrameParams &F) {
    unsigned long long base = 0;
    for (uint32_t l = 0; l < F.levels; ++l) {
        uint32_t cells = min(V.cell_count[l], F.cell_capacity);
        V.cell_count[l] = cells;
        V.level_base[l] = base;
        base += (unsigned long long)cells * F.dirs[l];
    }
    if (base > F.entry_capacity) atomicOr(V.error_flags, LUX_VIEW_ERR_ENTRY_CAPACITY);
    if (F.layout == LUX_LAYOUT_DENSE && base > F.ray_capacity) atomicOr(V.error_flags, LUX_VIEW_ERR_RAY_CAPACITY);
}

__global__ void layout_kernel(ViewDevice V, FrameParams F) {
    if (threadIdx.x == 0 && blockIdx.x == 0) layout_view(V, F);
}

__device__ __forceinline__ unsigned long long total_entries(const ViewDevice &V, const FrameParams &F) {
    unsigned long long base = 0;
    for (uint32_t l = 0; l < F.levels; ++l) base += (unsigned long long)V.cell_count[l] * F.dirs[l];
    return base;
}

__device__ __forceinline__ void clear_entry(const ViewDevice &V, unsigned long long i) {
    V.accum[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    V.count[i] = 0u;
}

__global__ void clear_entries_kernel(ViewDevice V, FrameParams F) {
    if (*V.error_flags) return;
    unsigned long long n = total_entries(V, F);
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x)
        clear_entry(V, i);
}

// ---------------------------------------------------------------------------
// Trace stage as a wavefront (the reference's deferred trace: traceDeferred,
// traceRecord, traceVisibility, traceResolve, shaders/split.slang:1276-1384):
//   closest   interval rays -> closest hits (lean traversal kernel)
//   shade     hit shading; next-event queries appended to one queue
//   shadow    every queued visibility query in its own lane (any hit)
//   deposit   next-event sum in sample order, then deposit into the levels
// ---------------------------------------------------------------------------

// Split ray of receiver i, ray k: direction decodeDirection(frac(0.5 +
// r2(sequence + 1) + jitter)) flipped into the normal's hemisphere
// (traceTransport, shaders/split.slang:1135-1146); (u, v) of the flipped
// direction give its bin at every level.
__device__ __forceinline__ void split_direction(const ViewDevice &V, const FrameParams &F, uint32_t frame, uint32_t i,
                                                uint32_t k, f3 n, f3 &dir, float &u, float &v) {
    float jx, jy, rx, ry;
    lux::r2(lux::transport_hash(frame ^ 0x5a17c9e3u), jx, jy);
    lux::r2(V.receiver_ordinal[i] * F.rays_per_receiver + k + 1u, rx, ry);
    u = lux::fracf((0.5f + rx) + jx);
    v = lux::fracf((0.5f + ry) + jy);
    dir = lux::decode_direction(u, v);
    if (lux::dot(dir, n) < 0.0f) {
        dir = -dir;
        u = lux::fracf(u + 0.5f);
        v = 1.0f - v;
    }
}

__device__ __forceinline__ void store_ray(const ViewDevice &V, uint32_t ray, f3 o, f3 d, const lux::Hit &h) {
    V.ts.ray_o[ray] = make_float4(o.x, o.y, o.z, h.t);
    V.ts.ray_d[ray] = make_float4(d.x, d.y, d.z, h.b1);
    V.ts.ray_h[ray] = make_uint4(h.tri, h.inst, h.errors, lux::as_uint(h.b2));
}

__device__ __forceinline__ void load_ray(const ViewDevice &V, uint32_t ray, f3 &o, f3 &d, lux::Hit &h) {
    float4 a = V.ts.ray_o[ray], b = V.ts.ray_d[ray];
    uint4 c = V.ts.ray_h[ray];
    o = f3{a.x, a.y, a.z};
    d = f3{b.x, b.y, b.z};
    h.t = a.w;
    h.b1 = b.w;
    h.tri = c.x;
    h.inst = c.y;
    h.errors = c.z;
    h.b2 = lux::as_float(c.w);
}

// Persistent warps with per-lane refill (lux::trace_persistent).
__global__ void __launch_bounds__(128, LUX_REFILL_MIN_BLOCKS) closest_split_refill_kernel(ViewDevice V, FrameParams F, SceneView S,
                                                            const float4 *__restrict__ pos,
                                                            const float4 *__restrict__ nrm, uint32_t ray_count) {
    if (*V.error_flags) return;
#if LUX_WARP_LEAVES
    __shared__ lux::LeafScratch scratch[4];
    lux::LeafScratch *L = &scratch[threadIdx.x >> 5];
#else
    lux::LeafScratch *L = nullptr;
#endif
    unsigned long long st[7] = {0, 0, 0, 0, 0, 0, 0};
    lux::TraceCounters cn{0, 0, 0};
    lux::trace_persistent<false>(
        S, &V.ts.work_counter[0], ray_count,
        [&](uint32_t slot, f3 &o, f3 &d, float &tmin, float &limit) {
            uint32_t ray = V.ray_order ? V.ray_order[slot] : slot;
            uint32_t i = ray / F.rays_per_receiver, k = ray % F.rays_per_receiver;
            float4 p4 = pos[i], n4 = nrm[i];
            f3 p{p4.x, p4.y, p4.z}, n{n4.x, n4.y, n4.z};
            float u, v;
            split_direction(V, F, F.shade.frame, i, k, n, d, u, v);
            o = lux::ray_offset(p, n, F.shade.normal_bias);
            tmin = 0.0f;
            limit = 1e20f;
            V.ts.ray_o[ray] = make_float4(o.x, o.y, o.z, 0.0f);
            V.ts.ray_d[ray] = make_float4(d.x, d.y, d.z, 0.0f);
        },
        [&](uint32_t slot, const lux::Hit &h) {
            uint32_t ray = V.ray_order ? V.ray_order[slot] : slot;
            V.ts.ray_o[ray].w = h.t;
            V.ts.ray_d[ray].w = h.b1;
            V.ts.ray_h[ray] = make_uint4(h.tri, h.inst, h.errors, lux::as_uint(h.b2));
            st[kStatInterval] += 1;
        },
        cn, L);
    st[kStatNodes] = cn.nodes;
    st[kStatTris] = cn.triangles;
    st[kStatInst] = cn.instances;
    add_stats(V.stats, st);
}

// One Split interval ray (traceTransport, shaders/split.slang:1122-1163):
// receiver i = ray / R, sample k = ray % R, from the biased receiver position
// to 1e20; the hit is stored for shading.
// Returns false for the rays of an absent receiver of a sparse set (stored
// as unsupported, not traced).
template <int kDepth = lux::kStack>
__device__ __forceinline__ bool closest_split_ray(const ViewDevice &V, const FrameParams &F, uint32_t frame,
                                                  const SceneView &S, const float4 *__restrict__ pos,
                                                  const float4 *__restrict__ nrm, uint32_t slot,
                                                  lux::TraceCounters &cn) {
    uint32_t ray = V.ray_order ? V.ray_order[slot] : slot;
    uint32_t i = ray / F.rays_per_receiver, k = ray % F.rays_per_receiver;
    float4 p4 = pos[i], n4 = nrm[i];
    if (F.sparse && p4.w == 0.0f) {
        lux::Hit none;
        none.t = 0.0f;
        none.b1 = none.b2 = 0.0f;
        none.tri = none.inst = lux::kEmpty;
        none.errors = lux::kQueryUnsupported;
        store_ray(V, ray, f3{0.0f, 0.0f, 0.0f}, f3{0.0f, 0.0f, 0.0f}, none);
        return false;
    }
    f3 p{p4.x, p4.y, p4.z}, n{n4.x, n4.y, n4.z};
    f3 dir;
    float u, v;
    split_direction(V, F, frame, i, k, n, dir, u, v);
    f3 origin = lux::ray_offset(p, n, F.shade.normal_bias);
    lux::Hit hit;
    lux::trace<false, kDepth>(S, origin, dir, 0.0f, 1e20f, hit, cn);
    store_ray(V, ray, origin, dir, hit);
    return true;
}

// closest_split_ray for a whole warp (every lane calls it; `valid`: the
// lane has a slot), with the warp's leaves tested together.
template <int kDepth = lux::kStack>
__device__ __forceinline__ bool closest_split_ray_warp(const ViewDevice &V, const FrameParams &F, uint32_t frame,
                                                       const SceneView &S, const float4 *__restrict__ pos,
                                                       const float4 *__restrict__ nrm, uint32_t slot, bool valid,
                                                       lux::TraceCounters &cn, lux::LeafScratch *L) {
    bool active = valid;
    uint32_t ray = 0;
    f3 origin{0.0f, 0.0f, 0.0f}, dir{0.0f, 0.0f, 0.0f};
    if (valid) {
        ray = V.ray_order ? V.ray_order[slot] : slot;
        uint32_t i = ray / F.rays_per_receiver, k = ray % F.rays_per_receiver;
        float4 p4 = pos[i], n4 = nrm[i];
        if (F.sparse && p4.w == 0.0f) {
            lux::Hit none;
            none.t = 0.0f;
            none.b1 = none.b2 = 0.0f;
            none.tri = none.inst = lux::kEmpty;
            none.errors = lux::kQueryUnsupported;
            store_ray(V, ray, f3{0.0f, 0.0f, 0.0f}, f3{0.0f, 0.0f, 0.0f}, none);
            active = false;
        } else {
            f3 p{p4.x, p4.y, p4.z}, n{n4.x, n4.y, n4.z};
            float u, v;
            split_direction(V, F, frame, i, k, n, dir, u, v);
            origin = lux::ray_offset(p, n, F.shade.normal_bias);
        }
    }
    lux::Hit hit;
    lux::trace_warp<false, kDepth>(S, active, origin, dir, 0.0f, 1e20f, hit, cn, L);
    if (active) store_ray(V, ray, origin, dir, hit);
    return active;
}

// Persistent warps: a tile of `tile` consecutive rays per fetch (one atomic
// per warp), taken 32 at a time.
__device__ __forceinline__ uint32_t warp_fetch(uint32_t *counter, uint32_t tile = 32u) {
    uint32_t base = 0;
    if ((threadIdx.x & 31u) == 0u) base = atomicAdd(counter, tile);
    return __shfl_sync(0xffffffffu, base, 0);
}

template <int kDepth>
__global__ void __launch_bounds__(128, LUX_CLOSEST_MIN_BLOCKS) closest_split_kernel(ViewDevice V, FrameParams F, SceneView S,
                                                            const float4 *__restrict__ pos,
                                                            const float4 *__restrict__ nrm, uint32_t ray_count,
                                                            uint32_t tile) {
    if (*V.error_flags) return;
#if LUX_WARP_LEAVES
    __shared__ lux::LeafScratch scratch[4];
    lux::LeafScratch *L = &scratch[threadIdx.x >> 5];
#endif
    unsigned long long st[7] = {0, 0, 0, 0, 0, 0, 0};
    lux::TraceCounters cn{0, 0, 0};
    while (true) {
        uint32_t base = warp_fetch(&V.ts.work_counter[0], tile);
        if (base >= ray_count) break;
        for (uint32_t k = 0; k < tile && base + k < ray_count; k += 32u) {
            uint32_t slot = base + k + (threadIdx.x & 31u);
#if LUX_WARP_LEAVES
            if (closest_split_ray_warp<kDepth>(V, F, F.shade.frame, S, pos, nrm, slot, slot < ray_count, cn, L))
                st[kStatInterval] += 1;
#else
            if (slot < ray_count && closest_split_ray<kDepth>(V, F, F.shade.frame, S, pos, nrm, slot, cn))
                st[kStatInterval] += 1;
#endif
        }
    }
    st[kStatNodes] = cn.nodes;
    st[kStatTris] = cn.triangles;
    st[kStatInst] = cn.instances;
    add_stats(V.stats, st);
}

// Dense layout: one ray per (cell, direction) record of one level; the ray
// starts at the cell centre and covers the level's interval (the dense
// reference of src/transport_tests.rs:179-248 with BVH geometry).  The ray
// index is the record index.
__global__ void __launch_bounds__(128, LUX_CLOSEST_MIN_BLOCKS) closest_dense_kernel(ViewDevice V, FrameParams F, SceneView S, uint32_t level) {
    if (*V.error_flags) return;
    unsigned long long n = (unsigned long long)V.cell_count[level] * F.dirs[level];
    unsigned long long base = V.level_base[level];
    const bool terminal = level + 1u == F.levels;
    const float tmin = F.start[level];
    const float limit = terminal ? 1e20f : nextafterf(F.end[level], INFINITY);
    const float sp = F.spacing[level];
    const uint32_t dirs = F.dirs[level];
    for (unsigned long long e = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
         e < ((n + 31ull) & ~31ull); e += (unsigned long long)gridDim.x * blockDim.x) {
        unsigned long long st[7] = {0, 0, 0, 0, 0, 0, 0};
        if (e < n) {
            uint32_t cell = (uint32_t)(e / dirs), d = (uint32_t)(e % dirs);
            int4 key = V.cell_keys[(size_t)level * F.cell_capacity + cell];
            f3 origin{((float)key.x + 0.5f) * sp, ((float)key.y + 0.5f) * sp, ((float)key.z + 0.5f) * sp};
            f3 dir = lux::bin_direction(d, F.columns[level], F.rows[level]);
            lux::TraceCounters cn{0, 0, 0};
            lux::Hit hit;
            lux::trace<false>(S, origin, dir, tmin, limit, hit, cn);
            store_ray(V, (uint32_t)(base + e), origin, dir, hit);
            st[kStatInterval] = 1;
            st[kStatNodes] = cn.nodes;
            st[kStatTris] = cn.triangles;
            st[kStatInst] = cn.instances;
        }
        add_stats(V.stats, st);
    }
}

// Coherence keys of split interval rays: (direction bin of an 8 x 4 grid,
// origin cell).
__global__ void ray_keys_kernel(ViewDevice V, FrameParams F, SceneView S, const float4 *__restrict__ pos,
                                const float4 *__restrict__ nrm, uint32_t ray_count) {
    for (uint32_t ray = blockIdx.x * blockDim.x + threadIdx.x; ray < ray_count; ray += gridDim.x * blockDim.x) {
        uint32_t i = ray / F.rays_per_receiver, k = ray % F.rays_per_receiver;
        float4 p4 = pos[i], n4 = nrm[i];
        f3 dir;
        float u, v;
        split_direction(V, F, F.shade.frame, i, k, f3{n4.x, n4.y, n4.z}, dir, u, v);
        uint32_t bin = lux::direction_index_uv(u, v, 8u, 4u);
        V.sort_keys[ray] = bin * kSortCells + cell16(S, f3{p4.x, p4.y, p4.z});
    }
}

// Counting sort of keys in [0, kSortBins): histogram, exclusive scan, scatter.
// Order within a bin is arbitrary; every item is processed exactly once and
// its result is written to its own slot, so the outputs do not depend on it.
__global__ void sort_hist_kernel(ViewDevice V, const uint32_t *count_ptr, uint32_t cap) {
    uint32_t n = count_ptr ? min(*count_ptr, cap) : cap;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicAdd(&V.sort_hist[V.sort_keys[i]], 1u);
}

__global__ void sort_scatter_kernel(ViewDevice V, const uint32_t *count_ptr, uint32_t cap) {
    uint32_t n = count_ptr ? min(*count_ptr, cap) : cap;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        V.sort_perm[atomicAdd(&V.sort_offs[V.sort_keys[i]], 1u)] = i;
}

// Exclusive prefix of the first `bins` counting-sort bins over the whole
// device (the interval-ray keys use only the first kRaySortBins).
static void enqueue_sort_scan(const ViewDevice &D, uint32_t bins, cudaStream_t st) {
    size_t bytes = D.scan_temp_bytes;
    cub::DeviceScan::ExclusiveSum(D.scan_temp, bytes, D.sort_hist, D.sort_offs, (int)bins, st);
}


// Hit shading up to the visibility traces; queries are appended to the
// queue with one atomic per warp.
// Hit shading of one warp's rays (one ray per lane, `ray` < `rays` active):
// base emission and next-event queries (outgoingTransportRadianceTracked,
// shaders/cascades.slang:196-268); the warp's queries are appended to the
// view's queue with one atomic.  Every lane of the warp belongs to one view.
__device__ __forceinline__ void shade_warp(const ViewDevice &V, const FrameParams &F, const lux::ShadeParams &P,
                                           const SceneView &S, uint32_t ray, uint32_t rays) {
    const uint32_t lane = threadIdx.x & 31u;
    // Queries are written at their slot (ray x 16 + sample) as they are
    // emitted, so nothing is buffered per lane; the warp then appends the
    // slots it used to the compact query list with one atomic.
    uint32_t used = 0, nq = 0, count = 0;
    bool supported = false, sky = false;
    f3 base{0.0f, 0.0f, 0.0f}, extra;
    const size_t slot0 = (size_t)ray * lux::kMaxNeeSamples;
    if (ray < rays) {
        f3 o, d;
        lux::Hit hit;
        lux::SurfaceRecord rec;
        load_ray(V, ray, o, d, hit);
        const bool keys = V.sort_keys != nullptr;
        supported = lux::outgoing_record(S, P, o, d, hit, base, extra, rec, count, sky,
                                         [&](uint32_t sample, const lux::NeeQuery &q) {
                                             if (sample >= lux::kMaxNeeSamples) return;  // host checks the slot count
                                             const size_t slot = slot0 + sample;
                                             // w of the direction: the query's coherence sort key.
                                             uint32_t key = keys ? (q.light & 7u) * kQueryCells + cell128(S, q.origin)
                                                                 : 0u;
                                             V.ts.queue_o[slot] = make_float4(q.origin.x, q.origin.y, q.origin.z, q.limit);
                                             V.ts.queue_d[slot] = make_float4(q.direction.x, q.direction.y,
                                                                              q.direction.z, lux::as_float(key));
                                             V.ts.slot_contrib[slot] = make_float4(q.contribution.x, q.contribution.y,
                                                                                   q.contribution.z, (float)q.group);
                                             used |= 1u << sample;
                                             ++nq;
                                         });
        // w: the emissive estimator's divisor | conventional-light slots << 5
        // | environment samples present << 9 | the used slots << 16.
        const uint32_t packed = count | (S.conventional_lights << 5) | ((sky ? 1u : 0u) << 9) | (used << 16);
        V.ts.ray_base[ray] = make_float4(base.x, base.y, base.z, lux::as_float(supported ? packed : lux::kEmpty));
        if (P.feedback) V.ts.ray_extra[ray] = make_float4(extra.x, extra.y, extra.z, 0.0f);
        // The multi-bounce secondary receiver of receiver i: its ray frame % R.
        if (F.record_hits && rec.valid && ray % F.rays_per_receiver == P.frame % F.rays_per_receiver) {
            uint32_t i = ray / F.rays_per_receiver;
            V.hit_pos[i] = make_float4(rec.position.x, rec.position.y, rec.position.z, 1.0f);
            V.hit_nrm[i] = make_float4(rec.normal.x, rec.normal.y, rec.normal.z, 0.0f);
        }
    }
    // Warp-aggregated append of this warp's used slots.
    uint32_t prefix = nq;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, prefix, off);
        if (lane >= (uint32_t)off) prefix += t;
    }
    uint32_t total = __shfl_sync(0xffffffffu, prefix, 31);
    uint32_t first = 0;
    if (lane == 31 && total) first = atomicAdd(V.ts.queue_count, total);
    first = __shfl_sync(0xffffffffu, first, 31);
    uint32_t qi = first + prefix - nq;
    for (uint32_t m = used; m; m &= m - 1u, ++qi) {
        const size_t slot = slot0 + (uint32_t)(__ffs(m) - 1);
        if (qi < F.queue_capacity) {
            V.ts.query_slot[qi] = (uint32_t)slot;
            if (V.sort_keys) V.sort_keys[qi] = lux::as_uint(V.ts.queue_d[slot].w);
        } else {
            V.ts.queue_result[slot] = 2;  // list overflow: unsupported
        }
    }
}

__global__ void __launch_bounds__(128, LUX_SHADE_MIN_BLOCKS) shade_kernel(ViewDevice V, FrameParams F, SceneView S, uint32_t ray_count,
                                                    bool dense) {
    if (*V.error_flags) return;
    uint32_t rays = dense ? (uint32_t)min(total_entries(V, F), (unsigned long long)ray_count) : ray_count;
    for (uint32_t base_ray = blockIdx.x * blockDim.x; base_ray < rays; base_ray += gridDim.x * blockDim.x)
        shade_warp(V, F, F.shade, S, base_ray + threadIdx.x, rays);
}

// Visibility queries, one per lane (traceVisibility, shaders/split.slang:1326-1339).
// result: 0 visible, 1 blocked, 2 unsupported.
__global__ void __launch_bounds__(128, LUX_REFILL_MIN_BLOCKS) shadow_refill_kernel(ViewDevice V, FrameParams F, SceneView S) {
    if (*V.error_flags) return;
#if LUX_WARP_LEAVES
    __shared__ lux::LeafScratch scratch[4];
    lux::LeafScratch *L = &scratch[threadIdx.x >> 5];
#else
    lux::LeafScratch *L = nullptr;
#endif
    uint32_t n = min(*V.ts.queue_count, F.queue_capacity);
    unsigned long long st[7] = {0, 0, 0, 0, 0, 0, 0};
    lux::TraceCounters cn{0, 0, 0};
    lux::trace_persistent<true>(
        S, &V.ts.work_counter[1], n,
        [&](uint32_t i, f3 &o, f3 &d, float &tmin, float &limit) {
            uint32_t qi = V.ts.query_slot[V.query_order ? V.query_order[i] : i];
            float4 a = V.ts.queue_o[qi], b = V.ts.queue_d[qi];
            o = f3{a.x, a.y, a.z};
            d = f3{b.x, b.y, b.z};
            tmin = 0.0f;
            limit = a.w;
        },
        [&](uint32_t i, const lux::Hit &sh) {
            uint32_t qi = V.ts.query_slot[V.query_order ? V.query_order[i] : i];
            V.ts.queue_result[qi] = sh.tri != lux::kEmpty ? 1 : ((sh.errors & lux::kQueryUnsupported) ? 2 : 0);
            st[kStatShadow] += 1;
        },
        cn, L);
    st[kStatNodes] = cn.nodes;
    st[kStatTris] = cn.triangles;
    st[kStatInst] = cn.instances;
    unsigned long long extra[3] = {cn.nodes, cn.triangles, cn.instances};
    add_stats(V.stats, st, extra);
}

// One visibility query (traceVisibility, shaders/split.slang:1326-1339):
// result 0 visible, 1 blocked, 2 unsupported.
template <int kDepth = lux::kStack>
__device__ __forceinline__ void shadow_query(const ViewDevice &V, const SceneView &S, uint32_t i,
                                             lux::TraceCounters &cn) {
    uint32_t qi = V.ts.query_slot[V.query_order ? V.query_order[i] : i];
    float4 a = V.ts.queue_o[qi], b = V.ts.queue_d[qi];
    lux::Hit sh;
    lux::trace<true, kDepth>(S, f3{a.x, a.y, a.z}, f3{b.x, b.y, b.z}, 0.0f, a.w, sh, cn);
    V.ts.queue_result[qi] = sh.tri != lux::kEmpty ? 1 : ((sh.errors & lux::kQueryUnsupported) ? 2 : 0);
}

// shadow_query for a whole warp (every lane calls it; `valid`: the lane has
// a query).
template <int kDepth = lux::kStack>
__device__ __forceinline__ void shadow_query_warp(const ViewDevice &V, const SceneView &S, uint32_t i, bool valid,
                                                  lux::TraceCounters &cn, lux::LeafScratch *L) {
    uint32_t qi = 0;
    float4 a = make_float4(0.0f, 0.0f, 0.0f, 0.0f), b = a;
    if (valid) {
        qi = V.ts.query_slot[V.query_order ? V.query_order[i] : i];
        a = V.ts.queue_o[qi];
        b = V.ts.queue_d[qi];
    }
    lux::Hit sh;
    lux::trace_warp<true, kDepth>(S, valid, f3{a.x, a.y, a.z}, f3{b.x, b.y, b.z}, 0.0f, a.w, sh, cn, L);
    if (valid) V.ts.queue_result[qi] = sh.tri != lux::kEmpty ? 1 : ((sh.errors & lux::kQueryUnsupported) ? 2 : 0);
}

template <int kDepth>
__global__ void __launch_bounds__(128, LUX_SHADOW_MIN_BLOCKS) shadow_kernel(ViewDevice V, FrameParams F, SceneView S,
                                                                             uint32_t tile) {
    if (*V.error_flags) return;
#if LUX_WARP_LEAVES
    __shared__ lux::LeafScratch scratch[4];
    lux::LeafScratch *L = &scratch[threadIdx.x >> 5];
#endif
    uint32_t n = min(*V.ts.queue_count, F.queue_capacity);
    unsigned long long st[7] = {0, 0, 0, 0, 0, 0, 0};
    lux::TraceCounters cn{0, 0, 0};
    while (true) {
        uint32_t base = warp_fetch(&V.ts.work_counter[1], tile);
        if (base >= n) break;
        for (uint32_t k = 0; k < tile && base + k < n; k += 32u) {
            uint32_t i = base + k + (threadIdx.x & 31u);
#if LUX_WARP_LEAVES
            shadow_query_warp<kDepth>(V, S, i, i < n, cn, L);
            if (i < n) st[kStatShadow] += 1;
#else
            if (i < n) {
                shadow_query<kDepth>(V, S, i, cn);
                st[kStatShadow] += 1;
            }
#endif
        }
    }
    st[kStatNodes] = cn.nodes;
    st[kStatTris] = cn.triangles;
    st[kStatInst] = cn.instances;
    unsigned long long extra[3] = {cn.nodes, cn.triangles, cn.instances};
    add_stats(V.stats, st, extra);
}

// Next-event sum in sample order (plus the multi-bounce term with
// `feedback`); false when the ray's query is unsupported.
__device__ __forceinline__ bool ray_radiance(const ViewDevice &V, uint32_t ray, f3 &radiance, bool feedback = false) {
    float4 b = V.ts.ray_base[ray];
    const uint32_t packed = lux::as_uint(b.w);
    if (packed == lux::kEmpty) return false;
    // The emissive samples (averaged), the environment samples (averaged over
    // the same count) then the conventional lights (summed).
    const uint32_t count = packed & 31u, conventional = (packed >> 5) & 15u;
    const uint32_t environment = ((packed >> 9) & 1u) != 0u ? count : 0u;
    const uint32_t used = packed >> 16;
    f3 sum{0.0f, 0.0f, 0.0f}, esum{0.0f, 0.0f, 0.0f}, csum{0.0f, 0.0f, 0.0f};
    for (uint32_t s = 0; s < count + environment + conventional && s < lux::kMaxNeeSamples; ++s) {
        if (!(used & (1u << s))) continue;
        size_t slot = (size_t)ray * lux::kMaxNeeSamples + s;
        uint8_t r = V.ts.queue_result[slot];
        if (r == 2) return false;
        if (r == 1) continue;
        float4 c = V.ts.slot_contrib[slot];
        if (s < count)
            sum = f3{sum.x + c.x, sum.y + c.y, sum.z + c.z};
        else if (s < count + environment)
            esum = f3{esum.x + c.x, esum.y + c.y, esum.z + c.z};
        else
            csum = f3{csum.x + c.x, csum.y + c.y, csum.z + c.z};
    }
    float4 e = feedback ? V.ts.ray_extra[ray] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    f3 extra{e.x, e.y, e.z};
    radiance = lux::finish_radiance(f3{b.x, b.y, b.z}, sum, count, environment ? &esum : nullptr,
                                    conventional ? &csum : nullptr, feedback ? &extra : nullptr);
    return true;
}

// deposit, shaders/split.slang:1056-1117: every level up to and including
// the one whose interval holds the hit; the last level owns the tail.
__device__ __forceinline__ void deposit_split_ray(const ViewDevice &V, const FrameParams &F, uint32_t frame,
                                                  const float4 *__restrict__ nrm, uint32_t ray,
                                                  unsigned long long st[7]) {
    uint32_t i = ray / F.rays_per_receiver, k = ray % F.rays_per_receiver;
    if (F.sparse && V.receiver_cell[i] == lux::kEmpty) return;  // absent receiver: no ray
    f3 radiance;
    if (!ray_radiance(V, ray, radiance, F.shade.feedback != 0u)) {
        st[kStatUnsupported] += 1;
        return;
    }
    float4 n4 = nrm[i];
    f3 dir;
    float u, v;
    split_direction(V, F, frame, i, k, f3{n4.x, n4.y, n4.z}, dir, u, v);
    float t = V.ts.ray_o[ray].w;
    // splitIntervalContainsHit at the receiver's LOD (ends scale by 2^lod,
    // shaders/split.slang:224-236).
    const float ls = F.lod_enabled ? lux::lod_scale(V.receiver_lod[i]) : 1.0f;
    uint32_t term = F.levels - 1u;
    for (uint32_t l = 0; l + 1u < F.levels; ++l)
        if (t > F.start[l] * ls && t <= F.end[l] * ls) {
            term = l;
            break;
        }
    for (uint32_t l = 0; l <= term; ++l) {
        uint32_t cell = V.receiver_cell[(size_t)l * F.receivers + i];
        if (cell == lux::kEmpty) continue;
        uint32_t bin = lux::direction_index_uv(u, v, F.columns[l], F.rows[l]);
        unsigned long long e = V.level_base[l] + (unsigned long long)cell * F.dirs[l] + bin;
        atomicAdd(&V.count[e], 1u);
        if (l == term)  // one 16-byte vector atomic (w += 0 leaves the count of passes unchanged)
            atomicAdd(&V.accum[e], make_float4(radiance.x, radiance.y, radiance.z, 0.0f));
        else
            atomicAdd(&V.accum[e].w, 1.0f);
        st[kStatDeposits] += 1;
    }
}

__global__ void __launch_bounds__(128) deposit_split_kernel(ViewDevice V, FrameParams F,
                                                            const float4 *__restrict__ nrm, uint32_t ray_count) {
    unsigned long long st[7] = {0, 0, 0, 0, 0, 0, 0};
    uint32_t ray = blockIdx.x * blockDim.x + threadIdx.x;
    if (*V.error_flags == 0u && ray < ray_count) deposit_split_ray(V, F, F.shade.frame, nrm, ray, st);
    add_stats(V.stats, st);
}

__global__ void __launch_bounds__(128) deposit_dense_kernel(ViewDevice V, FrameParams F) {
    if (*V.error_flags) return;
    unsigned long long n = total_entries(V, F);
    for (unsigned long long e = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
         e < ((n + 31ull) & ~31ull); e += (unsigned long long)gridDim.x * blockDim.x) {
        unsigned long long st[7] = {0, 0, 0, 0, 0, 0, 0};
        if (e < n) {
            uint32_t level = 0;
            while (level + 1u < F.levels && e >= V.level_base[level + 1u]) ++level;
            bool terminal = level + 1u == F.levels;
            f3 radiance;
            if (ray_radiance(V, (uint32_t)e, radiance)) {
                bool terminates = terminal || V.ts.ray_h[e].x != lux::kEmpty;
                V.count[e] = 1u;
                V.accum[e] = terminates ? make_float4(radiance.x, radiance.y, radiance.z, 0.0f)
                                        : make_float4(0.0f, 0.0f, 0.0f, 1.0f);
                st[kStatDeposits] = 1;
            } else {
                st[kStatUnsupported] = 1;
            }
        }
        add_stats(V.stats, st);
    }
}

// Spatial corners of every cell of `level` in level + 1 (mergeRadianceGroups
// grid, shaders/split.slang:1590-1596).
// One corner of cell c (corner 0 also writes the interpolation weights):
// the eight directory probes of a cell run in eight threads.
__device__ __forceinline__ void corner_item(const ViewDevice &V, const FrameParams &F, uint32_t level, uint32_t c,
                                            uint32_t corner) {
    int4 key = V.cell_keys[(size_t)level * F.cell_capacity + c];
    const uint32_t lod = lux::key_lod(key.w);
    const float sp = level_spacing(F, level, lod), sp1 = level_spacing(F, level + 1, lod);
    float ox = ((float)key.x + 0.5f) * sp, oy = ((float)key.y + 0.5f) * sp, oz = ((float)key.z + 0.5f) * sp;
    float gx = ox / sp1 - 0.5f, gy = oy / sp1 - 0.5f, gz = oz / sp1 - 0.5f;
    float fx = floorf(gx), fy = floorf(gy), fz = floorf(gz);
    int32_t bx = (int32_t)fx, by = (int32_t)fy, bz = (int32_t)fz;
    if (corner == 0u) V.corner_frac[(size_t)level * F.cell_capacity + c] = make_float4(gx - fx, gy - fy, gz - fz, 0.0f);
    V.corner_ids[((size_t)level * F.cell_capacity + c) * 8 + corner] =
        cell_id(V, F, level + 1, bx + (int32_t)(corner & 1u), by + (int32_t)((corner >> 1) & 1u),
                bz + (int32_t)(corner >> 2), lod);
}

__device__ __forceinline__ void corners_item(const ViewDevice &V, const FrameParams &F, uint32_t level, uint32_t c) {
    int4 key = V.cell_keys[(size_t)level * F.cell_capacity + c];
    // A cell's children are the next level's cells of the same LOD.
    const uint32_t lod = lux::key_lod(key.w);
    const float sp = level_spacing(F, level, lod), sp1 = level_spacing(F, level + 1, lod);
    float ox = ((float)key.x + 0.5f) * sp, oy = ((float)key.y + 0.5f) * sp, oz = ((float)key.z + 0.5f) * sp;
    float gx = ox / sp1 - 0.5f, gy = oy / sp1 - 0.5f, gz = oz / sp1 - 0.5f;
    float fx = floorf(gx), fy = floorf(gy), fz = floorf(gz);
    int32_t bx = (int32_t)fx, by = (int32_t)fy, bz = (int32_t)fz;
    V.corner_frac[(size_t)level * F.cell_capacity + c] = make_float4(gx - fx, gy - fy, gz - fz, 0.0f);
    uint32_t *ids = V.corner_ids + ((size_t)level * F.cell_capacity + c) * 8;
#pragma unroll
    for (uint32_t corner = 0; corner < 8u; ++corner)
        ids[corner] = cell_id(V, F, level + 1, bx + (int32_t)(corner & 1u), by + (int32_t)((corner >> 1) & 1u),
                              bz + (int32_t)(corner >> 2), lod);
}


#if !LUX_MERGE_CORNER_OUTER
// interpolateMergedChildSources, shaders/split.slang:389-479 (one group).
__device__ __forceinline__ float4 interpolate(const ViewDevice &V, const FrameParams &F, uint32_t child_level,
                                              const uint32_t ids[8], float4 frac, uint32_t dir) {
    float sx = 0.0f, sy = 0.0f, sz = 0.0f, total = 0.0f, potential = 0.0f;
    unsigned long long base = V.level_base[child_level];
    uint32_t dirs = F.dirs[child_level];
    // The eight corner records are fetched before any is used (record 0
    // stands in for a missing corner), so their latencies overlap.
    float4 corner_value[8];
#pragma unroll
    for (uint32_t corner = 0; corner < 8u; ++corner)
        corner_value[corner] = __ldg(V.merged + (ids[corner] == lux::kEmpty
                                                     ? 0ull
                                                     : base + (unsigned long long)ids[corner] * dirs + dir));
#pragma unroll
    for (uint32_t corner = 0; corner < 8u; ++corner) {
        float ax = (corner & 1u) == 0u ? 1.0f - frac.x : frac.x;
        float ay = ((corner >> 1) & 1u) == 0u ? 1.0f - frac.y : frac.y;
        float az = (corner >> 2) == 0u ? 1.0f - frac.z : frac.z;
        float w = (ax * ay) * az;
        if (!(w > 0.0f)) continue;
        potential += w;
        if (ids[corner] == lux::kEmpty) continue;
        float4 s = corner_value[corner];
        if (s.w > 0.0f && isfinite(s.x) && isfinite(s.y) && isfinite(s.z) && isfinite(s.w)) {
            float sw = w * lux::saturate(s.w);
            sx = sx + s.x * sw;
            sy = sy + s.y * sw;
            sz = sz + s.z * sw;
            total += sw;
        }
    }
    if (total > 0.0f) return make_float4(sx / total, sy / total, sz / total, lux::saturate(total / fmaxf(potential, 1e-8f)));
    return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}
#endif

// The four children of record (x, y) interpolated together: corners outer,
// children inner, so each corner's weight and validity are worked out once
// and its four child records (two adjacent pairs) are loaded together.  Per
// child the corners are summed in the same order as interpolate(), and the
// potential (the sum of positive weights) is the same for every child, so
// every result is bit-identical to four interpolate() calls.
__device__ __forceinline__ void interpolate_children(const ViewDevice &V, const FrameParams &F,
                                                     uint32_t child_level, const uint32_t ids[8], float4 frac,
                                                     uint32_t fine0, uint32_t fine_columns, float4 out[4]) {
    float acc[4][4];
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[k][0] = acc[k][1] = acc[k][2] = acc[k][3] = 0.0f;
    float potential = 0.0f;
    const unsigned long long base = V.level_base[child_level];
    const uint32_t dirs = F.dirs[child_level];
    const uint32_t offset[4] = {fine0, fine0 + 1u, fine0 + fine_columns, fine0 + fine_columns + 1u};
#pragma unroll
    for (uint32_t corner = 0; corner < 8u; ++corner) {
        float ax = (corner & 1u) == 0u ? 1.0f - frac.x : frac.x;
        float ay = ((corner >> 1) & 1u) == 0u ? 1.0f - frac.y : frac.y;
        float az = (corner >> 2) == 0u ? 1.0f - frac.z : frac.z;
        float w = (ax * ay) * az;
        if (!(w > 0.0f)) continue;
        potential += w;
        if (ids[corner] == lux::kEmpty) continue;
        const float4 *rec = V.merged + base + (unsigned long long)ids[corner] * dirs;
        float4 s[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) s[k] = __ldg(rec + offset[k]);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (s[k].w > 0.0f && isfinite(s[k].x) && isfinite(s[k].y) && isfinite(s[k].z) && isfinite(s[k].w)) {
                float sw = w * lux::saturate(s[k].w);
                acc[k][0] = acc[k][0] + s[k].x * sw;
                acc[k][1] = acc[k][1] + s[k].y * sw;
                acc[k][2] = acc[k][2] + s[k].z * sw;
                acc[k][3] += sw;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float total = acc[k][3];
        out[k] = total > 0.0f ? make_float4(acc[k][0] / total, acc[k][1] / total, acc[k][2] / total,
                                            lux::saturate(total / fmaxf(potential, 1e-8f)))
                              : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

// mergeEntry without history, shaders/split.slang:1523-1725.
// base^n by squaring and multiplying in a fixed order (the CPU restatement
// rounds identically); pow(blend, observations) of mergeRawRadianceGroup.
__device__ __forceinline__ float pow_count(float base, uint32_t n) {
    float r = 1.0f, b = base;
    while (n) {
        if (n & 1u) r = r * b;
        b = b * b;
        n >>= 1;
    }
    return r;
}

// The previous frame's dense id of every cell of `level` (kEmpty when the
// cell was not there or its history is invalidated), one directory probe per
// cell instead of one per record.
__device__ __forceinline__ bool record_dirty(const FrameParams &F, uint32_t level, int4 key);

__device__ __forceinline__ void history_map_item(const ViewDevice &V, const FrameParams &F, const HistoryDevice &H,
                                                 uint32_t level, uint32_t c) {
    uint32_t id = lux::kEmpty;
    int4 key = V.cell_keys[(size_t)level * F.cell_capacity + c];
    if (lux::cell_in_range(key.x, key.y, key.z) && !record_dirty(F, level, key)) {
        const uint32_t lod = lux::key_lod(key.w);
        unsigned long long packed = lux::pack_cell(key.x, key.y, key.z, lod);
        const unsigned long long *keys = H.dir_keys + (size_t)level * F.dir_capacity;
        uint32_t slot = lux::hash_key(key.x, key.y, key.z, (int32_t)(level | (lod << 18)), F.dir_capacity);
        for (uint32_t attempt = 0; attempt < F.dir_capacity; ++attempt) {
            unsigned long long k = keys[slot];
            if (k == packed) {
                uint32_t prev = H.dir_ids[(size_t)level * F.dir_capacity + slot];
                if (prev != lux::kEmpty && prev < H.cell_count[level]) id = prev;
                break;
            }
            if (k == lux::kEmptyCell) break;
            slot = (slot + 1u) & (F.dir_capacity - 1u);
        }
    }
    V.hist_cell[(size_t)level * F.cell_capacity + c] = id;
}

// Before the merge, one launch for every level: each cell's corners in the
// next level, and with history its previous frame's id.
__global__ void merge_prep_kernel(ViewDevice V, FrameParams F, HistoryDevice H) {
    if (*V.error_flags) return;
    if (blockIdx.x == 0 && threadIdx.x < F.levels) V.pass_count[threadIdx.x] = 0u;
    for (uint32_t l = 0; l < F.levels; ++l) {
        const uint32_t cells = min(V.cell_count[l], F.cell_capacity);
#if LUX_MERGE_PREP_SPLIT
        // Eight threads per cell, one corner each; the history map goes to
        // the thread of corner 7.
        const unsigned long long items = (unsigned long long)cells * 8u;
        for (unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < items;
             k += (unsigned long long)gridDim.x * blockDim.x) {
            const uint32_t c = (uint32_t)(k >> 3), corner = (uint32_t)k & 7u;
            if (l + 1u < F.levels) corner_item(V, F, l, c, corner);
            if (F.history && corner == 7u) history_map_item(V, F, H, l, c);
        }
#else
        for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += gridDim.x * blockDim.x) {
            if (l + 1u < F.levels) corners_item(V, F, l, c);
            if (F.history) history_map_item(V, F, H, l, c);
        }
#endif
    }
}

// A record's history is invalid when the region its rays may have crossed
// (the cell grown by the level's interval end; unbounded at the last level)
// meets an invalidation box (dirtyRawCacheEntry / betaHistoryEligible,
// shaders/split.slang:123-132, :201-203, with a box dependency).
__device__ __forceinline__ bool record_dirty(const FrameParams &F, uint32_t level, int4 key) {
    if (F.dirty_count == 0u) return false;
    if (level + 1u >= F.levels) return true;
    const float ls = lux::lod_scale(lux::key_lod(key.w));
    float s = F.spacing[level] * ls, reach = F.end[level] * ls;
    float lo[3] = {(float)key.x * s - reach, (float)key.y * s - reach, (float)key.z * s - reach};
    float hi[3] = {(float)(key.x + 1) * s + reach, (float)(key.y + 1) * s + reach, (float)(key.z + 1) * s + reach};
    for (uint32_t b = 0; b < F.dirty_count && b < (uint32_t)kMaxDirty; ++b) {
        bool meet = true;
        for (int a = 0; a < 3; ++a) meet = meet && lo[a] <= F.dirty_hi[b][a] && hi[a] >= F.dirty_lo[b][a];
        if (meet) return true;
    }
    return false;
}

// retain (shaders/split.slang:991-1054): with history on, the world cache is
// persistent (persistentWorldIntervals, shaders/common.slang:82-89, is set
// for the Split method at src/render.rs:8470), so every cell of the previous
// frame that no receiver seeded this frame stays in the cache with its
// records, which the merge carries forward unchanged (no fresh samples) and
// which parents and the resolve keep reading.  A cell whose history an
// invalidation box voids is dropped (betaHistoryEligible).  Capacity bounds
// the cache as commitCache's per-bucket quota does (youngest kept,
// :1919-1961): levels in order, whole age classes (frames since the cell's
// last receiver) youngest first, while the cells fit max_cells and all
// records the view's max_entries.
// Age class of the previous frame's cell `prev` of `level`, or kRetainBins
// when it is not retained (seeded this frame, or its history voided).
__device__ __forceinline__ uint32_t retain_bin(const ViewDevice &V, const FrameParams &F, const HistoryDevice &H,
                                               uint32_t level, uint32_t prev, int4 &key) {
    key = H.cell_keys[(size_t)level * F.cell_capacity + prev];
    if (dir_find(V, F, level, key.x, key.y, key.z, lux::key_lod(key.w)) != lux::kEmpty)
        return kRetainBins;  // seeded this frame
    if (record_dirty(F, level, key)) return kRetainBins;
    uint32_t age = F.shade.frame - H.cell_last[(size_t)level * F.cell_capacity + prev];
    return min(age, kRetainBins - 1u);
}

__global__ void retain_count_kernel(ViewDevice V, FrameParams F, HistoryDevice H) {
    for (uint32_t l = 0; l < F.levels; ++l) {
        uint32_t cells = min(H.cell_count[l], F.cell_capacity);
        for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += gridDim.x * blockDim.x) {
            int4 key;
            uint32_t bin = retain_bin(V, F, H, l, c, key);
            if (bin < kRetainBins) atomicAdd(&V.retain_hist[l * kRetainBins + bin], 1u);
        }
    }
}

// One block of kRetainBins threads: per level, an inclusive scan of the age
// histogram; the limit is the number of classes whose running total fits.
__device__ __forceinline__ void retain_limit_block(const ViewDevice &V, const FrameParams &F) {
    __shared__ unsigned long long scan[kRetainBins];
    __shared__ unsigned long long remaining;
    const uint32_t t = threadIdx.x;
    if (t == 0) {
        unsigned long long used = 0;
        for (uint32_t l = 0; l < F.levels; ++l)
            used += (unsigned long long)min(V.cell_count[l], F.cell_capacity) * F.dirs[l];
        remaining = used < F.entry_capacity ? F.entry_capacity - used : 0ull;
    }
    for (uint32_t l = 0; l < F.levels; ++l) {
        scan[t] = V.retain_hist[l * kRetainBins + t];
        __syncthreads();
        for (uint32_t off = 1; off < kRetainBins; off <<= 1) {
            unsigned long long add = t >= off ? scan[t - off] : 0ull;
            __syncthreads();
            scan[t] += add;
            __syncthreads();
        }
        unsigned long long seeded = min(V.cell_count[l], F.cell_capacity);
        unsigned long long room = min((unsigned long long)F.cell_capacity - seeded, remaining / F.dirs[l]);
        uint32_t fits = (uint32_t)__syncthreads_count(scan[t] <= room);  // the scan is non-decreasing
        if (t == 0) {
            V.retain_limit[l] = fits;
            remaining -= (fits ? scan[fits - 1] : 0ull) * F.dirs[l];
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kRetainBins) retain_limit_kernel(ViewDevice V, FrameParams F) {
    retain_limit_block(V, F);
}

// Inserts the retained cell `prev` of `level` into this frame's directory
// with a new dense id and its last-receiver frame.
__device__ __forceinline__ void retain_cell(const ViewDevice &V, const FrameParams &F, const HistoryDevice &H,
                                            uint32_t level, uint32_t prev, int4 k) {
    const uint32_t lod = lux::key_lod(k.w);
    unsigned long long key = lux::pack_cell(k.x, k.y, k.z, lod);
    unsigned long long *keys = V.dir_keys + (size_t)level * F.dir_capacity;
    uint32_t slot = lux::hash_key(k.x, k.y, k.z, (int32_t)(level | (lod << 18)), F.dir_capacity);
    // The directory is at most half full (dir_capacity >= 2 max_cells).
    for (uint32_t attempt = 0; attempt < F.dir_capacity; ++attempt) {
        if (atomicCAS(&keys[slot], lux::kEmptyCell, key) == lux::kEmptyCell) {
            uint32_t id = atomicAdd(&V.cell_count[level], 1u);  // below cell_capacity by retain_limit
            V.dir_ids[(size_t)level * F.dir_capacity + slot] = id;
            V.cell_keys[(size_t)level * F.cell_capacity + id] =
                make_int4(k.x, k.y, k.z, (int32_t)((level << 12) | (lod << 18)));
            V.cell_last[(size_t)level * F.cell_capacity + id] = H.cell_last[(size_t)level * F.cell_capacity + prev];
            return;
        }
        slot = (slot + 1u) & (F.dir_capacity - 1u);
    }
    atomicOr(V.error_flags, LUX_VIEW_ERR_CELL_CAPACITY);
}

__global__ void retain_insert_kernel(ViewDevice V, FrameParams F, HistoryDevice H) {
    for (uint32_t l = 0; l < F.levels; ++l) {
        uint32_t cells = min(H.cell_count[l], F.cell_capacity);
        for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += gridDim.x * blockDim.x) {
            int4 key;
            if (retain_bin(V, F, H, l, c, key) < V.retain_limit[l]) retain_cell(V, F, H, l, c, key);
        }
    }
}

// mergeEntry (shaders/split.slang:1624-1725) for one record: the fresh mean
// (J, beta) of this frame's observations blended with the previous frame's
// record by mergeRawRadianceGroup's masses (retention blend^n, mass limit
// 1 / (1 - blend); :1478-1521) for the summed radiance group and for the
// transmittance, then Eq. 7 with the children: I = [J (1 - beta) + beta
// mean_4(trilerp_8(I_child) support)] / support.
// Record (cell, d) of `level`; base = the level's first record.
// The record's own part (fresh mean, history blend, raw and mass records
// written): its radiance, support and transmittance, and whether the
// children must be interpolated (transmittance > 0 below the coarsest level).
struct MergeOwn {
    float rx, ry, rz, support, transmittance;
};

__device__ __forceinline__ bool merge_own(const ViewDevice &V, const FrameParams &F, const HistoryDevice &H,
                                          uint32_t level, unsigned long long base, uint32_t dirs, uint32_t cell,
                                          uint32_t d, MergeOwn &own) {
    const unsigned long long e = (unsigned long long)cell * dirs + d;
    const bool has_children = level + 1u < F.levels;
    const float jb = F.radiance_blend, tb = F.transmittance_blend;
    const float jlimit = 1.0f / (1.0f - jb), tlimit = 1.0f / (1.0f - tb);
    uint32_t cnt = V.count[base + e];
    float4 fresh = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (cnt) {
        float4 acc = V.accum[base + e];
        float fn = (float)cnt;
        fresh = make_float4(acc.x / fn, acc.y / fn, acc.z / fn, acc.w / fn);
    }
    // History of this record.
    bool reuse = false;
    float4 old = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float2 old_mass = make_float2(0.0f, 0.0f);
    if (F.history) {
        uint32_t prev = V.hist_cell[(size_t)level * F.cell_capacity + cell];
        if (prev != lux::kEmpty) {
            unsigned long long r = H.level_base[level] + (unsigned long long)prev * dirs + d;
            old = H.raw[r];
            old_mass = H.mass[r];
            reuse = true;
        }
    }
    float rm = old_mass.x, tm = old_mass.y;
    if (!isfinite(rm) || rm < 0.0f) rm = 0.0f;
    if (!isfinite(tm) || tm < 0.0f) tm = 0.0f;
    const bool reuse_r = reuse && jb > 0.0f, reuse_t = reuse && tb > 0.0f;
    float jx = 0.0f, jy = 0.0f, jz = 0.0f, beta = 1.0f, rmass = 0.0f, tmass = 0.0f;
    if (cnt) {
        float ret = pow_count(jb, cnt);
        rmass = (1.0f - ret) * jlimit;
        jx = fresh.x;
        jy = fresh.y;
        jz = fresh.z;
        float om = fminf(rm, jlimit) * ret;
        if (reuse_r && om > 0.0f) {
            jx = (jx * rmass + old.x * om) / (rmass + om);
            jy = (jy * rmass + old.y * om) / (rmass + om);
            jz = (jz * rmass + old.z * om) / (rmass + om);
            rmass = rmass + om;
        }
        float tret = pow_count(tb, cnt);
        tmass = (1.0f - tret) * tlimit;
        beta = fresh.w;
        float otm = fminf(tm, tlimit) * tret;
        if (reuse_t && otm > 0.0f) {
            beta = (beta * tmass + old.w * otm) / (tmass + otm);
            tmass = tmass + otm;
        }
    } else {
        if (reuse_r && rm > 0.0f) {
            jx = old.x;
            jy = old.y;
            jz = old.z;
            rmass = rm;
        }
        if (reuse_t && tm > 0.0f) {
            beta = old.w;
            tmass = tm;
        }
    }
    float transmittance = tmass > 0.0f ? lux::saturate(beta) : 0.0f;
    float support = rmass > 0.0f && tmass > 0.0f ? 1.0f - transmittance : 0.0f;
    float rx = 0.0f, ry = 0.0f, rz = 0.0f;
    if (support > 0.0f) {
        rx = jx;
        ry = jy;
        rz = jz;
    }
    // The raw record does not depend on the children: stored first, so its
    // values need no registers across the child interpolation.
    V.raw[base + e] = (cnt || rmass > 0.0f || tmass > 0.0f) ? make_float4(jx, jy, jz, beta)
                                                             : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    V.mass[base + e] = make_float2(rmass, tmass);
    own = MergeOwn{rx, ry, rz, support, transmittance};
    return transmittance > 0.0f && has_children;
}

// The children's part (with `children`) and the merged record written.
__device__ __forceinline__ void merge_finish(const ViewDevice &V, const FrameParams &F, uint32_t level,
                                             unsigned long long base, uint32_t dirs, uint32_t cell, uint32_t d,
                                             MergeOwn own, bool children) {
    const unsigned long long e = (unsigned long long)cell * dirs + d;
    float rx = own.rx, ry = own.ry, rz = own.rz, support = own.support;
    const float transmittance = own.transmittance;
    float cx = 0.0f, cy = 0.0f, cz = 0.0f, csup = 0.0f;
    if (children) {
        size_t ci = (size_t)level * F.cell_capacity + cell;
        uint32_t ids[8];
        const uint4 *cid = reinterpret_cast<const uint4 *>(V.corner_ids + ci * 8);  // 32-byte rows
        uint4 c0 = __ldg(cid), c1 = __ldg(cid + 1);
        ids[0] = c0.x;
        ids[1] = c0.y;
        ids[2] = c0.z;
        ids[3] = c0.w;
        ids[4] = c1.x;
        ids[5] = c1.y;
        ids[6] = c1.z;
        ids[7] = c1.w;
        float4 frac = __ldg(V.corner_frac + ci);
        uint32_t x = d % F.columns[level], y = d / F.columns[level];
        uint32_t fine_columns = F.columns[level + 1];
#if LUX_MERGE_CORNER_OUTER
        float4 child_value[4];
        interpolate_children(V, F, level + 1, ids, frac, x * 2u + y * 2u * fine_columns, fine_columns, child_value);
#pragma unroll
        for (uint32_t child = 0; child < 4u; ++child) {
            float4 v = child_value[child];
            if (!(v.w > 0.0f)) continue;
            cx = cx + v.x * v.w;
            cy = cy + v.y * v.w;
            cz = cz + v.z * v.w;
            csup += v.w;
        }
#else
#pragma unroll
        for (uint32_t child = 0; child < 4u; ++child) {
            uint32_t fine = (x * 2u + (child & 1u)) + (y * 2u + (child >> 1)) * fine_columns;
            float4 v = interpolate(V, F, level + 1, ids, frac, fine);
            if (!(v.w > 0.0f)) continue;
            cx = cx + v.x * v.w;
            cy = cy + v.y * v.w;
            cz = cz + v.z * v.w;
            csup += v.w;
        }
#endif
    }
    if (csup > 0.0f) {
        rx = rx + (transmittance * cx) * 0.25f;
        ry = ry + (transmittance * cy) * 0.25f;
        rz = rz + (transmittance * cz) * 0.25f;
        support = support + (transmittance * csup) * 0.25f;
    }
    float4 out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (support > 0.0f) out = make_float4(rx / support, ry / support, rz / support, lux::saturate(support));
    V.merged[base + e] = out;
}

// Processing order of a level's records: item i of cells x dirs is record
// (cell, d) taken in direction blocks of kMergeRun consecutive directions,
// every cell's run of a block before the next block.  A warp still covers
// 32 consecutive records of one cell (coalesced), while the warps in flight
// at any moment span few directions of many cells, so the child records they
// interpolate (four fine directions per record, in the same eight corner
// cells for neighbouring cells) are shared in cache instead of being re-read
// once per parent cell, as a cell-major order does on the coarse levels
// (few cells, up to 2^19 directions each).
constexpr uint32_t kMergeRun = 32;

__device__ __forceinline__ void merge_item(unsigned long long i, uint32_t cells, uint32_t dirs, uint32_t &cell,
                                           uint32_t &d) {
    if (dirs % kMergeRun != 0u) {  // no direction blocks: cell-major
        cell = (uint32_t)(i / dirs);
        d = (uint32_t)(i % dirs);
        return;
    }
    const unsigned long long block = (unsigned long long)cells * kMergeRun;
    if ((unsigned long long)cells * dirs <= 0xffffffffull) {  // 32-bit divisions
        const uint32_t i32 = (uint32_t)i, b32 = (uint32_t)block;
        const uint32_t run = i32 / b32, rem = i32 - run * b32;
        cell = rem / kMergeRun;
        d = run * kMergeRun + (rem % kMergeRun);
    } else {
        const unsigned long long run = i / block, rem = i - run * block;
        cell = (uint32_t)(rem / kMergeRun);
        d = (uint32_t)(run * kMergeRun + rem % kMergeRun);
    }
}

// The merge in two passes.  A record's own part (fresh mean, history blend,
// raw and mass records) does not depend on the children, so one launch takes
// it for the records of every level at once, in storage order, and finishes
// the records whose merged value needs no children (no transmittance, or the
// coarsest level).  Then, coarsest level first, one launch per level takes
// the records that pass light on: their own part is read back from the raw
// and mass records just written (transmittance = saturate(beta) when the
// transmittance mass is positive; support = 1 - transmittance when the
// radiance mass is positive too; the radiance is the raw record's), which
// gives exactly the values merge_own returned, and adds the children.
// Record r of a level (cell-major): its cell and direction, by a shift when
// the level's direction count is a power of two, else by a 32-bit division
// when r fits in 32 bits (a 64-bit one otherwise).
__device__ __forceinline__ void record_cell(unsigned long long r, uint32_t dirs, uint32_t &cell, uint32_t &d) {
    if ((dirs & (dirs - 1u)) == 0u) {
        const uint32_t shift = (uint32_t)__ffs(dirs) - 1u;
        cell = (uint32_t)(r >> shift);
        d = (uint32_t)r & (dirs - 1u);
    } else if (r <= 0xffffffffull) {
        cell = (uint32_t)r / dirs;
        d = (uint32_t)r - cell * dirs;
    } else {
        cell = (uint32_t)(r / dirs);
        d = (uint32_t)(r - (unsigned long long)cell * dirs);
    }
}

__device__ __forceinline__ void merge_own_record(const ViewDevice &V, const FrameParams &F, const HistoryDevice &H,
                                                 uint32_t level, unsigned long long base, uint32_t dirs,
                                                 unsigned long long r) {
    uint32_t cell, d;
    record_cell(r, dirs, cell, d);
    MergeOwn own;
    if (!merge_own(V, F, H, level, base, dirs, cell, d, own)) merge_finish(V, F, level, base, dirs, cell, d, own, false);
}

// Record e of the frame (all levels in storage order): its level by a scan
// of the level bases.
__device__ __forceinline__ void merge_own_entry(const ViewDevice &V, const FrameParams &F, const HistoryDevice &H,
                                                unsigned long long e) {
    uint32_t level = 0;
    while (level + 1u < F.levels && e >= V.level_base[level + 1u]) ++level;
    const unsigned long long base = V.level_base[level];
    merge_own_record(V, F, H, level, base, F.dirs[level], e - base);
}

__device__ __forceinline__ void merge_children_record(const ViewDevice &V, const FrameParams &F, uint32_t level,
                                                      unsigned long long base, uint32_t dirs, uint32_t cell,
                                                      uint32_t d) {
    const unsigned long long e = base + (unsigned long long)cell * dirs + d;
    const float2 mass = V.mass[e];
    if (!(mass.y > 0.0f)) return;  // no transmittance: finished by the own pass
    const float4 raw = V.raw[e];
    const float transmittance = lux::saturate(raw.w);
    if (!(transmittance > 0.0f)) return;
    const float support = mass.x > 0.0f ? 1.0f - transmittance : 0.0f;
    MergeOwn own{0.0f, 0.0f, 0.0f, support, transmittance};
    if (support > 0.0f) {
        own.rx = raw.x;
        own.ry = raw.y;
        own.rz = raw.z;
    }
    merge_finish(V, F, level, base, dirs, cell, d, own, true);
}

__global__ void __launch_bounds__(256, LUX_MERGE_OWN_MIN_BLOCKS) merge_own_kernel(ViewDevice V, FrameParams F, HistoryDevice H) {
    if (*V.error_flags) return;
    for (uint32_t l = 0; l < F.levels; ++l) {
        const uint32_t dirs = F.dirs[l];
        const unsigned long long n = (unsigned long long)V.cell_count[l] * dirs, base = V.level_base[l];
        for (unsigned long long r = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; r < n;
             r += (unsigned long long)gridDim.x * blockDim.x)
            merge_own_record(V, F, H, l, base, dirs, r);
    }
}

__global__ void __launch_bounds__(LUX_MERGE_THREADS, LUX_MERGE_MIN_BLOCKS)
    merge_children_kernel(ViewDevice V, FrameParams F, uint32_t level) {
    if (*V.error_flags) return;
    const uint32_t dirs = F.dirs[level], cells = V.cell_count[level];
    const unsigned long long n = (unsigned long long)cells * dirs;
    const unsigned long long base = V.level_base[level];
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        uint32_t cell, d;
        merge_item(i, cells, dirs, cell, d);
        merge_children_record(V, F, level, base, dirs, cell, d);
    }
}

// The own pass that lists, level by level, the records whose merged value
// needs the children (pass_list at the level's record base, pass_count per
// level), taken in storage order as merge_own_kernel takes them; a warp
// appends its records of a round together (one atomic per warp and round).
// Levels hold fewer than 2^32 records (checked on the host).
__global__ void __launch_bounds__(256, LUX_MERGE_OWN_MIN_BLOCKS) merge_own_list_kernel(ViewDevice V, FrameParams F,
                                                                                      HistoryDevice H) {
    if (*V.error_flags) return;
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t l = 0; l < F.levels; ++l) {
        const uint32_t dirs = F.dirs[l];
        const unsigned long long n = (unsigned long long)V.cell_count[l] * dirs, base = V.level_base[l];
        for (unsigned long long r = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; r < n;
             r += (unsigned long long)gridDim.x * blockDim.x) {
            uint32_t cell, d;
            record_cell(r, dirs, cell, d);
            MergeOwn own;
            const bool children = merge_own(V, F, H, l, base, dirs, cell, d, own);
            if (!children) merge_finish(V, F, l, base, dirs, cell, d, own, false);
            const unsigned active = __activemask();
            const unsigned want = __ballot_sync(active, children);
            if (want) {
                const uint32_t leader = (uint32_t)__ffs(want) - 1u;
                uint32_t at = 0;
                if (lane == leader) at = atomicAdd(&V.pass_count[l], (uint32_t)__popc(want));
                at = __shfl_sync(active, at, leader);
                if (children) V.pass_list[base + at + (uint32_t)__popc(want & ((1u << lane) - 1u))] = (uint32_t)r;
            }
        }
    }
}

// The children pass of one level over its listed records.
__global__ void __launch_bounds__(LUX_MERGE_THREADS, LUX_MERGE_MIN_BLOCKS)
    merge_children_list_kernel(ViewDevice V, FrameParams F, uint32_t level) {
    if (*V.error_flags) return;
    const uint32_t dirs = F.dirs[level], n = V.pass_count[level];
    const unsigned long long base = V.level_base[level];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t cell, d;
        record_cell(__ldg(V.pass_list + base + i), dirs, cell, d);
        merge_children_record(V, F, level, base, dirs, cell, d);
    }
}

// packProbes, shaders/split.slang:1786-1918: one block per cascade-0 cell.
// The cascade-0 bin directions of a view (the block's shared table).
__device__ __forceinline__ void pack_directions(const FrameParams &F, float4 *dir) {
    for (uint32_t d = threadIdx.x; d < F.dirs[0]; d += blockDim.x) {
        f3 b = lux::bin_direction(d, F.columns[0], F.rows[0]);
        dir[d] = make_float4(b.x, b.y, b.z, 0.0f);
    }
}

// One cascade-0 cell's 36 texels, by the whole block (val: [dirs] shared).
__device__ __forceinline__ void pack_cell(const ViewDevice &V, const FrameParams &F, uint32_t cell, float4 *val,
                                          const float4 *dir) {
    const uint32_t dirs = F.dirs[0];
    __syncthreads();
    for (uint32_t d = threadIdx.x; d < dirs; d += blockDim.x) {
        float4 m = V.merged[V.level_base[0] + (unsigned long long)cell * dirs + d];
        bool ok = m.w > 0.0f && isfinite(m.x) && isfinite(m.y) && isfinite(m.z) && isfinite(m.w);
        val[d] = ok ? m : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    __syncthreads();
    if (threadIdx.x < 36u) {
        uint32_t texel = threadIdx.x;
        f3 normal = lux::decode_normal(((float)(texel % 6u) + 0.5f) / 6.0f, ((float)(texel / 6u) + 0.5f) / 6.0f);
        float sx = 0.0f, sy = 0.0f, sz = 0.0f, nominal = 0.0f, observed = 0.0f;
        for (uint32_t d = 0; d < dirs; ++d) {
            float4 dv = dir[d];
            float cosine = fmaxf(lux::dot(normal, f3{dv.x, dv.y, dv.z}), 0.0f);
            nominal += cosine;
            if (cosine <= 0.0f) continue;
            float4 v = val[d];
            if (v.w > 0.0f) {
                float w = cosine * lux::saturate(v.w);
                sx = sx + v.x * w;
                sy = sy + v.y * w;
                sz = sz + v.z * w;
                observed += w;
            }
        }
        float4 out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (nominal > 0.0f) {
            float scale = nominal * (4.0f / (float)dirs);
            if (observed > 0.0f)
                out = make_float4((sx / observed) * scale, (sy / observed) * scale, (sz / observed) * scale,
                                  lux::saturate(observed / nominal));
        }
        V.tables[(size_t)cell * 36 + texel] = out;
    }
}

__global__ void __launch_bounds__(64) pack_kernel(ViewDevice V, FrameParams F) {
    if (*V.error_flags) return;
    extern __shared__ float4 smem[];
    float4 *val = smem;            // [dirs]
    float4 *dir = smem + F.dirs[0]; // [dirs] xyz
    pack_directions(F, dir);
    for (uint32_t cell = blockIdx.x; cell < V.cell_count[0]; cell += gridDim.x) pack_cell(V, F, cell, val, dir);
}

// diffuseAtLod (shaders/world_resolve.slang:96-150): trilinear over the 8
// cascade-0 probes of LOD `lod` around p, each looked up with the
// octahedral weights (diffuseProbePage, :51-89); rgb and coverage.
__device__ __forceinline__ void diffuse_at_lod(const ViewDevice &V, const FrameParams &F, float4 p,
                                               const float weight[4], const uint32_t texel[4], uint32_t lod, float &lx,
                                               float &ly, float &lz, float &cov) {
    float s0 = level_spacing(F, 0, lod);
    float g[3] = {p.x / s0 - 0.5f, p.y / s0 - 0.5f, p.z / s0 - 0.5f};
    float b[3] = {floorf(g[0]), floorf(g[1]), floorf(g[2])};
    float fr[3] = {g[0] - b[0], g[1] - b[1], g[2] - b[2]};
    float sx = 0.0f, sy = 0.0f, sz = 0.0f, observed = 0.0f, potential = 0.0f;
    for (uint32_t corner = 0; corner < 8u; ++corner) {
        float ax = (corner & 1u) == 0u ? 1.0f - fr[0] : fr[0];
        float ay = ((corner >> 1) & 1u) == 0u ? 1.0f - fr[1] : fr[1];
        float az = (corner >> 2) == 0u ? 1.0f - fr[2] : fr[2];
        float w = (ax * ay) * az;
        if (!(w > 0.0f)) continue;
        potential += w;
        uint32_t cell = cell_id(V, F, 0, (int32_t)b[0] + (int32_t)(corner & 1u),
                                (int32_t)b[1] + (int32_t)((corner >> 1) & 1u), (int32_t)b[2] + (int32_t)(corner >> 2),
                                lod);
        if (cell == lux::kEmpty) continue;
        float px = 0.0f, py = 0.0f, pz = 0.0f, pobs = 0.0f;
        for (int c = 0; c < 4; ++c) {
            float bw = weight[c];
            if (!(bw > 0.0f)) continue;
            float4 s = __ldg(V.tables + (size_t)cell * 36 + texel[c]);
            if (!(s.w > 0.0f) || !(isfinite(s.x) && isfinite(s.y) && isfinite(s.z) && isfinite(s.w))) continue;
            float ww = bw * lux::saturate(s.w);
            px = px + s.x * ww;
            py = py + s.y * ww;
            pz = pz + s.z * ww;
            pobs += ww;
        }
        float qx = pobs > 0.0f ? px / pobs : 0.0f, qy = pobs > 0.0f ? py / pobs : 0.0f,
              qz = pobs > 0.0f ? pz / pobs : 0.0f;
        float support = lux::saturate(pobs);
        if (!(support > 0.0f)) continue;
        float weight_s = w * support;
        sx = sx + qx * weight_s;
        sy = sy + qy * weight_s;
        sz = sz + qz * weight_s;
        observed += weight_s;
    }
    lx = ly = lz = cov = 0.0f;
    if (potential > 0.0f) {
        cov = lux::saturate(observed / potential);
        if (observed > 0.0f) {
            lx = sx / observed;
            ly = sy / observed;
            lz = sz / observed;
        }
    }
}

// worldResolve, shaders/world_resolve.slang:96-196, :281-313.
__global__ void __launch_bounds__(128) resolve_kernel(ViewDevice V, FrameParams F, const float4 *__restrict__ pos,
                                                      const float4 *__restrict__ nrm, uint32_t count,
                                                      float4 *__restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float4 p = pos[i], n4 = nrm[i];
    f3 n3{n4.x, n4.y, n4.z};
    float dx = 0.0f, dy = 0.0f, dz = 0.0f, coverage = 0.0f;
    bool supported = false;
    if (*V.error_flags == 0u && lux::finite3(n3) && lux::dot(n3, n3) > 0.01f) {
        float l = lux::length(n3);
        f3 normal{n3.x / l, n3.y / l, n3.z / l};
        float ex, ey;
        lux::encode_normal(normal, ex, ey);
        float gx = ex * 6.0f - 0.5f, gy = ey * 6.0f - 0.5f;
        float bxf = floorf(gx), byf = floorf(gy);
        float fx = gx - bxf, fy = gy - byf;
        float cx = 1.0f - fx, cy = 1.0f - fy;
        float weight[4] = {cx * cy, fx * cy, cx * fy, fx * fy};
        int32_t ix = (int32_t)bxf, iy = (int32_t)byf;
        uint32_t texel[4] = {lux::texel_index(ix, iy), lux::texel_index(ix + 1, iy), lux::texel_index(ix, iy + 1),
                             lux::texel_index(ix + 1, iy + 1)};
        // resolveSplitDiffuse (shaders/world_resolve.slang:163-196): the LOD
        // pair of the point, then resolveLodSource (a single LOD takes high
        // coverage 1 and blend 0).
        uint32_t low, high;
        float blend;
        point_lod(F, f3{p.x, p.y, p.z}, low, high, blend);
        float lx, ly, lz, low_cov;
        diffuse_at_lod(V, F, p, weight, texel, low, lx, ly, lz, low_cov);
        float hx = 0.0f, hy = 0.0f, hz = 0.0f, high_cov = 1.0f;
        if (high != low) diffuse_at_lod(V, F, p, weight, texel, high, hx, hy, hz, high_cov);
        float low_weight = low_cov * (1.0f - blend);
        float high_weight = high_cov * blend;
        float total = low_weight + high_weight;
        coverage = lux::saturate(total);
        dx = total > 0.0f ? (lx * low_weight + hx * high_weight) / total : 0.0f;
        dy = total > 0.0f ? (ly * low_weight + hy * high_weight) / total : 0.0f;
        dz = total > 0.0f ? (lz * low_weight + hz * high_weight) / total : 0.0f;
        supported = coverage > 0.0f && isfinite(dx) && isfinite(dy) && isfinite(dz);
    }
    // rawGiSupportAlpha, shaders/common.slang:323-326.
    out[i] = make_float4(dx, dy, dz, supported ? 1.0f + 0.25f * coverage : -1.0f);
}

uint32_t next_pow2(uint64_t v) {
    uint64_t p = 64;
    while (p < v) p <<= 1;
    return (uint32_t)p;
}

// ---- batched trace stages ----------------------------------------------
// One job = one view's frame: its device state, parameters, scene and
// receivers.  Ray (and visibility-query) indices of all jobs are
// concatenated with every job's range padded to a multiple of 32, so each
// warp-sized chunk lies inside one job: the job is warp-uniform, per-view
// warp aggregation (query append, stats) works unchanged, and a warp reads
// its job's parameters as broadcasts.
struct BatchJob {
    ViewDevice V;
    FrameParams F;
    SceneView S;
    HistoryDevice H;  // the view's previous frame (F.history)
    const float4 *pos, *nrm;
    uint32_t rays;
    uint32_t pad;
};

// Largest j < n with begin[j] <= x (begin[0] = 0, non-decreasing).
__device__ __forceinline__ uint32_t find_job(const uint32_t *__restrict__ begin, uint32_t n, uint32_t x) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1u) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(begin + mid) <= x)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void flush_stats(unsigned long long *stats, unsigned long long st[7],
                                            lux::TraceCounters &cn, bool shadow) {
    st[kStatNodes] += cn.nodes;
    st[kStatTris] += cn.triangles;
    st[kStatInst] += cn.instances;
    unsigned long long extra[3] = {cn.nodes, cn.triangles, cn.instances};
    add_stats(stats, st, shadow ? extra : nullptr);
#pragma unroll
    for (int k = 0; k < 7; ++k) st[k] = 0;
    cn = lux::TraceCounters{0, 0, 0};
}

// The four trace phases over all jobs' rays and queries; each is a kernel of
// its own or one phase of trace_batch_kernel.
// A tile of `tile` rays may span jobs: the job is found per 32-ray chunk.
__device__ __forceinline__ void closest_batch_phase(const BatchJob *__restrict__ jobs,
                                                    const uint32_t *__restrict__ begin, uint32_t n, uint32_t total,
                                                    uint32_t fr, uint32_t *counter, uint32_t tile,
                                                    lux::LeafScratch *L) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t cur = lux::kEmpty;
    unsigned long long st[7] = {0, 0, 0, 0, 0, 0, 0};
    lux::TraceCounters cn{0, 0, 0};
    while (true) {
        const uint32_t first = warp_fetch(counter, tile);
        if (first >= total) break;
        for (uint32_t base = first; base < first + tile && base < total; base += 32u) {
            uint32_t j = find_job(begin, n, base);
            const BatchJob &J = jobs[j];
            if (j != cur) {
                if (cur != lux::kEmpty) flush_stats(jobs[cur].V.stats, st, cn, false);
                cur = j;
            }
            if (__shfl_sync(0xffffffffu, *J.V.error_flags, 0)) continue;  // one value for the warp
            uint32_t slot = base - __ldg(begin + j) + lane;
            SceneView S = J.S;
            closest_split_ray_warp(J.V, J.F, fr, S, J.pos, J.nrm, slot, slot < J.rays, cn, L);
            if (slot < J.rays) st[kStatInterval] += 1;
        }
    }
    if (cur != lux::kEmpty) flush_stats(jobs[cur].V.stats, st, cn, false);
}

__device__ __forceinline__ void shade_batch_phase(const BatchJob *__restrict__ jobs, const uint32_t *__restrict__ begin,
                                                  uint32_t n, uint32_t total, uint32_t fr) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < total / 32u; w += warps) {
        uint32_t base = w * 32u;
        uint32_t j = find_job(begin, n, base);
        const BatchJob &J = jobs[j];
        if (__shfl_sync(0xffffffffu, *J.V.error_flags, 0)) continue;  // one value for the warp
        lux::ShadeParams P = J.F.shade;
        P.frame = fr;
        SceneView S = J.S;
        shade_warp(J.V, J.F, P, S, base - __ldg(begin + j) + lane, J.rays);
    }
}

__device__ __forceinline__ uint32_t job_queries(const BatchJob &J) {
    return *J.V.error_flags ? 0u : min(*J.V.ts.queue_count, J.F.queue_capacity);
}

// Padded prefix of every job's visibility-query count (known only on the
// device after shading); qbegin[n] is the padded total.  One block: each
// thread sums a run of jobs, thread 0 scans the runs.
__device__ __forceinline__ void query_prefix_block(const BatchJob *__restrict__ jobs, uint32_t n,
                                                   uint32_t *__restrict__ qbegin) {
    __shared__ uint32_t run[128];
    const uint32_t t = threadIdx.x, threads = min(blockDim.x, 128u);
    const uint32_t chunk = (n + threads - 1u) / threads;
    const uint32_t lo = min(n, t * chunk), hi = min(n, lo + chunk);
    uint32_t sum = 0;
    if (t < threads)
        for (uint32_t j = lo; j < hi; ++j) sum += (job_queries(jobs[j]) + 31u) & ~31u;
    if (t < threads) run[t] = sum;
    __syncthreads();
    if (t == 0) {
        uint32_t acc = 0;
        for (uint32_t k = 0; k < threads; ++k) {
            uint32_t v = run[k];
            run[k] = acc;
            acc += v;
        }
        qbegin[n] = acc;
    }
    __syncthreads();
    if (t < threads) {
        uint32_t acc = run[t];
        for (uint32_t j = lo; j < hi; ++j) {
            qbegin[j] = acc;
            acc += (job_queries(jobs[j]) + 31u) & ~31u;
        }
    }
}

// qbegin is written on the device in the same launch when the trace stage
// is fused: it is read with coherent loads (no read-only path).
__device__ __forceinline__ uint32_t find_query_job(const uint32_t *qbegin, uint32_t n, uint32_t x) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1u) {
        uint32_t mid = (lo + hi) >> 1;
        if (qbegin[mid] <= x)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void shadow_batch_phase(const BatchJob *__restrict__ jobs, const uint32_t *qbegin,
                                                   uint32_t n, uint32_t *counter, uint32_t tile, lux::LeafScratch *L) {
    const uint32_t total = qbegin[n];
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t cur = lux::kEmpty;
    unsigned long long st[7] = {0, 0, 0, 0, 0, 0, 0};
    lux::TraceCounters cn{0, 0, 0};
    while (true) {
        const uint32_t first = warp_fetch(counter, tile);
        if (first >= total) break;
        for (uint32_t base = first; base < first + tile && base < total; base += 32u) {
            uint32_t j = find_query_job(qbegin, n, base);
            const BatchJob &J = jobs[j];
            if (j != cur) {
                if (cur != lux::kEmpty) flush_stats(jobs[cur].V.stats, st, cn, true);
                cur = j;
            }
            uint32_t i = base - qbegin[j] + lane;
            const bool valid = i < job_queries(J);
            SceneView S = J.S;
            shadow_query_warp(J.V, S, i, valid, cn, L);
            if (valid) st[kStatShadow] += 1;
        }
    }
    if (cur != lux::kEmpty) flush_stats(jobs[cur].V.stats, st, cn, true);
}

__device__ __forceinline__ void deposit_batch_phase(const BatchJob *__restrict__ jobs,
                                                    const uint32_t *__restrict__ begin, uint32_t n, uint32_t total,
                                                    uint32_t fr) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < total / 32u; w += warps) {
        uint32_t base = w * 32u;
        uint32_t j = find_job(begin, n, base);
        const BatchJob &J = jobs[j];
        if (__shfl_sync(0xffffffffu, *J.V.error_flags, 0)) continue;  // one value for the warp
        unsigned long long st[7] = {0, 0, 0, 0, 0, 0, 0};
        uint32_t ray = base - __ldg(begin + j) + lane;
        if (ray < J.rays) deposit_split_ray(J.V, J.F, fr, J.nrm, ray, st);
        add_stats(J.V.stats, st);
    }
}

__global__ void __launch_bounds__(128, LUX_BATCH_MIN_BLOCKS)
    closest_batch_kernel(const BatchJob *__restrict__ jobs, const uint32_t *__restrict__ begin, uint32_t n,
                         uint32_t total, const uint32_t *__restrict__ frame, uint32_t *counter, uint32_t tile) {
    __shared__ lux::LeafScratch scratch[4];
    closest_batch_phase(jobs, begin, n, total, *frame, counter, tile, &scratch[threadIdx.x >> 5]);
}

__global__ void __launch_bounds__(128, LUX_SHADE_MIN_BLOCKS) shade_batch_kernel(const BatchJob *__restrict__ jobs,
                                                          const uint32_t *__restrict__ begin, uint32_t n,
                                                          uint32_t total, const uint32_t *__restrict__ frame) {
    shade_batch_phase(jobs, begin, n, total, *frame);
}

__global__ void __launch_bounds__(128) query_prefix_kernel(const BatchJob *__restrict__ jobs, uint32_t n,
                                                           uint32_t *__restrict__ qbegin) {
    if (blockIdx.x == 0) query_prefix_block(jobs, n, qbegin);
}

__global__ void __launch_bounds__(128, LUX_BATCH_MIN_BLOCKS)
    shadow_batch_kernel(const BatchJob *__restrict__ jobs, const uint32_t *qbegin, uint32_t n, uint32_t *counter,
                        uint32_t tile) {
    __shared__ lux::LeafScratch scratch[4];
    shadow_batch_phase(jobs, qbegin, n, counter, tile, &scratch[threadIdx.x >> 5]);
}

__global__ void __launch_bounds__(128) deposit_batch_kernel(const BatchJob *__restrict__ jobs,
                                                            const uint32_t *__restrict__ begin, uint32_t n,
                                                            uint32_t total, const uint32_t *__restrict__ frame) {
    deposit_batch_phase(jobs, begin, n, total, *frame);
}

// ---- the trace stage as one persistent launch --------------------------------
// A cooperative launch (every block resident) runs the four phases with a
// grid barrier between them.  Every barrier wait is bounded: a block that
// waits longer than limit_ns sets the abort word, marks every job's error
// word LUX_VIEW_ERR_TIMEOUT (the first block to give up does) and returns,
// and so does every block that sees the abort word; the later passes skip
// flagged views and the next frame clears the words.  `missing` arrivals
// that never come are added to every barrier's target (a test's way to make
// a wait run out).
struct GridBarrier {
    uint32_t *arrive;  // arrivals, monotonic over the frame's barriers
    uint32_t *abort;
    unsigned long long limit_ns;
    uint32_t missing;
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t load_acquire(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ bool grid_sync(const GridBarrier &B, uint32_t index, const BatchJob *__restrict__ jobs, uint32_t n) {
    __shared__ uint32_t passed;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();  // the block's writes before its arrival
        atomicAdd(B.arrive, 1u);
        const uint32_t target = index * gridDim.x + B.missing;
        const unsigned long long t0 = global_ns();
        uint32_t ok = 1;
        while (load_acquire(B.arrive) < target) {
            if (load_acquire(B.abort)) {
                ok = 0;
                break;
            }
            if (global_ns() - t0 > B.limit_ns) {
                ok = 0;
                if (atomicExch(B.abort, 1u) == 0u)
                    for (uint32_t j = 0; j < n; ++j) atomicOr(jobs[j].V.error_flags, LUX_VIEW_ERR_TIMEOUT);
                break;
            }
            __nanosleep(256);
        }
        __threadfence();
        passed = ok;
    }
    __syncthreads();
    return passed != 0u;
}

__global__ void __launch_bounds__(128, LUX_FUSED_MIN_BLOCKS)
    trace_batch_kernel(const BatchJob *__restrict__ jobs, const uint32_t *__restrict__ begin, uint32_t n,
                       uint32_t total, const uint32_t *__restrict__ frame, uint32_t *counters,
                       uint32_t *qbegin, GridBarrier B, uint32_t tile) {
    __shared__ lux::LeafScratch scratch[4];
    lux::LeafScratch *L = &scratch[threadIdx.x >> 5];
    const uint32_t fr = *frame;
    closest_batch_phase(jobs, begin, n, total, fr, counters, tile, L);
    if (!grid_sync(B, 1, jobs, n)) return;
    shade_batch_phase(jobs, begin, n, total, fr);
    if (!grid_sync(B, 2, jobs, n)) return;
    if (blockIdx.x == 0) query_prefix_block(jobs, n, qbegin);
    if (!grid_sync(B, 3, jobs, n)) return;
    shadow_batch_phase(jobs, qbegin, n, counters + 1, tile, L);
    if (!grid_sync(B, 4, jobs, n)) return;
    deposit_batch_phase(jobs, begin, n, total, fr);
}

// ---- batched setup, merge and pack -----------------------------------------
// Every per-view pass of a frame runs once over all jobs: a job's items
// (directory slots, receivers x levels, records of a level, ...) form one
// range of a concatenated domain, padded to a multiple of 32 so each warp
// chunk lies in one job.  Row r of the domain table (rows x (n + 1) 64-bit
// exclusive prefixes) is one such domain; the host writes the rows whose
// sizes it knows, batch_layout_kernel the rows that depend on the seeded
// cell counts, with the unpadded per-job sizes beside them.
constexpr uint32_t kRowDir = 0;      // levels x directory slots (clear, assign)
constexpr uint32_t kRowSeed = 1;     // receivers x levels (insert, lookup)
constexpr uint32_t kRowRecv = 2;     // receivers (sequence sort, ordinals)
constexpr uint32_t kRowEntries = 3;  // the frame's records (clear)
constexpr uint32_t kRowCells = 4;    // + level: cells of the level (corners, pack)
constexpr uint32_t kRowRecords = kRowCells + LUX_MAX_LEVELS;  // + level: records of the level (merge)
constexpr uint32_t kRowListed = kRowRecords + LUX_MAX_LEVELS;  // + level: listed records of the level (merge)
constexpr uint32_t kBatchRows = kRowListed + LUX_MAX_LEVELS;
constexpr uint32_t kDeviceRows = kRowListed - kRowEntries;    // rows batch_layout_kernel writes

// Largest j < n with begin[j] <= x.
__device__ __forceinline__ uint32_t find_job64(const unsigned long long *__restrict__ begin, uint32_t n,
                                               unsigned long long x) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1u) {
        uint32_t mid = (lo + hi) >> 1;
        if (begin[mid] <= x)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// fn(job, item) for every item of a padded domain row, one warp chunk at a
// time (the caller bounds item by the job's own size).
template <typename Fn>
__device__ __forceinline__ void for_batch_items(const unsigned long long *__restrict__ begin, uint32_t n, Fn &&fn) {
    const unsigned long long total = begin[n];
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned long long warps = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
    for (unsigned long long w = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) >> 5; w * 32ull < total;
         w += warps) {
        const unsigned long long base = w * 32ull;
        const uint32_t j = find_job64(begin, n, base);
        fn(j, base - begin[j] + lane);
    }
}

__device__ __forceinline__ const unsigned long long *batch_row(const unsigned long long *dom, uint32_t n, uint32_t row) {
    return dom + (size_t)row * (n + 1);
}

// The directory clear, and the retain age histograms of the jobs that
// blend history.
__global__ void batch_clear_kernel(const BatchJob *__restrict__ jobs, const unsigned long long *__restrict__ dom,
                                   uint32_t n) {
    for_batch_items(batch_row(dom, n, kRowDir), n,
                    [&](uint32_t j, unsigned long long i) { clear_item(jobs[j].V, jobs[j].F, i); });
    const size_t bins = (size_t)LUX_MAX_LEVELS * kRetainBins;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)n * bins;
         i += (size_t)gridDim.x * blockDim.x) {
        const BatchJob &J = jobs[i / bins];
        if (J.F.history) J.V.retain_hist[i % bins] = 0u;
    }
}

__global__ void batch_seed_insert_kernel(const BatchJob *__restrict__ jobs, const unsigned long long *__restrict__ dom,
                                         uint32_t n) {
    for_batch_items(batch_row(dom, n, kRowSeed), n, [&](uint32_t j, unsigned long long i) {
        seed_insert_item(jobs[j].V, jobs[j].F, jobs[j].pos, i);
    });
}

__global__ void batch_seed_assign_kernel(const BatchJob *__restrict__ jobs, const unsigned long long *__restrict__ dom,
                                         uint32_t n) {
    for_batch_items(batch_row(dom, n, kRowDir), n,
                    [&](uint32_t j, unsigned long long i) { seed_assign_item(jobs[j].V, jobs[j].F, i); });
}

// Sequence keys of all jobs' receivers go to one array (job j's at the
// receiver row's offset) for the segmented sort.
__global__ void batch_seed_lookup_kernel(const BatchJob *__restrict__ jobs, const unsigned long long *__restrict__ dom,
                                         uint32_t n, unsigned long long *keys, uint32_t *vals) {
    const unsigned long long *recv = batch_row(dom, n, kRowRecv);
    for_batch_items(batch_row(dom, n, kRowSeed), n, [&](uint32_t j, unsigned long long i) {
        seed_lookup_item(jobs[j].V, jobs[j].F, jobs[j].pos, i, keys + recv[j], vals + recv[j]);
    });
}

__global__ void batch_ordinal_kernel(const BatchJob *__restrict__ jobs, const unsigned long long *__restrict__ dom,
                                     uint32_t n, const uint32_t *__restrict__ sorted) {
    const unsigned long long *recv = batch_row(dom, n, kRowRecv);
    for_batch_items(recv, n, [&](uint32_t j, unsigned long long i) {
        if (i < jobs[j].F.receivers) jobs[j].V.receiver_ordinal[sorted[recv[j] + i]] = (uint32_t)i;
    });
}

// retain over all jobs that blend history: the previous frame's cells of job
// blockIdx.y (+ k gridDim.y), each level, strided over blockIdx.x.
__global__ void batch_retain_count_kernel(const BatchJob *__restrict__ jobs, uint32_t n) {
    for (uint32_t j = blockIdx.y; j < n; j += gridDim.y) {
        const BatchJob &J = jobs[j];
        if (!J.F.history) continue;
        for (uint32_t l = 0; l < J.F.levels; ++l) {
            const uint32_t cells = min(J.H.cell_count[l], J.F.cell_capacity);
            for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += gridDim.x * blockDim.x) {
                int4 key;
                uint32_t bin = retain_bin(J.V, J.F, J.H, l, c, key);
                if (bin < kRetainBins) atomicAdd(&J.V.retain_hist[l * kRetainBins + bin], 1u);
            }
        }
    }
}

__global__ void __launch_bounds__(kRetainBins) batch_retain_limit_kernel(const BatchJob *__restrict__ jobs,
                                                                         uint32_t n) {
    for (uint32_t j = blockIdx.x; j < n; j += gridDim.x)
        if (jobs[j].F.history) retain_limit_block(jobs[j].V, jobs[j].F);
}

__global__ void batch_retain_insert_kernel(const BatchJob *__restrict__ jobs, uint32_t n) {
    for (uint32_t j = blockIdx.y; j < n; j += gridDim.y) {
        const BatchJob &J = jobs[j];
        if (!J.F.history) continue;
        for (uint32_t l = 0; l < J.F.levels; ++l) {
            const uint32_t cells = min(J.H.cell_count[l], J.F.cell_capacity);
            for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += gridDim.x * blockDim.x) {
                int4 key;
                if (retain_bin(J.V, J.F, J.H, l, c, key) < J.V.retain_limit[l]) retain_cell(J.V, J.F, J.H, l, c, key);
            }
        }
    }
}

// Every job's record layout, then the device rows: count[r][j] the job's
// unpadded size in row kRowEntries + r (zero for a job whose error word is
// set), dom's rows the padded exclusive prefixes.  One block.
__global__ void __launch_bounds__(1024) batch_layout_kernel(const BatchJob *__restrict__ jobs, uint32_t n,
                                                            unsigned long long *__restrict__ dom,
                                                            unsigned long long *__restrict__ count) {
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
        const ViewDevice &V = jobs[j].V;
        const FrameParams &F = jobs[j].F;
        layout_view(V, F);
        const bool ok = *V.error_flags == 0u;
        unsigned long long entries = 0;
        for (uint32_t l = 0; l < LUX_MAX_LEVELS; ++l) {
            const unsigned long long cells = ok && l < F.levels ? V.cell_count[l] : 0ull;
            const unsigned long long records = cells * (l < F.levels ? F.dirs[l] : 0u);
            count[(size_t)(kRowCells - kRowEntries + l) * n + j] = cells;
            count[(size_t)(kRowRecords - kRowEntries + l) * n + j] = records;
            entries += records;
        }
        count[j] = entries;
    }
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t r = threadIdx.x >> 5; r < kDeviceRows; r += blockDim.x >> 5) {
        unsigned long long *row = dom + (size_t)(kRowEntries + r) * (n + 1);
        const unsigned long long *cnt = count + (size_t)r * n;
        unsigned long long carry = 0;
        for (uint32_t c = 0; c < n; c += 32u) {
            const uint32_t j = c + lane;
            unsigned long long v = j < n ? (cnt[j] + 31ull) & ~31ull : 0ull, incl = v;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                unsigned long long t = __shfl_up_sync(0xffffffffu, incl, off);
                if (lane >= (uint32_t)off) incl += t;
            }
            if (j < n) row[j] = carry + incl - v;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) row[n] = carry;
    }
}

__global__ void batch_clear_entries_kernel(const BatchJob *__restrict__ jobs,
                                           const unsigned long long *__restrict__ dom, uint32_t n,
                                           const unsigned long long *__restrict__ count) {
    for_batch_items(batch_row(dom, n, kRowEntries), n, [&](uint32_t j, unsigned long long i) {
        if (i < count[j]) clear_entry(jobs[j].V, i);
    });
}

// Before the merge, one launch for all levels and jobs: each cell's corners
// in the next level, and with history its previous frame's id.
__global__ void batch_merge_prep_kernel(const BatchJob *__restrict__ jobs, const unsigned long long *__restrict__ dom,
                                        uint32_t n, const unsigned long long *__restrict__ count, uint32_t levels) {
    // Every job's list lengths start at zero (the listing own pass follows).
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n * LUX_MAX_LEVELS; k += gridDim.x * blockDim.x)
        jobs[k / LUX_MAX_LEVELS].V.pass_count[k % LUX_MAX_LEVELS] = 0u;
    for (uint32_t l = 0; l < levels; ++l) {
        const unsigned long long *cells = count + (size_t)(kRowCells - kRowEntries + l) * n;
        for_batch_items(batch_row(dom, n, kRowCells + l), n, [&](uint32_t j, unsigned long long c) {
            const BatchJob &J = jobs[j];
            if (c >= cells[j] || *J.V.error_flags) return;
            if (l + 1 < J.F.levels) corners_item(J.V, J.F, l, (uint32_t)c);
            if (J.F.history) history_map_item(J.V, J.F, J.H, l, (uint32_t)c);
        });
    }
}

// The two-pass merge over all jobs: the own part of every record of every
// level, then per level the records that pass light on.
__global__ void __launch_bounds__(256) batch_merge_own_kernel(const BatchJob *__restrict__ jobs,
                                                              const unsigned long long *__restrict__ dom, uint32_t n,
                                                              const unsigned long long *__restrict__ count) {
    for_batch_items(batch_row(dom, n, kRowEntries), n, [&](uint32_t j, unsigned long long e) {
        const BatchJob &J = jobs[j];
        if (e >= count[j] || *J.V.error_flags) return;
        merge_own_entry(J.V, J.F, J.H, e);
    });
}

// The listing own pass over all jobs (merge_own_list_kernel's list for each
// job's view): a warp chunk belongs to one job; lanes with records of one
// level that pass light on append them together.
__global__ void __launch_bounds__(256) batch_merge_own_list_kernel(const BatchJob *__restrict__ jobs,
                                                                   const unsigned long long *__restrict__ dom,
                                                                   uint32_t n,
                                                                   const unsigned long long *__restrict__ count) {
    const uint32_t lane = threadIdx.x & 31u;
    for_batch_items(batch_row(dom, n, kRowEntries), n, [&](uint32_t j, unsigned long long e) {
        const BatchJob &J = jobs[j];
        if (e >= count[j] || *J.V.error_flags) return;
        uint32_t level = 0;
        while (level + 1u < J.F.levels && e >= J.V.level_base[level + 1u]) ++level;
        const unsigned long long base = J.V.level_base[level];
        const uint32_t dirs = J.F.dirs[level];
        const unsigned long long r = e - base;
        uint32_t cell, d;
        record_cell(r, dirs, cell, d);
        MergeOwn own;
        if (!merge_own(J.V, J.F, J.H, level, base, dirs, cell, d, own)) {
            merge_finish(J.V, J.F, level, base, dirs, cell, d, own, false);
            return;
        }
        const unsigned group = __match_any_sync(__activemask(), level);
        const uint32_t leader = (uint32_t)__ffs(group) - 1u;
        uint32_t at = 0;
        if (lane == leader) at = atomicAdd(&J.V.pass_count[level], (uint32_t)__popc(group));
        at = __shfl_sync(group, at, leader);
        J.V.pass_list[base + at + (uint32_t)__popc(group & ((1u << lane) - 1u))] = (uint32_t)r;
    });
}

// Domain rows of the listed records: per level, the 32-padded prefix over the
// jobs of their list lengths (one warp per level).
__global__ void batch_list_prefix_kernel(const BatchJob *__restrict__ jobs, unsigned long long *__restrict__ dom,
                                         uint32_t n, uint32_t levels) {
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t l = threadIdx.x >> 5; l < levels; l += blockDim.x >> 5) {
        unsigned long long *row = dom + (size_t)(kRowListed + l) * (n + 1);
        unsigned long long carry = 0;
        for (uint32_t c = 0; c < n; c += 32u) {
            const uint32_t j = c + lane;
            unsigned long long v = 0;
            if (j < n) {
                const BatchJob &J = jobs[j];
                if (l + 1u < J.F.levels && *J.V.error_flags == 0u) v = ((unsigned long long)J.V.pass_count[l] + 31ull) & ~31ull;
            }
            unsigned long long incl = v;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const unsigned long long t = __shfl_up_sync(0xffffffffu, incl, off);
                if (lane >= (uint32_t)off) incl += t;
            }
            if (j < n) row[j] = carry + incl - v;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) row[n] = carry;
    }
}

// The children pass of one level over every job's listed records.
__global__ void __launch_bounds__(LUX_MERGE_THREADS, LUX_MERGE_MIN_BLOCKS)
    batch_merge_children_list_kernel(const BatchJob *__restrict__ jobs, const unsigned long long *__restrict__ dom,
                                     uint32_t n, uint32_t level) {
    for_batch_items(batch_row(dom, n, kRowListed + level), n, [&](uint32_t j, unsigned long long i) {
        const BatchJob &J = jobs[j];
        if (level + 1u >= J.F.levels || *J.V.error_flags || i >= J.V.pass_count[level]) return;
        const uint32_t dirs = J.F.dirs[level];
        const unsigned long long base = J.V.level_base[level];
        uint32_t cell, d;
        record_cell(__ldg(J.V.pass_list + base + i), dirs, cell, d);
        merge_children_record(J.V, J.F, level, base, dirs, cell, d);
    });
}

__global__ void __launch_bounds__(LUX_MERGE_THREADS, LUX_MERGE_MIN_BLOCKS)
    batch_merge_children_kernel(const BatchJob *__restrict__ jobs, const unsigned long long *__restrict__ dom,
                                uint32_t n, const unsigned long long *__restrict__ count, uint32_t level) {
    const unsigned long long *records = count + (size_t)(kRowRecords - kRowEntries + level) * n;
    for_batch_items(batch_row(dom, n, kRowRecords + level), n, [&](uint32_t j, unsigned long long e) {
        const BatchJob &J = jobs[j];
        if (e >= records[j] || level + 1u >= J.F.levels || *J.V.error_flags) return;
        const uint32_t dirs = J.F.dirs[level];
        uint32_t cell, d;
        merge_item(e, J.V.cell_count[level], dirs, cell, d);
        merge_children_record(J.V, J.F, level, J.V.level_base[level], dirs, cell, d);
    });
}

// One block per cascade-0 cell over all jobs; the shared direction table is
// rebuilt when the block's job changes (dynamic shared memory: 2 x the
// largest cascade-0 direction count).
__global__ void __launch_bounds__(64) batch_pack_kernel(const BatchJob *__restrict__ jobs,
                                                        const unsigned long long *__restrict__ dom, uint32_t n,
                                                        const unsigned long long *__restrict__ count,
                                                        uint32_t max_dirs) {
    extern __shared__ float4 smem[];
    float4 *val = smem, *dir = smem + max_dirs;
    const unsigned long long *begin = batch_row(dom, n, kRowCells);
    const unsigned long long *cells = count + (size_t)(kRowCells - kRowEntries) * n;
    const unsigned long long total = begin[n];
    uint32_t cur = lux::kEmpty;
    for (unsigned long long x = blockIdx.x; x < total; x += gridDim.x) {
        const uint32_t j = find_job64(begin, n, x);
        const unsigned long long c = x - begin[j];
        const BatchJob &J = jobs[j];
        if (c >= cells[j] || *J.V.error_flags) continue;
        if (j != cur) {
            __syncthreads();  // the previous job's table is no longer read
            pack_directions(J.F, dir);
            cur = j;
        }
        pack_cell(J.V, J.F, (uint32_t)c, val, dir);
    }
}

// Interval-ray hits of a Split frame as LuxHit records.
__global__ void read_hits_kernel(ViewDevice V, uint32_t count, LuxHit *__restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    f3 o, d;
    lux::Hit h;
    load_ray(V, i, o, d, h);
    LuxHit r;
    r.distance = h.t;
    r.triangle = h.tri;
    r.instance = h.inst;
    r.errors = h.errors;
    r.barycentric[0] = (1.0f - h.b1) - h.b2;
    r.barycentric[1] = h.b1;
    r.barycentric[2] = h.b2;
    r.visited = 0;
    out[i] = r;
}

// ---- learned-cache form ----------------------------------------------------
constexpr uint32_t kFallbackSlots = 1u << 17;
constexpr uint32_t kFallbackProbes = 16;
enum CacheCounter : uint32_t {
    kCntQueries = 0, kCntCandidates = 1, kCntTrain = 2, kCntCached = 3, kCntValidated = 4, kCntValidatedCells = 5,
    kCntFailedCells = 6, kCntFallbackRays = 7, kCntCount = 8
};
constexpr uint8_t kRayPlain = 0, kRayCached = 1, kRayValidated = 2;

struct CacheDevice {
    uint8_t *flags;                // per ray
    LuxCacheSample *queries;       // per ray (compacted)
    uint32_t *query_ray;           // per compacted query: ray index
    float4 *pred;                  // per compacted query
    LuxCacheSample *train;         // [train_cap]
    float4 *target;                // [train_cap]
    float4 *cell_error;            // per cascade-0 cell: sums of (cache - traced), traced, traced^2; rgb summed
    float *global_error;           // [2]: the same sums over every validated cell
    unsigned long long *fb_key;    // fallback table
    uint32_t *fb_expiry;
    uint32_t *counters;            // CacheCounter
    uint32_t cutoff, period, frame, fallback_frames, train_cap;
    float near_limit, far_t, bound;
};

__device__ __forceinline__ uint32_t cell_hash(unsigned long long key) {
    return lux::transport_hash((uint32_t)key ^ lux::transport_hash((uint32_t)(key >> 32)));
}

__device__ __forceinline__ bool fallback_active(const CacheDevice &C, unsigned long long key) {
    uint32_t h = cell_hash(key) & (kFallbackSlots - 1u);
    for (uint32_t p = 0; p < kFallbackProbes; ++p) {
        uint32_t slot = (h + p) & (kFallbackSlots - 1u);
        unsigned long long k = C.fb_key[slot];
        if (k == key) return C.fb_expiry[slot] > C.frame;
        if (k == lux::kEmptyCell) return false;
    }
    return false;
}

__device__ __forceinline__ void fallback_insert(const CacheDevice &C, unsigned long long key, uint32_t expiry) {
    uint32_t h = cell_hash(key) & (kFallbackSlots - 1u);
    for (uint32_t p = 0; p < kFallbackProbes; ++p) {
        uint32_t slot = (h + p) & (kFallbackSlots - 1u);
        unsigned long long prev = atomicCAS(&C.fb_key[slot], lux::kEmptyCell, key);
        if (prev == lux::kEmptyCell || prev == key) {
            atomicMax(&C.fb_expiry[slot], expiry);
            return;
        }
    }
}

__device__ __forceinline__ unsigned long long receiver_key(const FrameParams &F, f3 p) {
    int32_t x, y, z;
    cell_of(F, 0, p, x, y, z);
    return lux::pack_cell(x, y, z);
}

// Interval rays of the learned-cache form: full traces for validated and
// fallback cells, otherwise up to the cutoff; a truncated ray that meets
// nothing is answered by the cache at level `cutoff` (its stored distance
// is that level's interval end, so the deposit terminates there).
__global__ void __launch_bounds__(128, LUX_CLOSEST_MIN_BLOCKS)
    closest_cache_kernel(ViewDevice V, FrameParams F, SceneView S, const float4 *__restrict__ pos,
                         const float4 *__restrict__ nrm, uint32_t ray_count, CacheDevice C) {
    if (*V.error_flags) return;
    __shared__ lux::LeafScratch scratch[4];
    lux::LeafScratch *L = &scratch[threadIdx.x >> 5];
    unsigned long long st[7] = {0, 0, 0, 0, 0, 0, 0};
    lux::TraceCounters cn{0, 0, 0};
    uint32_t fallback_rays = 0;
    while (true) {
        uint32_t base = warp_fetch(&V.ts.work_counter[0]);
        if (base >= ray_count) break;
        uint32_t ray = base + (threadIdx.x & 31u);
        const bool active = ray < ray_count;
        bool validate = false, fallback = false, full = false;
        f3 dir{0.0f, 0.0f, 0.0f}, origin{0.0f, 0.0f, 0.0f};
        float4 n4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (active) {
            uint32_t i = ray / F.rays_per_receiver, k = ray % F.rays_per_receiver;
            float4 p4 = pos[i];
            n4 = nrm[i];
            f3 p{p4.x, p4.y, p4.z}, n{n4.x, n4.y, n4.z};
            unsigned long long key = receiver_key(F, p);
            validate = cell_hash(key) % C.period == C.frame % C.period;
            fallback = !validate && fallback_active(C, key);
            full = validate || fallback;
            float u, v;
            split_direction(V, F, F.shade.frame, i, k, n, dir, u, v);
            origin = lux::ray_offset(p, n, F.shade.normal_bias);
        }
        lux::Hit hit;
        lux::trace_warp<false>(S, active, origin, dir, 0.0f, full ? 1e20f : C.near_limit, hit, cn, L);
        uint8_t flag = kRayPlain;
        if (active) {
            if (!full && hit.tri == lux::kEmpty) {
                flag = kRayCached;
                hit.t = C.far_t;
            } else if (validate && hit.t > F.end[C.cutoff - 1u]) {
                flag = kRayValidated;
            }
            fallback_rays += fallback ? 1u : 0u;
            C.flags[ray] = flag;
            store_ray(V, ray, origin, dir, hit);
            st[kStatInterval] += 1;
        }
        // The cache query of every cached or validated ray, keyed by its
        // origin and direction at its receiver's normal (albedo unknown:
        // zero), appended to the compact query list one atomic per warp.
        const bool want = active && flag != kRayPlain;
        const uint32_t lane = threadIdx.x & 31u;
        const uint32_t mask = __ballot_sync(0xffffffffu, want);
        uint32_t first = 0;
        if (lane == 0 && mask) first = atomicAdd(&C.counters[kCntQueries], (uint32_t)__popc(mask));
        first = __shfl_sync(0xffffffffu, first, 0);
        if (want) {
            const uint32_t slot = first + (uint32_t)__popc(mask & ((1u << lane) - 1u));
            LuxCacheSample q;
            q.position[0] = origin.x;
            q.position[1] = origin.y;
            q.position[2] = origin.z;
            q.weight = 1.0f;
            q.direction[0] = dir.x;
            q.direction[1] = dir.y;
            q.direction[2] = dir.z;
            q.pad0 = 0.0f;
            q.normal[0] = n4.x;
            q.normal[1] = n4.y;
            q.normal[2] = n4.z;
            q.pad1 = 0.0f;
            q.albedo[0] = q.albedo[1] = q.albedo[2] = 0.0f;
            q.pad2 = 0.0f;
            C.queries[slot] = q;
            C.query_ray[slot] = ray;
        }
    }
    st[kStatNodes] = cn.nodes;
    st[kStatTris] = cn.triangles;
    st[kStatInst] = cn.instances;
    add_stats(V.stats, st);
    for (int off = 16; off > 0; off >>= 1) fallback_rays += __shfl_down_sync(0xffffffffu, fallback_rays, off);
    if ((threadIdx.x & 31u) == 0u && fallback_rays) atomicAdd(&C.counters[kCntFallbackRays], fallback_rays);
}

// Cached rays take the prediction as their hit radiance (no next-event
// samples); validated rays compare it with what they traced, per cell.
__global__ void cache_apply_kernel(ViewDevice V, FrameParams F, uint32_t ray_count, CacheDevice C) {
    uint32_t n = min(C.counters[kCntQueries], ray_count);
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        uint32_t ray = C.query_ray[q];
        float4 pr = C.pred[q];
        if (C.flags[ray] == kRayCached) {
            V.ts.ray_base[ray] = make_float4(pr.x, pr.y, pr.z, lux::as_float(0u));
            atomicAdd(&C.counters[kCntCached], 1u);
        } else {
            f3 traced;
            if (!ray_radiance(V, ray, traced)) continue;
            uint32_t cell = V.receiver_cell[ray / F.rays_per_receiver];
            if (cell == lux::kEmpty) continue;
            // Signed: the per-ray traced radiance carries next-event noise,
            // so the cell's summed difference measures the cache's bias.
            float err = (pr.x - traced.x) + (pr.y - traced.y) + (pr.z - traced.z);
            float t = traced.x + traced.y + traced.z;
            atomicAdd(&C.cell_error[cell].x, err);
            atomicAdd(&C.cell_error[cell].y, t);
            atomicAdd(&C.cell_error[cell].z, t * t);
            atomicAdd(&C.counters[kCntValidated], 1u);
        }
    }
}

__device__ __forceinline__ bool train_candidate(const ViewDevice &V, const FrameParams &F, const CacheDevice &C,
                                                uint32_t ray, f3 &radiance) {
    uint8_t flag = C.flags[ray];
    if (flag == kRayCached) return false;
    if (flag != kRayValidated) {
        uint4 h = V.ts.ray_h[ray];
        if (h.x == lux::kEmpty || V.ts.ray_o[ray].w > F.end[F.levels > 1u ? 1u : 0u]) return false;
    }
    return ray_radiance(V, ray, radiance);
}

__global__ void cache_count_kernel(ViewDevice V, FrameParams F, uint32_t ray_count, CacheDevice C) {
    uint32_t count = 0;
    for (uint32_t ray = blockIdx.x * blockDim.x + threadIdx.x; ray < ray_count; ray += gridDim.x * blockDim.x) {
        f3 r;
        count += train_candidate(V, F, C, ray, r) ? 1u : 0u;
    }
    for (int off = 16; off > 0; off >>= 1) count += __shfl_down_sync(0xffffffffu, count, off);
    if ((threadIdx.x & 31u) == 0u && count) atomicAdd(&C.counters[kCntCandidates], count);
}

// Training samples: each candidate is kept with probability cap / candidates
// (a hash of ray and frame), up to cap.
__global__ void cache_select_kernel(ViewDevice V, FrameParams F, const float4 *__restrict__ nrm, uint32_t ray_count,
                                    CacheDevice C) {
    uint32_t candidates = C.counters[kCntCandidates];
    float keep = candidates > C.train_cap ? (float)C.train_cap / (float)candidates : 1.0f;
    for (uint32_t ray = blockIdx.x * blockDim.x + threadIdx.x; ray < ray_count; ray += gridDim.x * blockDim.x) {
        f3 r;
        if (!train_candidate(V, F, C, ray, r)) continue;
        float u = (float)(lux::transport_hash(ray * 0x9E3779B9u ^ lux::transport_hash(C.frame)) >> 8) / 16777216.0f;
        if (u >= keep) continue;
        uint32_t slot = atomicAdd(&C.counters[kCntTrain], 1u);
        if (slot >= C.train_cap) continue;
        float4 o = V.ts.ray_o[ray], d = V.ts.ray_d[ray], n = nrm[ray / F.rays_per_receiver];
        LuxCacheSample s;
        s.position[0] = o.x;
        s.position[1] = o.y;
        s.position[2] = o.z;
        s.weight = 1.0f;
        s.direction[0] = d.x;
        s.direction[1] = d.y;
        s.direction[2] = d.z;
        s.pad0 = 0.0f;
        s.normal[0] = n.x;
        s.normal[1] = n.y;
        s.normal[2] = n.z;
        s.pad1 = 0.0f;
        s.albedo[0] = s.albedo[1] = s.albedo[2] = 0.0f;
        s.pad2 = 0.0f;
        C.train[slot] = s;
        C.target[slot] = make_float4(r.x, r.y, r.z, 0.0f);
    }
}

// Validated cells whose cache error exceeds the bound fall back to full
// tracing for the next frames.
__global__ void cache_fallback_kernel(ViewDevice V, FrameParams F, CacheDevice C) {
    uint32_t cells = min(V.cell_count[0], F.cell_capacity);
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += gridDim.x * blockDim.x) {
        float4 e = C.cell_error[c];
        C.cell_error[c] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (!(e.y > 0.0f) && e.x == 0.0f) continue;
        atomicAdd(&C.counters[kCntValidatedCells], 1u);
        atomicAdd(&C.global_error[0], e.x);
        atomicAdd(&C.global_error[1], e.y);
        // Fail when the bias is both large (bound x traced) and significant:
        // beyond three standard deviations of a sum of per-ray values whose
        // second moment is sum t^2.
        if (fabsf(e.x) > C.bound * e.y + 3.0f * sqrtf(e.z) + 1e-6f) {
            int4 key = V.cell_keys[c];
            fallback_insert(C, lux::pack_cell(key.x, key.y, key.z), C.frame + C.fallback_frames);
            atomicAdd(&C.counters[kCntFailedCells], 1u);
        }
    }
}

}  // namespace

constexpr int kTimingEvents = 7;

struct LuxView {
    LuxContext *ctx = nullptr;
    LuxTuning tuning{0, 0, 16, 16, 0, 0, 64, 0, 32, 0};
    bool timing = false;
    cudaEvent_t ev[kTimingEvents] = {};
    LuxViewDesc desc{};
    ViewDevice dev{};
    uint32_t dir_capacity = 0;
    void *stage_pos = nullptr, *stage_nrm = nullptr, *stage_ppos = nullptr, *stage_pnrm = nullptr, *stage_out = nullptr;
    uint32_t stage_receivers = 0, stage_points = 0;
    // lux_view_frame_host: the resolve points' upload runs on this stream
    // while the frame traces; `stage_ready` orders the resolve after it.
    cudaStream_t stage_stream = nullptr;
    cudaEvent_t stage_ready = nullptr;
    // Unbatched Split frames: retain, layout and record clearing run on this
    // stream during the closest-hit pass (`seeded` forks it after the seed,
    // `laid_out` joins it before hit shading).
    cudaStream_t setup_stream = nullptr;
    cudaEvent_t seeded = nullptr, laid_out = nullptr;
    FrameParams last{};
    bool has_frame = false;
    // World history: the other buffer set (swapped with dev's at each
    // frame start), whether it holds a usable previous frame, and the
    // invalidation boxes queued for the next frame.
    struct {
        unsigned long long *dir_keys = nullptr;
        uint32_t *dir_ids = nullptr;
        unsigned long long *level_base = nullptr;
        uint32_t *cell_count = nullptr;
        float4 *raw = nullptr;
        float2 *mass = nullptr;
        uint32_t *cell_last = nullptr;
        int4 *cell_keys = nullptr;
    } hist;
    bool hist_valid = false;
    uint32_t hist_levels = 0;
    uint32_t hist_dirs[LUX_MAX_LEVELS] = {};
    uint64_t generation = 0;  // bumped at every buffer swap (batch job tables hold pointers)
    std::vector<std::array<float, 6>> dirty;
    // Learned-cache form (lux_view_set_cache).
    LuxCacheMode cache{};
    CacheDevice cdev{};
    bool cache_alloc = false;
    // Multi-bounce (RadianceCascades::multi_bounce): the secondary cache, a
    // second view whose receivers are this view's interval-ray hits, and the
    // snapshot of its cascade-0 probes that hit shading reads one frame late.
    LuxView *secondary = nullptr;
    LuxCamera camera{};  // distance LODs (enabled = 0: LOD 0)
    struct {
        unsigned long long *keys = nullptr;
        uint32_t *ids = nullptr;
        float4 *tables = nullptr;
        float spacing = 0.0f;
        bool valid = false;
    } fb;
};

static void cache_buffers_free(LuxView *v) {
    CacheDevice &C = v->cdev;
    void *ptrs[] = {C.flags, C.queries, C.query_ray, C.pred, C.train, C.target, C.cell_error, C.global_error,
                    C.fb_key, C.fb_expiry, C.counters};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    C = CacheDevice{};
    v->cache_alloc = false;
}

// Device-wide scan scratch for the counting-sort histogram.
static size_t scan_temp_bytes() {
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)kSortBins);
    return std::max<size_t>(bytes, 16);
}

// Radix-sort scratch for ordering `receivers` sequence keys.
static size_t order_temp_bytes(uint32_t receivers) {
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const unsigned long long *)nullptr, (unsigned long long *)nullptr,
                                    (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)std::max(receivers, 1u), 0,
                                    62);
    return std::max<size_t>(bytes, 16);
}

static lux_status view_alloc(LuxView *v) {
    LuxContext *ctx = v->ctx;
    const LuxViewDesc &d = v->desc;
    ViewDevice &D = v->dev;
    v->dir_capacity = next_pow2(2ull * d.max_cells);
    size_t L = LUX_MAX_LEVELS;
    struct A {
        void **p;
        size_t bytes;
    } allocs[] = {
        {(void **)&D.dir_keys, L * v->dir_capacity * sizeof(unsigned long long)},
        {(void **)&D.dir_ids, L * v->dir_capacity * sizeof(uint32_t)},
        {(void **)&D.cell_keys, L * d.max_cells * sizeof(int4)},
        {(void **)&D.cell_count, L * sizeof(uint32_t)},
        {(void **)&D.level_base, L * sizeof(unsigned long long)},
        {(void **)&D.receiver_cell, L * (size_t)d.max_receivers * sizeof(uint32_t)},
        {(void **)&D.receiver_lod, (size_t)d.max_receivers * sizeof(uint32_t)},
        {(void **)&D.receiver_ordinal, (size_t)d.max_receivers * sizeof(uint32_t)},
        {(void **)&D.order_keys, 2 * (size_t)d.max_receivers * sizeof(unsigned long long)},
        {(void **)&D.order_vals, 2 * (size_t)d.max_receivers * sizeof(uint32_t)},
        {(void **)&D.order_temp, order_temp_bytes(d.max_receivers)},
        {(void **)&D.corner_ids, L * (size_t)d.max_cells * 8 * sizeof(uint32_t)},
        {(void **)&D.corner_frac, L * (size_t)d.max_cells * sizeof(float4)},
        {(void **)&D.accum, (size_t)d.max_entries * sizeof(float4)},
        {(void **)&D.count, (size_t)d.max_entries * sizeof(uint32_t)},
        {(void **)&D.merged, (size_t)d.max_entries * sizeof(float4)},
        {(void **)&D.raw, (size_t)d.max_entries * sizeof(float4)},
        {(void **)&D.mass, (size_t)d.max_entries * sizeof(float2)},
        {(void **)&D.pass_list, LUX_MERGE_COMPACT ? (size_t)d.max_entries * sizeof(uint32_t) : 16},
        {(void **)&D.pass_count, L * sizeof(uint32_t)},
        {(void **)&D.hist_cell, L * (size_t)d.max_cells * sizeof(uint32_t)},
        {(void **)&D.cell_last, L * (size_t)d.max_cells * sizeof(uint32_t)},
        {(void **)&v->hist.cell_last, L * (size_t)d.max_cells * sizeof(uint32_t)},
        {(void **)&v->hist.cell_keys, L * (size_t)d.max_cells * sizeof(int4)},
        {(void **)&D.retain_hist, L * kRetainBins * sizeof(uint32_t)},
        {(void **)&D.retain_limit, L * sizeof(uint32_t)},
        {(void **)&v->hist.dir_keys, L * v->dir_capacity * sizeof(unsigned long long)},
        {(void **)&v->hist.dir_ids, L * v->dir_capacity * sizeof(uint32_t)},
        {(void **)&v->hist.level_base, L * sizeof(unsigned long long)},
        {(void **)&v->hist.cell_count, L * sizeof(uint32_t)},
        {(void **)&v->hist.raw, (size_t)d.max_entries * sizeof(float4)},
        {(void **)&v->hist.mass, (size_t)d.max_entries * sizeof(float2)},
        {(void **)&D.tables, (size_t)d.max_cells * 36 * sizeof(float4)},
        {(void **)&D.error_flags, sizeof(uint32_t) * 4},
        {(void **)&D.stats, 16 * sizeof(unsigned long long)},
        {(void **)&D.ts.ray_o, (size_t)d.max_rays * sizeof(float4)},
        {(void **)&D.ts.ray_d, (size_t)d.max_rays * sizeof(float4)},
        {(void **)&D.ts.ray_h, (size_t)d.max_rays * sizeof(uint4)},
        {(void **)&D.ts.ray_base, (size_t)d.max_rays * sizeof(float4)},
        {(void **)&D.ts.ray_extra, (size_t)d.max_rays * sizeof(float4)},
        {(void **)&D.ts.query_slot, (size_t)d.max_rays * lux::kMaxNeeSamples * sizeof(uint32_t)},
        {(void **)&D.ts.slot_contrib, (size_t)d.max_rays * lux::kMaxNeeSamples * sizeof(float4)},
        {(void **)&D.ts.queue_o, (size_t)d.max_rays * lux::kMaxNeeSamples * sizeof(float4)},
        {(void **)&D.ts.queue_d, (size_t)d.max_rays * lux::kMaxNeeSamples * sizeof(float4)},
        {(void **)&D.ts.queue_result, (size_t)d.max_rays * lux::kMaxNeeSamples},
        {(void **)&D.ts.queue_count, 16},
        {(void **)&D.ts.work_counter, 16},
    };
    D.order_temp_bytes = order_temp_bytes(d.max_receivers);
    for (auto &a : allocs) {
        if (cudaMalloc(a.p, std::max<size_t>(a.bytes, 16)) != cudaSuccess) {
            cudaGetLastError();
            return lux_fail(ctx, LUX_ERR_OUT_OF_MEMORY, "view: device allocation failed");
        }
    }
    cudaMemsetAsync(D.error_flags, 0, 16, ctx->stream);
    cudaMemsetAsync(D.stats, 0, 128, ctx->stream);
    cudaMemsetAsync(D.cell_count, 0, L * 4, ctx->stream);
    return lux_cuda_check(ctx, (int)cudaGetLastError(), "view allocation");
}

// Coherence-sort buffers (keys and permutation per ray or query, the 2^24-bin
// histogram and its offsets, the scan scratch: about 8 x max_rays x 16 B +
// 128 MiB), allocated when a frame of the view first runs with sort_rays or
// sort_queries set; views that never sort do not hold them.
static lux_status ensure_sort_buffers(LuxView *v) {
    ViewDevice &D = v->dev;
    if (D.sort_hist) return LUX_OK;
    const size_t items = (size_t)v->desc.max_rays * lux::kMaxNeeSamples;
    D.scan_temp_bytes = scan_temp_bytes();
    struct A {
        void **p;
        size_t bytes;
    } allocs[] = {
        {(void **)&D.sort_keys, items * sizeof(uint32_t)},
        {(void **)&D.sort_perm, items * sizeof(uint32_t)},
        {(void **)&D.sort_offs, (size_t)kSortBins * sizeof(uint32_t)},
        {(void **)&D.scan_temp, D.scan_temp_bytes},
        {(void **)&D.sort_hist, (size_t)kSortBins * sizeof(uint32_t)},  // last: marks the set complete
    };
    for (auto &a : allocs) {
        if (*a.p) continue;
        if (cudaMalloc(a.p, std::max<size_t>(a.bytes, 16)) != cudaSuccess) {
            cudaGetLastError();
            *a.p = nullptr;
            return lux_fail(v->ctx, LUX_ERR_OUT_OF_MEMORY, "view: coherence-sort buffer allocation failed");
        }
    }
    return LUX_OK;
}

extern "C" lux_status lux_view_create(LuxContext *ctx, const LuxViewDesc *desc, LuxView **out) {
    if (!ctx || !desc || !out) return LUX_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (desc->max_receivers == 0 || desc->max_cells == 0 || desc->max_entries == 0 || desc->max_rays == 0)
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "view: capacities must be positive");
    if ((uint64_t)desc->max_rays * lux::kMaxNeeSamples > 0xffffffffull)
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "view: max_rays above 2^28");
    if (desc->max_receivers > 0x7fffffffu)  // the sample-sequence sort counts receivers in an int
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "view: max_receivers above 2^31 - 1");
    if (desc->max_cells > (1u << 30))
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "view: max_cells above 2^30");
    LuxView *v = new LuxView();
    v->ctx = ctx;
    v->desc = *desc;
    lux_status s = view_alloc(v);
    if (s != LUX_OK) {
        lux_view_destroy(v);
        return s;
    }
    *out = v;
    return LUX_OK;
}

extern "C" lux_status lux_view_destroy(LuxView *v) {
    if (!v) return LUX_OK;
    ViewDevice &D = v->dev;
    void *ptrs[] = {D.dir_keys, D.dir_ids, D.cell_keys, D.cell_count, D.level_base, D.receiver_cell, D.receiver_lod,
                    D.receiver_ordinal, D.order_keys, D.order_vals, D.order_temp,
                    D.corner_ids,
                    D.corner_frac, D.accum, D.count, D.merged, D.raw, D.mass, D.hist_cell, D.cell_last,
                    D.retain_hist, D.retain_limit, D.tables, D.error_flags, D.stats,
                    v->hist.dir_keys, v->hist.dir_ids, v->hist.level_base, v->hist.cell_count, v->hist.raw,
                    v->hist.mass, v->hist.cell_last, v->hist.cell_keys,
                    D.ts.ray_o, D.ts.ray_d, D.ts.ray_h, D.ts.ray_base, D.ts.ray_extra, D.ts.query_slot, D.ts.slot_contrib, D.ts.queue_o, D.ts.queue_d,
                    D.ts.queue_result, D.ts.queue_count, D.ts.work_counter, D.sort_keys, D.sort_perm, D.sort_hist, D.sort_offs, D.scan_temp,
                    v->stage_pos, v->stage_nrm, v->stage_ppos, v->stage_pnrm, v->stage_out};
    if (v->stage_stream) cudaStreamSynchronize(v->stage_stream);
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (v->stage_ready) cudaEventDestroy(v->stage_ready);
    if (v->stage_stream) cudaStreamDestroy(v->stage_stream);
    if (v->setup_stream) cudaStreamSynchronize(v->setup_stream);
    if (v->seeded) cudaEventDestroy(v->seeded);
    if (v->laid_out) cudaEventDestroy(v->laid_out);
    if (v->setup_stream) cudaStreamDestroy(v->setup_stream);
    for (int i = 0; i < kTimingEvents; ++i)
        if (v->ev[i]) cudaEventDestroy(v->ev[i]);
    cache_buffers_free(v);
    void *bounce[] = {D.hit_pos, D.hit_nrm, v->fb.keys, v->fb.ids, v->fb.tables};
    for (void *p : bounce)
        if (p) cudaFree(p);
    lux_view_destroy(v->secondary);
    delete v;
    return LUX_OK;
}

extern "C" lux_status lux_view_set_cache(LuxView *v, const LuxCacheMode *mode) {
    if (!v) return LUX_ERR_INVALID_ARGUMENT;
    LuxContext *ctx = v->ctx;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (!mode || !mode->cache) {
        cache_buffers_free(v);
        v->cache = LuxCacheMode{};
        return LUX_OK;
    }
    LuxCacheMode m = *mode;
    if (lux_cache_context(m.cache) != ctx)
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "set_cache: the cache belongs to another context");
    if (m.cutoff_level < 1 || m.cutoff_level >= LUX_MAX_LEVELS || m.validate_period < 1 || m.train_samples < 128 ||
        m.train_samples > (1u << 22) || !(m.error_bound > 0.0f) || m.fallback_frames < 1)
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "set_cache: mode out of range");
    cache_buffers_free(v);
    CacheDevice &C = v->cdev;
    size_t rays = v->desc.max_rays, cells = v->desc.max_cells;
    bool ok = cudaMalloc((void **)&C.flags, rays) == cudaSuccess &&
              cudaMalloc((void **)&C.queries, rays * sizeof(LuxCacheSample)) == cudaSuccess &&
              cudaMalloc((void **)&C.query_ray, rays * 4) == cudaSuccess &&
              cudaMalloc((void **)&C.pred, rays * sizeof(float4)) == cudaSuccess &&
              cudaMalloc((void **)&C.train, (size_t)m.train_samples * sizeof(LuxCacheSample)) == cudaSuccess &&
              cudaMalloc((void **)&C.target, (size_t)m.train_samples * sizeof(float4)) == cudaSuccess &&
              cudaMalloc((void **)&C.cell_error, cells * sizeof(float4)) == cudaSuccess &&
              cudaMalloc((void **)&C.global_error, 16) == cudaSuccess &&
              cudaMalloc((void **)&C.fb_key, (size_t)kFallbackSlots * 8) == cudaSuccess &&
              cudaMalloc((void **)&C.fb_expiry, (size_t)kFallbackSlots * 4) == cudaSuccess &&
              cudaMalloc((void **)&C.counters, kCntCount * 4) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        cache_buffers_free(v);
        return lux_fail(ctx, LUX_ERR_OUT_OF_MEMORY, "set_cache: device allocation failed");
    }
    cudaMemset(C.cell_error, 0, cells * sizeof(float4));
    cudaMemset(C.fb_key, 0xff, (size_t)kFallbackSlots * 8);
    cudaMemset(C.fb_expiry, 0, (size_t)kFallbackSlots * 4);
    cudaMemset(C.counters, 0, kCntCount * 4);
    v->cache_alloc = true;
    v->cache = m;
    return lux_cuda_check(ctx, (int)cudaDeviceSynchronize(), "set_cache");
}

extern "C" lux_status lux_view_cache_stats(LuxView *v, LuxCacheFrameStats *out) {
    if (!v || !out) return LUX_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof *out);
    if (!v->cache_alloc) return LUX_OK;
    lux_status rc = lux_cuda_check(v->ctx, (int)cudaStreamSynchronize(v->ctx->stream), "cache stats");
    if (rc != LUX_OK) return rc;
    uint32_t c[kCntCount];
    float g[2];
    cudaMemcpy(c, v->cdev.counters, sizeof c, cudaMemcpyDeviceToHost);
    cudaMemcpy(g, v->cdev.global_error, sizeof g, cudaMemcpyDeviceToHost);
    out->validated_bias = g[1] > 0.0f ? g[0] / g[1] : 0.0f;
    out->cached_rays = c[kCntCached];
    out->validated_rays = c[kCntValidated];
    out->train_candidates = c[kCntCandidates];
    out->trained_samples = std::min(c[kCntTrain], v->cache.train_samples);
    out->validated_cells = c[kCntValidatedCells];
    out->failed_cells = c[kCntFailedCells];
    out->fallback_rays = c[kCntFallbackRays];
    return lux_cuda_check(v->ctx, (int)cudaGetLastError(), "cache stats copy");
}

static lux_status make_params(LuxView *v, const LuxSettings *settings_in, uint32_t receivers, FrameParams &F) {
    LuxSettings s = *settings_in;
    lux_settings_sanitize(&s);
    std::memset(&F, 0, sizeof F);
    F.levels = s.levels;
    F.layout = s.layout;
    F.rays_per_receiver = s.rays_per_receiver;
    F.receivers = receivers;
    F.dir_capacity = v->dir_capacity;
    F.cell_capacity = v->desc.max_cells;
    F.ray_capacity = v->desc.max_rays;
    F.queue_capacity = v->desc.max_rays * lux::kMaxNeeSamples;
    F.entry_capacity = v->desc.max_entries;
    for (uint32_t l = 0; l < s.levels; ++l) {
        F.spacing[l] = s.probe_spacing * (float)(1u << l);
        F.end[l] = lux_interval_end(&s, l);
        F.start[l] = l == 0 ? 0.0f : lux_interval_end(&s, l - 1);
        F.columns[l] = s.base_columns << l;
        F.rows[l] = s.base_rows << l;
        F.dirs[l] = F.columns[l] * F.rows[l];
    }
    F.shade.probe_spacing = s.probe_spacing;
    F.shade.normal_bias = s.normal_bias;
    F.shade.exposure = s.exposure;
    F.shade.emissive_samples = s.emissive_samples;
    F.shade.frame = s.frame_index;
    F.shade.environment = f3{s.environment[0], s.environment[1], s.environment[2]};
    F.radiance_blend = s.temporal_blend;
    F.transmittance_blend = s.transmittance_blend;
    F.history = 0;
    F.dirty_count = 0;
    // Distance LODs: the camera terms of splitLodBlendForParameters
    // (shaders/common.slang:431-461), evaluated once per frame.
    const LuxCamera &cam = v->camera;
    if (cam.enabled && F.layout == LUX_LAYOUT_SPLIT) {
        const float *m = cam.clip_from_world;
        const float px = m[12], py = m[13], pz = m[14];
        const bool perspective = std::isfinite(px) && std::isfinite(py) && std::isfinite(pz) &&
                                 (px * px + py * py) + pz * pz > 1e-12f;
        const float focal = 0.5f * (float)cam.viewport_height * std::sqrt((m[4] * m[4] + m[5] * m[5]) + m[6] * m[6]);
        const float target = (float)(cam.target_pixels > 1u ? cam.target_pixels : 1u);
        F.lod_enabled = 1;
        F.lod_perspective = perspective ? 1u : 0u;
        for (int a = 0; a < 3; ++a) F.lod_camera[a] = cam.position[a];
        F.lod_base = std::fmax(focal * s.probe_spacing / target, s.probe_spacing);
        F.lod_ortho_scale = target / std::fmax(focal * s.probe_spacing, 1e-20f);
    }
    if ((size_t)F.dirs[0] * 2 * sizeof(float4) > 48 * 1024)
        return lux_fail(v->ctx, LUX_ERR_INVALID_ARGUMENT, "trace_merge: too many cascade-0 directions");
    return LUX_OK;
}

// seed -> layout: the receivers' cells of every level, dense ids, record
// offsets, cleared records (clear .. prefix, shaders/split.slang:734-983).
static HistoryDevice history_device(const LuxView *v) {
    return HistoryDevice{v->hist.dir_keys, v->hist.dir_ids, v->hist.level_base, v->hist.cell_count,
                         v->hist.raw,      v->hist.mass,    v->hist.cell_last, v->hist.cell_keys};
}

// seed: clear, the receivers' cells and dense ids, the sample-sequence order.
static void enqueue_seed(LuxView *v, const FrameParams &F, const float4 *pos, cudaStream_t st) {
    const ViewDevice &D = v->dev;
    const int grid = v->ctx->sm_count * 8;
    clear_kernel<<<grid, 256, 0, st>>>(D, F);
    if (F.receivers) {
        seed_insert_kernel<<<grid, 256, 0, st>>>(D, F, pos);
        seed_assign_kernel<<<grid, 256, 0, st>>>(D, F);
        seed_lookup_kernel<<<grid, 256, 0, st>>>(D, F, pos);
        if (F.layout == LUX_LAYOUT_SPLIT) {  // the receivers' places in the sample sequence
            size_t bytes = D.order_temp_bytes;
            cub::DeviceRadixSort::SortPairs(D.order_temp, bytes, D.order_keys, D.order_keys + v->desc.max_receivers,
                                            D.order_vals, D.order_vals + v->desc.max_receivers, (int)F.receivers, 0,
                                            62, st);
            ordinal_kernel<<<grid, 256, 0, st>>>(D, D.order_vals + v->desc.max_receivers, F.receivers);
        }
    }
}

// layout: retained cells, record offsets, cleared records.
static void enqueue_layout(LuxView *v, const FrameParams &F, cudaStream_t st) {
    const ViewDevice &D = v->dev;
    const int grid = v->ctx->sm_count * 8;
    if (F.history && F.layout == LUX_LAYOUT_SPLIT) {  // retain: the previous frame's unseen cells stay
        const HistoryDevice H = history_device(v);
        cudaMemsetAsync(D.retain_hist, 0, (size_t)LUX_MAX_LEVELS * kRetainBins * sizeof(uint32_t), st);
        retain_count_kernel<<<grid, 256, 0, st>>>(D, F, H);
        retain_limit_kernel<<<1, kRetainBins, 0, st>>>(D, F);
        retain_insert_kernel<<<grid, 256, 0, st>>>(D, F, H);
    }
    layout_kernel<<<1, 32, 0, st>>>(D, F);
    clear_entries_kernel<<<grid, 256, 0, st>>>(D, F);
}

static void enqueue_setup(LuxView *v, const FrameParams &F, const float4 *pos, cudaStream_t st) {
    enqueue_seed(v, F, pos, st);
    enqueue_layout(v, F, st);
}

// Corners then the merge of every level, coarsest first (mergeEntry over
// levels n-1 .. 0, shaders/split.slang:1624-1725).
static void enqueue_merge(LuxView *v, const FrameParams &F, cudaStream_t st) {
    const ViewDevice &D = v->dev;
    const int grid = v->ctx->sm_count * 8;
    const HistoryDevice H = history_device(v);
    if (F.levels > 1 || F.history) merge_prep_kernel<<<grid, 128, 0, st>>>(D, F, H);
    // Record indices in the pass list are 32-bit (a level's records).
    const bool listed = LUX_MERGE_COMPACT && F.levels > 1 && v->desc.max_entries <= 0xffffffffull;
    if (listed) {
        merge_own_list_kernel<<<grid * 2, 256, 0, st>>>(D, F, H);
        for (int l = (int)F.levels - 2; l >= 0; --l)
            merge_children_list_kernel<<<grid * 512 / LUX_MERGE_THREADS, LUX_MERGE_THREADS, 0, st>>>(D, F,
                                                                                                   (uint32_t)l);
        return;
    }
    merge_own_kernel<<<grid * 2, 256, 0, st>>>(D, F, H);
    for (int l = (int)F.levels - 2; l >= 0; --l)
        merge_children_kernel<<<grid * 512 / LUX_MERGE_THREADS, LUX_MERGE_THREADS, 0, st>>>(D, F, (uint32_t)l);
}

// Start of an unbatched frame: the last frame's records become the history
// (a pointer swap, no copy); history is used when enabled and the previous
// frame had the same cascade shape.  Queued invalidation boxes apply now.
static void begin_history(LuxView *v, FrameParams &F, const LuxSettings &s) {
    const bool enabled = s.history_frames > 0 && (s.temporal_blend > 0.0f || s.transmittance_blend > 0.0f);
    bool same_shape = v->hist_valid && v->hist_levels == F.levels;
    for (uint32_t l = 0; same_shape && l < F.levels; ++l) same_shape = v->hist_dirs[l] == F.dirs[l];
    F.history = enabled && same_shape ? 1u : 0u;
    if (enabled) {  // without history the current buffers are simply reused
        ViewDevice &D = v->dev;
        std::swap(D.dir_keys, v->hist.dir_keys);
        std::swap(D.dir_ids, v->hist.dir_ids);
        std::swap(D.level_base, v->hist.level_base);
        std::swap(D.cell_count, v->hist.cell_count);
        std::swap(D.raw, v->hist.raw);
        std::swap(D.mass, v->hist.mass);
        std::swap(D.cell_last, v->hist.cell_last);
        std::swap(D.cell_keys, v->hist.cell_keys);
        ++v->generation;
    }
    F.dirty_count = 0;
    for (size_t i = 0; i < v->dirty.size(); ++i) {
        const auto &box = v->dirty[i];
        uint32_t slot = i < (size_t)kMaxDirty ? (uint32_t)i : (uint32_t)kMaxDirty - 1u;
        for (int a = 0; a < 3; ++a) {
            F.dirty_lo[slot][a] = i < (size_t)kMaxDirty ? box[a] : std::min(F.dirty_lo[slot][a], box[a]);
            F.dirty_hi[slot][a] = i < (size_t)kMaxDirty ? box[3 + a] : std::max(F.dirty_hi[slot][a], box[3 + a]);
        }
        F.dirty_count = std::max(F.dirty_count, slot + 1u);
    }
    v->dirty.clear();
}

static void end_history(LuxView *v, const FrameParams &F) {
    v->hist_valid = true;
    v->hist_levels = F.levels;
    for (uint32_t l = 0; l < F.levels; ++l) v->hist_dirs[l] = F.dirs[l];
}

// packProbes (shaders/split.slang:1786-1918); the direction count is
// checked by make_params.
static void enqueue_pack(LuxView *v, const FrameParams &F, cudaStream_t st) {
    size_t smem = (size_t)F.dirs[0] * 2 * sizeof(float4);
    pack_kernel<<<v->ctx->sm_count * 8, 64, smem, st>>>(v->dev, F);
}

// Next-event slots of one hit: the emissive samples (max(1, n / 2)), as many
// environment samples with a non-black environment, and one per conventional
// light must fit the per-ray slot arrays.
static lux_status check_nee_slots(LuxContext *ctx, const LuxSettings *settings, const LuxScene *scene) {
    LuxSettings s = *settings;
    lux_settings_sanitize(&s);
    uint32_t emissive = s.emissive_samples / 2u < 1u ? 1u : s.emissive_samples / 2u;
    bool environment = s.environment[0] > 0.0f || s.environment[1] > 0.0f || s.environment[2] > 0.0f;
    if (emissive * (environment ? 2u : 1u) + scene->view.conventional_lights > lux::kMaxNeeSamples)
        return lux_fail(ctx, LUX_ERR_CAPACITY,
                        "trace: emissive samples / 2 (twice with a non-black environment) + conventional lights "
                        "exceed the 16 next-event slots of a hit");
    return LUX_OK;
}

// Per-frame roles of a view in a multi-bounce frame.
struct FrameRole {
    uint32_t sparse = 0;         // receivers with position.w == 0 are absent (the secondary cache)
    uint32_t skip_emission = 0;  // no first-hit emission (the secondary cache)
    uint32_t record_hits = 0;    // write the receivers' hit surfaces (the primary cache)
    bool feedback = false;       // hit shading reads the secondary snapshot
    uint32_t cached_sky = 0;     // cachedHitSky (both caches of a multi-bounce frame with cached_hit_sky)
};

static lux_status view_frame(LuxView *v, const LuxScene *scene, const LuxSettings *settings, const LuxReceivers *rc,
                             const FrameRole &role, const LuxView *fb_owner);

// The secondary view, hit buffers and probe snapshot, created with the first
// multi-bounce frame (the secondary has the primary's capacities).
static lux_status ensure_multi_bounce(LuxView *v) {
    if (v->secondary) return LUX_OK;
    LuxContext *ctx = v->ctx;
    LuxViewDesc d = v->desc;
    LuxView *sec = nullptr;
    lux_status s = lux_view_create(ctx, &d, &sec);
    if (s != LUX_OK) return s;
    ViewDevice &D = v->dev;
    bool ok = cudaMalloc((void **)&D.hit_pos, (size_t)d.max_receivers * sizeof(float4)) == cudaSuccess &&
              cudaMalloc((void **)&D.hit_nrm, (size_t)d.max_receivers * sizeof(float4)) == cudaSuccess &&
              cudaMalloc((void **)&v->fb.keys, (size_t)sec->dir_capacity * 8) == cudaSuccess &&
              cudaMalloc((void **)&v->fb.ids, (size_t)sec->dir_capacity * 4) == cudaSuccess &&
              cudaMalloc((void **)&v->fb.tables, (size_t)d.max_cells * 36 * sizeof(float4)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        lux_view_destroy(sec);
        void *ptrs[] = {D.hit_pos, D.hit_nrm, v->fb.keys, v->fb.ids, v->fb.tables};
        for (void *p : ptrs)
            if (p) cudaFree(p);
        D.hit_pos = D.hit_nrm = nullptr;
        v->fb.keys = nullptr;
        v->fb.ids = nullptr;
        v->fb.tables = nullptr;
        return lux_fail(ctx, LUX_ERR_OUT_OF_MEMORY, "multi_bounce: device allocation failed");
    }
    v->secondary = sec;
    v->fb.valid = false;
    return lux_view_set_timing(sec, v->timing ? 1u : 0u);
}

// Snapshot of the secondary cache's cascade-0 probes for the next frame's
// hit shading: the level-0 directory and the tables of its live cells.
__global__ void feedback_snapshot_kernel(ViewDevice S, uint32_t dir_capacity, unsigned long long *keys, uint32_t *ids,
                                         float4 *tables) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < dir_capacity; i += stride) {
        keys[i] = S.dir_keys[i];
        ids[i] = S.dir_ids[i];
    }
    // Tables only when the secondary frame completed (pack ran).
    const size_t n = *S.error_flags ? 0 : (size_t)S.cell_count[0] * 36;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += stride) tables[i] = S.tables[i];
}

// A multi-bounce frame (RadianceCascades::multi_bounce; the secondary
// passes of src/render.rs:9662-9752): the primary cache traces with the
// previous snapshot's bounce light and records each receiver's hit surface;
// the secondary cache (LOD + 2: spacing and intervals x4) takes those
// surfaces as receivers, leaves out first-hit emission and reads the same
// snapshot; its cascade-0 probes then become the next frame's snapshot.
extern "C" lux_status lux_view_trace_merge(LuxView *v, const LuxScene *scene, const LuxSettings *settings,
                                           const LuxReceivers *rc) {
    if (!v || !scene || !settings || !rc) return LUX_ERR_INVALID_ARGUMENT;
    LuxSettings s = *settings;
    lux_settings_sanitize(&s);
    if (!s.multi_bounce || s.layout != LUX_LAYOUT_SPLIT) return view_frame(v, scene, settings, rc, FrameRole{}, nullptr);
    lux_status st = ensure_multi_bounce(v);
    if (st != LUX_OK) return st;
    LuxContext *ctx = v->ctx;
    cudaStream_t stream = ctx->stream;
    if (rc->count > v->desc.max_receivers)
        return lux_fail(ctx, LUX_ERR_CAPACITY, "trace_merge: more receivers than the view's max_receivers");
    // Dirty boxes void the snapshot's probes for this frame (their merged
    // values depend on the whole cascade reach) and the secondary's history.
    const bool dirty = !v->dirty.empty();
    for (const auto &box : v->dirty) v->secondary->dirty.push_back(box);
    FrameRole primary;
    primary.record_hits = 1;
    primary.feedback = v->fb.valid && !dirty;
    primary.cached_sky = s.cached_hit_sky;
    cudaMemsetAsync(v->dev.hit_pos, 0, (size_t)rc->count * sizeof(float4), stream);
    st = view_frame(v, scene, settings, rc, primary, v);
    if (st != LUX_OK) return st;
    LuxView *sec = v->secondary;
    LuxTuning t = v->tuning;
    t.closest_mode = 0;
    sec->tuning = t;
    LuxSettings s2 = s;
    s2.multi_bounce = 0;
    s2.probe_spacing = s.probe_spacing * 4.0f;
    s2.interval_length = s.interval_length * 4.0f;
    LuxReceivers hits{(const float *)v->dev.hit_pos, (const float *)v->dev.hit_nrm, rc->count};
    FrameRole secondary;
    secondary.sparse = 1;
    secondary.skip_emission = 1;
    secondary.feedback = primary.feedback;
    secondary.cached_sky = primary.cached_sky;
    st = view_frame(sec, scene, &s2, &hits, secondary, v);
    if (st != LUX_OK) return st;
    feedback_snapshot_kernel<<<ctx->sm_count * 4, 256, 0, stream>>>(sec->dev, sec->dir_capacity, v->fb.keys,
                                                                     v->fb.ids, v->fb.tables);
    v->fb.spacing = s2.probe_spacing;
    v->fb.valid = true;
    return lux_cuda_check(ctx, (int)cudaGetLastError(), "multi_bounce launch");
}

extern "C" lux_status lux_view_set_camera(LuxView *v, const LuxCamera *camera) {
    if (!v) return LUX_ERR_INVALID_ARGUMENT;
    if (!camera || !camera->enabled) {
        v->camera = LuxCamera{};
        return LUX_OK;
    }
    for (int i = 0; i < 16; ++i)
        if (!std::isfinite(camera->clip_from_world[i]))
            return lux_fail(v->ctx, LUX_ERR_INVALID_ARGUMENT, "set_camera: clip_from_world must be finite");
    for (int a = 0; a < 3; ++a)
        if (!std::isfinite(camera->position[a]))
            return lux_fail(v->ctx, LUX_ERR_INVALID_ARGUMENT, "set_camera: position must be finite");
    if (camera->viewport_height == 0)
        return lux_fail(v->ctx, LUX_ERR_INVALID_ARGUMENT, "set_camera: viewport_height must be positive");
    v->camera = *camera;
    return LUX_OK;
}

extern "C" lux_status lux_view_secondary(LuxView *v, LuxView **secondary) {
    if (!v || !secondary) return LUX_ERR_INVALID_ARGUMENT;
    *secondary = v->secondary;
    return LUX_OK;
}

static lux_status view_frame(LuxView *v, const LuxScene *scene, const LuxSettings *settings, const LuxReceivers *rc,
                             const FrameRole &role, const LuxView *fb_owner) {
    LuxContext *ctx = v->ctx;
    lux_status slots = check_nee_slots(ctx, settings, scene);
    if (slots != LUX_OK) return slots;
    if (rc->count > v->desc.max_receivers)
        return lux_fail(ctx, LUX_ERR_CAPACITY, "trace_merge: more receivers than the view's max_receivers");
    if (rc->count && (!rc->position || (!rc->normal && settings->layout == LUX_LAYOUT_SPLIT)))
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "trace_merge: missing receiver buffers");
    FrameParams F;
    lux_status ps = make_params(v, settings, rc->count, F);
    if (ps != LUX_OK) return ps;
    if (v->cache_alloc && v->cache.cutoff_level < F.levels) {
        // Learned-cache frames: LOD 0, and no level past the cutoff: every
        // ray's light from beyond the cutoff (the cache's answer, or the
        // traced hit of a validated or fallback ray) ends at level `cutoff`,
        // which then takes the whole tail like a last level.
        F.lod_enabled = 0;
        F.levels = v->cache.cutoff_level + 1u;
    }
    if (F.layout == LUX_LAYOUT_SPLIT && (uint64_t)rc->count * F.rays_per_receiver > v->desc.max_rays)
        return lux_fail(ctx, LUX_ERR_CAPACITY, "trace_merge: receivers x rays_per_receiver exceeds max_rays");
    if (F.layout == LUX_LAYOUT_SPLIT && (v->tuning.sort_rays || v->tuning.sort_queries)) {
        lux_status sb = ensure_sort_buffers(v);  // before any work of the frame is queued
        if (sb != LUX_OK) return sb;
    }
    const ViewDevice &D = v->dev;
    cudaStream_t st = ctx->stream;
    const float4 *pos = (const float4 *)rc->position;
    const float4 *nrm = (const float4 *)rc->normal;
    auto mark = [&](int i) {
        if (v->timing) cudaEventRecord(v->ev[i], st);
    };
    LuxSettings sanitized = *settings;
    lux_settings_sanitize(&sanitized);
    begin_history(v, F, sanitized);
    F.sparse = role.sparse;
    F.record_hits = role.record_hits;
    F.shade.skip_emission = role.skip_emission;
    F.shade.cached_sky = role.cached_sky;
    if (role.feedback && fb_owner) {
        F.shade.feedback = 1;
        F.shade.fb = lux::Feedback{fb_owner->fb.keys, fb_owner->fb.ids, fb_owner->fb.tables,
                                   fb_owner->secondary->dir_capacity, fb_owner->fb.spacing};
    }
    mark(0);
    const bool cached_frame = v->cache_alloc && v->cache.cutoff_level < F.levels;
    // The closest-hit pass needs only the seed (cells, sequence order), so the
    // rest of the setup runs beside it on the setup stream.
    bool forked = false;
    if (F.layout == LUX_LAYOUT_SPLIT && rc->count && !cached_frame) {
        if (!v->setup_stream &&
            (cudaStreamCreateWithFlags(&v->setup_stream, cudaStreamNonBlocking) != cudaSuccess ||
             cudaEventCreateWithFlags(&v->seeded, cudaEventDisableTiming) != cudaSuccess ||
             cudaEventCreateWithFlags(&v->laid_out, cudaEventDisableTiming) != cudaSuccess)) {
            cudaGetLastError();
            return lux_fail(ctx, LUX_ERR_CUDA, "trace_merge: setup stream creation failed");
        }
        enqueue_seed(v, F, pos, st);
        cudaEventRecord(v->seeded, st);
        cudaStreamWaitEvent(v->setup_stream, v->seeded, 0);
        enqueue_layout(v, F, v->setup_stream);
        cudaEventRecord(v->laid_out, v->setup_stream);
        forked = true;
    } else {
        enqueue_setup(v, F, pos, st);
    }
    mark(1);
    if (F.layout == LUX_LAYOUT_SPLIT) {
        uint32_t rays = rc->count * F.rays_per_receiver;
        if (rays) {
            const LuxTuning &T = v->tuning;
            ViewDevice Dr = D;  // ray pass view: optional coherence order of interval rays
            Dr.sort_keys = nullptr;
            if (T.sort_rays) {
                cudaMemsetAsync(D.sort_hist, 0, (size_t)kRaySortBins * 4, st);
                ray_keys_kernel<<<ctx->sm_count * 8, 256, 0, st>>>(D, F, scene->view, pos, nrm, rays);
                sort_hist_kernel<<<ctx->sm_count * 8, 256, 0, st>>>(D, nullptr, rays);
                enqueue_sort_scan(D, kRaySortBins, st);
                sort_scatter_kernel<<<ctx->sm_count * 8, 256, 0, st>>>(D, nullptr, rays);
                Dr.ray_order = D.sort_perm;
            }
            const bool cached = v->cache_alloc && v->cache.cutoff_level < F.levels;
            CacheDevice C = v->cdev;
            if (cached) {
                C.cutoff = v->cache.cutoff_level;
                C.period = v->cache.validate_period;
                C.frame = F.shade.frame;
                C.fallback_frames = v->cache.fallback_frames;
                C.train_cap = v->cache.train_samples;
                C.near_limit = nextafterf(F.end[C.cutoff - 1u], INFINITY);
                C.far_t = F.end[C.cutoff];
                C.bound = v->cache.error_bound;
                cudaMemsetAsync(C.counters, 0, kCntCount * 4, st);
                cudaMemsetAsync(C.global_error, 0, 8, st);
                closest_cache_kernel<<<ctx->sm_count * T.closest_blocks_per_sm, 128, 0, st>>>(D, F, scene->view, pos,
                                                                                             nrm, rays, C);
            } else if (T.closest_mode == 1)
                closest_split_refill_kernel<<<ctx->sm_count * T.closest_blocks_per_sm, 128, 0, st>>>(
                    Dr, F, scene->view, pos, nrm, rays);
            else if (T.stack_depth == 32)
                closest_split_kernel<32><<<ctx->sm_count * T.closest_blocks_per_sm, 128, 0, st>>>(
                    Dr, F, scene->view, pos, nrm, rays, tile_of(T));
            else
                closest_split_kernel<64><<<ctx->sm_count * T.closest_blocks_per_sm, 128, 0, st>>>(
                    Dr, F, scene->view, pos, nrm, rays, tile_of(T));
            if (forked) cudaStreamWaitEvent(st, v->laid_out, 0);  // join the setup stream
            ViewDevice Dq = D;  // query pass view: keys written by shade, optional order
            if (!T.sort_queries) Dq.sort_keys = nullptr;
            shade_kernel<<<(rays + 127) / 128, 128, 0, st>>>(Dq, F, scene->view, rays, false);
            if (T.sort_queries) {
                cudaMemsetAsync(D.sort_hist, 0, (size_t)kSortBins * 4, st);
                sort_hist_kernel<<<ctx->sm_count * 8, 256, 0, st>>>(D, D.ts.queue_count, F.queue_capacity);
                enqueue_sort_scan(D, kSortBins, st);
                sort_scatter_kernel<<<ctx->sm_count * 8, 256, 0, st>>>(D, D.ts.queue_count, F.queue_capacity);
                Dq.query_order = D.sort_perm;
            }
            if (T.shadow_mode == 1)
                shadow_refill_kernel<<<ctx->sm_count * T.shadow_blocks_per_sm, 128, 0, st>>>(Dq, F, scene->view);
            else if (T.stack_depth == 32)
                shadow_kernel<32><<<ctx->sm_count * T.shadow_blocks_per_sm, 128, 0, st>>>(Dq, F, scene->view,
                                                                                         tile_of(T));
            else
                shadow_kernel<64><<<ctx->sm_count * T.shadow_blocks_per_sm, 128, 0, st>>>(Dq, F, scene->view,
                                                                                         tile_of(T));
            if (cached) {
                const int g = ctx->sm_count * 8;
                lux_status qrc = lux_cache_query_device_count(v->cache.cache, C.queries, C.counters + kCntQueries, rays,
                                                              (float *)C.pred);
                if (qrc != LUX_OK) return qrc;
                cache_apply_kernel<<<g, 256, 0, st>>>(D, F, rays, C);
            }
            deposit_split_kernel<<<(rays + 127) / 128, 128, 0, st>>>(D, F, nrm, rays);
            if (cached) {
                const int g = ctx->sm_count * 8;
                cache_count_kernel<<<g, 256, 0, st>>>(D, F, rays, C);
                cudaMemsetAsync(C.train, 0, (size_t)C.train_cap * sizeof(LuxCacheSample), st);
                cache_select_kernel<<<g, 256, 0, st>>>(D, F, nrm, rays, C);
                lux_status trc = lux_cache_train(v->cache.cache, C.train, (const float *)C.target, C.train_cap);
                if (trc != LUX_OK) return trc;
                cache_fallback_kernel<<<g, 256, 0, st>>>(D, F, C);
            }
        }
    } else {
        for (uint32_t l = 0; l < F.levels; ++l)
            closest_dense_kernel<<<ctx->sm_count * 16, 128, 0, st>>>(D, F, scene->view, l);
        shade_kernel<<<ctx->sm_count * 16, 128, 0, st>>>(D, F, scene->view, F.ray_capacity, true);
        shadow_kernel<64><<<ctx->sm_count * v->tuning.shadow_blocks_per_sm, 128, 0, st>>>(D, F, scene->view,
                                                                                      tile_of(v->tuning));
        deposit_dense_kernel<<<ctx->sm_count * 16, 128, 0, st>>>(D, F);
    }
    mark(2);
    enqueue_merge(v, F, st);
    mark(3);
    enqueue_pack(v, F, st);
    mark(4);
    end_history(v, F);
    v->last = F;
    v->has_frame = true;
    return lux_cuda_check(ctx, (int)cudaGetLastError(), "trace_merge launch");
}

extern "C" lux_status lux_view_reset_history(LuxView *v) {
    if (!v) return LUX_ERR_INVALID_ARGUMENT;
    v->hist_valid = false;
    v->dirty.clear();
    v->fb.valid = false;
    if (v->secondary) lux_view_reset_history(v->secondary);
    return LUX_OK;
}

extern "C" lux_status lux_view_invalidate_bounds(LuxView *v, const float lo[3], const float hi[3]) {
    if (!v || !lo || !hi) return LUX_ERR_INVALID_ARGUMENT;
    std::array<float, 6> box;
    for (int a = 0; a < 3; ++a) {
        if (!std::isfinite(lo[a]) || !std::isfinite(hi[a]) || lo[a] > hi[a])
            return lux_fail(v->ctx, LUX_ERR_INVALID_ARGUMENT, "invalidate_bounds: need finite lo <= hi");
        box[a] = lo[a];
        box[3 + a] = hi[a];
    }
    v->dirty.push_back(box);
    return LUX_OK;
}

extern "C" lux_status lux_view_resolve(LuxView *v, const LuxSettings *settings, const float *ppos, const float *pnrm,
                                       uint32_t count, float *out) {
    if (!v || !settings || (count && (!ppos || !pnrm || !out))) return LUX_ERR_INVALID_ARGUMENT;
    if (!v->has_frame) return lux_fail(v->ctx, LUX_ERR_INVALID_ARGUMENT, "resolve: no frame traced yet");
    if (count == 0) return LUX_OK;
    if (v->timing) cudaEventRecord(v->ev[5], v->ctx->stream);
    resolve_kernel<<<(count + 127) / 128, 128, 0, v->ctx->stream>>>(v->dev, v->last, (const float4 *)ppos,
                                                                      (const float4 *)pnrm, count, (float4 *)out);
    if (v->timing) cudaEventRecord(v->ev[6], v->ctx->stream);
    return lux_cuda_check(v->ctx, (int)cudaGetLastError(), "resolve launch");
}

static lux_status ensure_stage(LuxView *v, uint32_t receivers, uint32_t points) {
    if (!v->stage_stream) {
        if (cudaStreamCreateWithFlags(&v->stage_stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&v->stage_ready, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return lux_fail(v->ctx, LUX_ERR_CUDA, "frame_host: staging stream creation failed");
        }
    }
    if (receivers > v->stage_receivers) {
        cudaFree(v->stage_pos);
        cudaFree(v->stage_nrm);
        v->stage_pos = v->stage_nrm = nullptr;
        if (cudaMalloc(&v->stage_pos, (size_t)receivers * 16) != cudaSuccess ||
            cudaMalloc(&v->stage_nrm, (size_t)receivers * 16) != cudaSuccess) {
            cudaGetLastError();
            v->stage_receivers = 0;
            return lux_fail(v->ctx, LUX_ERR_OUT_OF_MEMORY, "frame_host: staging allocation failed");
        }
        v->stage_receivers = receivers;
    }
    if (points > v->stage_points) {
        cudaFree(v->stage_ppos);
        cudaFree(v->stage_pnrm);
        cudaFree(v->stage_out);
        v->stage_ppos = v->stage_pnrm = v->stage_out = nullptr;
        if (cudaMalloc(&v->stage_ppos, (size_t)points * 16) != cudaSuccess ||
            cudaMalloc(&v->stage_pnrm, (size_t)points * 16) != cudaSuccess ||
            cudaMalloc(&v->stage_out, (size_t)points * 16) != cudaSuccess) {
            cudaGetLastError();
            v->stage_points = 0;
            return lux_fail(v->ctx, LUX_ERR_OUT_OF_MEMORY, "frame_host: staging allocation failed");
        }
        v->stage_points = points;
    }
    return LUX_OK;
}

extern "C" lux_status lux_view_frame_host(LuxView *v, const LuxScene *scene, const LuxSettings *settings,
                                          const float *rpos, const float *rnrm, uint32_t receivers, const float *ppos,
                                          const float *pnrm, uint32_t points, float *out) {
    if (!v || !scene || !settings || (receivers && (!rpos || !rnrm)) || (points && (!ppos || !pnrm || !out)))
        return LUX_ERR_INVALID_ARGUMENT;
    cudaSetDevice(v->ctx->device);
    lux_status s = ensure_stage(v, receivers, points);
    if (s != LUX_OK) return s;
    cudaStream_t st = v->ctx->stream;
    // The receivers go first on the frame's stream; the resolve points (the
    // larger upload) follow on the staging stream and overlap the trace.
    // The previous call ended with a synchronize, so no resolve still reads
    // the staging buffers.
    cudaMemcpyAsync(v->stage_pos, rpos, (size_t)receivers * 16, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(v->stage_nrm, rnrm, (size_t)receivers * 16, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(v->stage_ppos, ppos, (size_t)points * 16, cudaMemcpyHostToDevice, v->stage_stream);
    cudaMemcpyAsync(v->stage_pnrm, pnrm, (size_t)points * 16, cudaMemcpyHostToDevice, v->stage_stream);
    cudaEventRecord(v->stage_ready, v->stage_stream);
    LuxReceivers rc{(const float *)v->stage_pos, (const float *)v->stage_nrm, receivers};
    s = lux_view_trace_merge(v, scene, settings, &rc);
    if (s != LUX_OK) {
        cudaStreamSynchronize(v->stage_stream);
        return s;
    }
    cudaStreamWaitEvent(st, v->stage_ready, 0);
    s = lux_view_resolve(v, settings, (const float *)v->stage_ppos, (const float *)v->stage_pnrm, points,
                         (float *)v->stage_out);
    if (s != LUX_OK) return s;
    cudaMemcpyAsync(out, v->stage_out, (size_t)points * 16, cudaMemcpyDeviceToHost, st);
    s = lux_cuda_check(v->ctx, (int)cudaStreamSynchronize(st), "frame_host");
    if (s != LUX_OK) return s;
    uint32_t flags = 0;
    cudaMemcpy(&flags, v->dev.error_flags, 4, cudaMemcpyDeviceToHost);
    if (flags) return lux_fail(v->ctx, LUX_ERR_CAPACITY, "frame_host: view capacity exceeded (see lux_view_stats)");
    return LUX_OK;
}

extern "C" lux_status lux_view_stats(LuxView *v, LuxStats *out) {
    if (!v || !out) return LUX_ERR_INVALID_ARGUMENT;
    cudaStream_t st = v->ctx->stream;
    lux_status s = lux_cuda_check(v->ctx, (int)cudaStreamSynchronize(st), "stats");
    if (s != LUX_OK) return s;
    unsigned long long stats[16];
    uint32_t counts[LUX_MAX_LEVELS];
    uint32_t flags = 0;
    cudaMemcpy(stats, v->dev.stats, sizeof stats, cudaMemcpyDeviceToHost);
    cudaMemcpy(counts, v->dev.cell_count, sizeof counts, cudaMemcpyDeviceToHost);
    cudaMemcpy(&flags, v->dev.error_flags, 4, cudaMemcpyDeviceToHost);
    std::memset(out, 0, sizeof *out);
    out->interval_rays = stats[kStatInterval];
    out->shadow_rays = stats[kStatShadow];
    out->nodes_visited = stats[kStatNodes];
    out->triangles_tested = stats[kStatTris];
    out->instances_visited = stats[kStatInst];
    out->deposits = stats[kStatDeposits];
    out->unsupported = stats[kStatUnsupported];
    out->shadow_nodes = stats[kStatShadowNodes];
    out->shadow_triangles = stats[kStatShadowTris];
    out->shadow_instances = stats[kStatShadowInst];
    out->levels = v->last.levels;
    for (uint32_t l = 0; l < v->last.levels; ++l) {
        out->cells[l] = counts[l];
        out->entries[l] = (uint64_t)counts[l] * v->last.dirs[l];
    }
    out->error_flags = flags;
    return lux_cuda_check(v->ctx, (int)cudaGetLastError(), "stats copy");
}

extern "C" lux_status lux_view_read_level(LuxView *v, uint32_t level, int32_t *keys, float *merged, float *raw,
                                          uint32_t *samples) {
    if (!v) return LUX_ERR_INVALID_ARGUMENT;
    if (!v->has_frame || level >= v->last.levels) return lux_fail(v->ctx, LUX_ERR_INVALID_ARGUMENT, "read_level: bad level");
    cudaStreamSynchronize(v->ctx->stream);
    uint32_t counts[LUX_MAX_LEVELS];
    unsigned long long bases[LUX_MAX_LEVELS];
    cudaMemcpy(counts, v->dev.cell_count, sizeof counts, cudaMemcpyDeviceToHost);
    cudaMemcpy(bases, v->dev.level_base, sizeof bases, cudaMemcpyDeviceToHost);
    uint32_t cells = counts[level];
    size_t entries = (size_t)cells * v->last.dirs[level];
    if (keys) cudaMemcpy(keys, v->dev.cell_keys + (size_t)level * v->desc.max_cells, (size_t)cells * 16, cudaMemcpyDeviceToHost);
    if (merged) cudaMemcpy(merged, v->dev.merged + bases[level], entries * 16, cudaMemcpyDeviceToHost);
    if (raw) cudaMemcpy(raw, v->dev.raw + bases[level], entries * 16, cudaMemcpyDeviceToHost);
    if (samples) cudaMemcpy(samples, v->dev.count + bases[level], entries * 4, cudaMemcpyDeviceToHost);
    return lux_cuda_check(v->ctx, (int)cudaGetLastError(), "read_level");
}

extern "C" lux_status lux_view_read_probes(LuxView *v, int32_t *keys, float *tables) {
    if (!v) return LUX_ERR_INVALID_ARGUMENT;
    if (!v->has_frame) return lux_fail(v->ctx, LUX_ERR_INVALID_ARGUMENT, "read_probes: no frame");
    cudaStreamSynchronize(v->ctx->stream);
    uint32_t cells = 0;
    cudaMemcpy(&cells, v->dev.cell_count, 4, cudaMemcpyDeviceToHost);
    if (keys) cudaMemcpy(keys, v->dev.cell_keys, (size_t)cells * 16, cudaMemcpyDeviceToHost);
    if (tables) cudaMemcpy(tables, v->dev.tables, (size_t)cells * 36 * 16, cudaMemcpyDeviceToHost);
    return lux_cuda_check(v->ctx, (int)cudaGetLastError(), "read_probes");
}

extern "C" lux_status lux_view_set_timing(LuxView *v, uint32_t enable) {
    if (!v) return LUX_ERR_INVALID_ARGUMENT;
    if (enable && !v->ev[0]) {
        for (int i = 0; i < kTimingEvents; ++i)
            if (cudaEventCreate(&v->ev[i]) != cudaSuccess)
                return lux_cuda_check(v->ctx, (int)cudaGetLastError(), "timing events");
    }
    v->timing = enable != 0;
    return v->secondary ? lux_view_set_timing(v->secondary, enable) : LUX_OK;
}

// Per-stage device times of the last frame in milliseconds (the reference's
// per-pass timestamp spans, src/render.rs:9323-9333): seed, trace, merge,
// pack, resolve.
extern "C" lux_status lux_view_timings(LuxView *v, LuxTimings *out) {
    if (!v || !out) return LUX_ERR_INVALID_ARGUMENT;
    if (!v->timing) return lux_fail(v->ctx, LUX_ERR_INVALID_ARGUMENT, "timings: timing is disabled");
    lux_status s = lux_cuda_check(v->ctx, (int)cudaStreamSynchronize(v->ctx->stream), "timings");
    if (s != LUX_OK) return s;
    float ms[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; ++i) cudaEventElapsedTime(&ms[i], v->ev[i], v->ev[i + 1]);
    cudaEventElapsedTime(&ms[4], v->ev[5], v->ev[6]);
    cudaGetLastError();
    out->seed_ms = ms[0];
    out->trace_ms = ms[1];
    out->merge_ms = ms[2];
    out->pack_ms = ms[3];
    out->resolve_ms = ms[4];
    return LUX_OK;
}

static bool tile_valid(uint32_t tile) { return tile == 0 || tile == 32 || tile == 64 || tile == 128 || tile == 256; }

extern "C" lux_status lux_view_set_tuning(LuxView *v, const LuxTuning *t) {
    if (!v || !t) return LUX_ERR_INVALID_ARGUMENT;
    if (t->closest_mode > 1 || t->shadow_mode > 1 || t->closest_blocks_per_sm < 1 || t->closest_blocks_per_sm > 64 ||
        t->shadow_blocks_per_sm < 1 || t->shadow_blocks_per_sm > 64 || t->sort_queries > 1 || t->sort_rays > 1 ||
        (t->stack_depth != 0 && t->stack_depth != 32 && t->stack_depth != 64) || !tile_valid(t->tile_rays) ||
        t->fused_trace > 1)
        return lux_fail(v->ctx, LUX_ERR_INVALID_ARGUMENT, "set_tuning: value out of range");
    v->tuning = *t;
    if (t->sort_queries || t->sort_rays) return ensure_sort_buffers(v);
    return LUX_OK;
}

extern "C" lux_status lux_view_get_tuning(const LuxView *v, LuxTuning *t) {
    if (!v || !t) return LUX_ERR_INVALID_ARGUMENT;
    *t = v->tuning;
    return LUX_OK;
}

// ---------------------------------------------------------------------------
// Interval radiance of caller rays: traceTransport's closest hit followed by
// finishTransportVariant's outgoing radiance (shaders/split.slang:1122-1216,
// shaders/cascades.slang:196-268) without the deposit.  Uses the same
// wavefront kernels as a view's trace stage on trace scratch of the context.
// ---------------------------------------------------------------------------
namespace {

__global__ void scratch_clear_kernel(ViewDevice V) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        *V.error_flags = 0;
        *V.ts.queue_count = 0;
        V.ts.work_counter[0] = 0;
        V.ts.work_counter[1] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x < 16) V.stats[threadIdx.x] = 0;
}

__global__ void __launch_bounds__(128, LUX_CLOSEST_MIN_BLOCKS) closest_rays_kernel(ViewDevice V, SceneView S, const LuxRay *__restrict__ rays,
                                                           uint32_t count) {
    unsigned long long st[7] = {0, 0, 0, 0, 0, 0, 0};
    lux::TraceCounters cn{0, 0, 0};
    while (true) {
        uint32_t base = warp_fetch(&V.ts.work_counter[0]);
        if (base >= count) break;
        uint32_t i = base + (threadIdx.x & 31u);
        if (i < count) {
            LuxRay r = rays[i];
            f3 o{r.origin[0], r.origin[1], r.origin[2]}, d{r.direction[0], r.direction[1], r.direction[2]};
            lux::Hit hit;
            lux::trace<false>(S, o, d, r.tmin, r.limit, hit, cn);
            store_ray(V, i, o, d, hit);
            st[kStatInterval] += 1;
        }
    }
    st[kStatNodes] = cn.nodes;
    st[kStatTris] = cn.triangles;
    st[kStatInst] = cn.instances;
    add_stats(V.stats, st);
}

// out[i] = (radiance rgb, hit distance) or (0, 0, 0, -1) when unsupported.
__global__ void radiance_out_kernel(ViewDevice V, uint32_t count, float4 *__restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    f3 radiance;
    if (ray_radiance(V, i, radiance))
        out[i] = make_float4(radiance.x, radiance.y, radiance.z, V.ts.ray_o[i].w);
    else
        out[i] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
}

lux_status launch_interval_radiance(LuxContext *ctx, const LuxScene *scene, const LuxSettings *settings_in,
                                    const LuxRay *rays, uint32_t count, float *out, const ViewDevice &V,
                                    uint32_t capacity) {
    lux_status slots = check_nee_slots(ctx, settings_in, scene);
    if (slots != LUX_OK) return slots;
    LuxSettings s = *settings_in;
    lux_settings_sanitize(&s);
    FrameParams F;
    std::memset(&F, 0, sizeof F);
    F.ray_capacity = capacity;
    F.queue_capacity = capacity * lux::kMaxNeeSamples;
    F.shade.probe_spacing = s.probe_spacing;
    F.shade.normal_bias = s.normal_bias;
    F.shade.exposure = s.exposure;
    F.shade.emissive_samples = s.emissive_samples;
    F.shade.frame = s.frame_index;
    F.shade.environment = f3{s.environment[0], s.environment[1], s.environment[2]};
    cudaStream_t st = ctx->stream;
    scratch_clear_kernel<<<1, 32, 0, st>>>(V);
    if (count) {
        closest_rays_kernel<<<ctx->sm_count * 16, 128, 0, st>>>(V, scene->view, rays, count);
        shade_kernel<<<(count + 127) / 128, 128, 0, st>>>(V, F, scene->view, count, false);
        shadow_kernel<64><<<ctx->sm_count * 16, 128, 0, st>>>(V, F, scene->view, 32u);
        radiance_out_kernel<<<(count + 127) / 128, 128, 0, st>>>(V, count, (float4 *)out);
    }
    return lux_cuda_check(ctx, (int)cudaGetLastError(), "interval_radiance launch");
}

}  // namespace

extern "C" lux_status lux_interval_radiance(LuxContext *ctx, const LuxScene *scene, const LuxSettings *settings,
                                           const LuxRay *rays, uint32_t count, float *out) {
    if (!ctx || !scene || !settings || (count && (!rays || !out))) return LUX_ERR_INVALID_ARGUMENT;
    if ((uint64_t)count * lux::kMaxNeeSamples > 0xffffffffull)
        return lux_fail(ctx, LUX_ERR_CAPACITY, "interval_radiance: more than 2^28 rays");
    if (count > ctx->scratch_rays) {
        cudaStreamSynchronize(ctx->stream);
        if (ctx->scratch_mem) cudaFree(ctx->scratch_mem);
        ctx->scratch_mem = nullptr;
        ctx->scratch_rays = 0;
        if (cudaMalloc(&ctx->scratch_mem, carved_scratch_bytes(count)) != cudaSuccess) {
            cudaGetLastError();
            return lux_fail(ctx, LUX_ERR_OUT_OF_MEMORY, "interval_radiance: scratch allocation failed");
        }
        ctx->scratch_rays = count;
    }
    ViewDevice V;
    std::memset(&V, 0, sizeof V);
    carve_trace_scratch((unsigned char *)ctx->scratch_mem, ctx->scratch_rays, V.ts, V.error_flags, V.stats);
    return launch_interval_radiance(ctx, scene, settings, rays, count, out, V, ctx->scratch_rays);
}

// ---------------------------------------------------------------------------
// lux_interval_radiance_noalloc: lux_interval_radiance for callers that must
// not allocate device memory.  Its trace scratch is one fixed array in the
// library's own device image (reserved when the module loads on a device), so
// the call makes no cudaMalloc, cudaFree or allocating library call.
// ---------------------------------------------------------------------------
namespace {

constexpr uint32_t kNoAllocMaxRays = 8192u;
constexpr size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
// Same partition as carve_trace_scratch for kNoAllocMaxRays rays.
constexpr size_t kNoAllocBytes = 4 * align256((size_t)kNoAllocMaxRays * 16) +
                                 align256((size_t)kNoAllocMaxRays * 16 * 4) +
                                 3 * align256((size_t)kNoAllocMaxRays * 16 * 16) +
                                 align256((size_t)kNoAllocMaxRays * 16) + 3 * align256(16) + align256(128);

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char *g_noalloc_address[kNoAllocMaxDevices] = {};

}  // namespace

// About 7.5 MiB, held on every device that loads the library, until exit.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

extern "C" lux_status lux_interval_radiance_noalloc(LuxContext *ctx, const LuxScene *scene,
                                                    const LuxSettings *settings, const LuxRay *rays, uint32_t count,
                                                    float *out) {
    if (!ctx || !scene || !settings || (count && (!rays || !out))) return LUX_ERR_INVALID_ARGUMENT;
    if (count > kNoAllocMaxRays)
        return lux_fail(ctx, LUX_ERR_CAPACITY,
                        "interval_radiance_noalloc: " + std::to_string(count) +
                            " rays exceed the fixed scratch capacity of 8192 rays; split the batch");
    if (ctx->device < 0 || ctx->device >= kNoAllocMaxDevices)
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "interval_radiance_noalloc: device ordinal out of range");
    unsigned char *base = nullptr;
    {
        // Set-up once per device, with that device current: the host-side
        // name of the array is not a device address; ask the runtime for it.
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        base = g_noalloc_address[ctx->device];
        if (!base) {
            // The caller's current device is put back afterwards, so a render
            // thread working on another device does not see it change.
            int previous = -1;
            lux_status s = lux_cuda_check(ctx, (int)cudaGetDevice(&previous), "interval_radiance_noalloc get device");
            if (s != LUX_OK) return s;
            s = lux_cuda_check(ctx, (int)cudaSetDevice(ctx->device), "interval_radiance_noalloc set device");
            if (s != LUX_OK) return s;
            void *address = nullptr;
            s = lux_cuda_check(ctx, (int)cudaGetSymbolAddress(&address, g_noalloc_scratch),
                               "interval_radiance_noalloc scratch address");
            if (previous != ctx->device) cudaSetDevice(previous);
            if (s != LUX_OK) return s;
            base = (unsigned char *)address;
            g_noalloc_address[ctx->device] = base;
        }
    }
    ViewDevice V;
    std::memset(&V, 0, sizeof V);
    unsigned char *end = carve_trace_scratch(base, kNoAllocMaxRays, V.ts, V.error_flags, V.stats);
    if ((size_t)(end - base) > kNoAllocBytes)
        return lux_fail(ctx, LUX_ERR_INTERNAL, "interval_radiance_noalloc: scratch partition exceeds the array");
    return launch_interval_radiance(ctx, scene, settings, rays, count, out, V, kNoAllocMaxRays);
}

// ---- lux_view_read_hits ----------------------------------------------------

extern "C" lux_status lux_view_read_hits(LuxView *v, LuxHit *out, uint32_t count) {
    if (!v || (count && !out)) return LUX_ERR_INVALID_ARGUMENT;
    if (!v->has_frame || v->last.layout != LUX_LAYOUT_SPLIT)
        return lux_fail(v->ctx, LUX_ERR_INVALID_ARGUMENT, "read_hits: no Split frame traced yet");
    if ((uint64_t)count > (uint64_t)v->last.receivers * v->last.rays_per_receiver)
        return lux_fail(v->ctx, LUX_ERR_INVALID_ARGUMENT, "read_hits: more hits than the frame's interval rays");
    if (count == 0) return LUX_OK;
    LuxContext *ctx = v->ctx;
    cudaStream_t st = ctx->stream;
    LuxHit *d = nullptr;
    lux_status rc = lux_cuda_check(ctx, (int)cudaMallocAsync((void **)&d, (size_t)count * sizeof(LuxHit), st),
                                   "read_hits: staging");
    if (rc != LUX_OK) return rc;
    read_hits_kernel<<<(count + 255) / 256, 256, 0, st>>>(v->dev, count, d);
    cudaMemcpyAsync(out, d, (size_t)count * sizeof(LuxHit), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(d, st);
    rc = lux_cuda_check(ctx, (int)cudaStreamSynchronize(st), "read_hits");
    if (rc != LUX_OK) return rc;
    return lux_cuda_check(ctx, (int)cudaGetLastError(), "read_hits launch");
}

// ---- batches ---------------------------------------------------------------

struct LuxBatch {
    LuxContext *ctx = nullptr;
    LuxTuning tuning{0, 0, 16, 16, 0, 0, 64, 0, 32, 0};
    bool use_graph = true;
    // Configuration the device tables and graph were built for.
    std::vector<LuxBatchJob> jobs;
    LuxSettings settings{};  // frame_index zeroed
    bool history = false;    // the settings blend history: retain and history mapping run
    std::vector<FrameParams> params;
    uint32_t total = 0;      // padded interval rays
    uint64_t rays = 0;
    bool built = false;
    BatchJob *d_jobs = nullptr;
    uint32_t *d_begin = nullptr, *d_qbegin = nullptr, *d_counters = nullptr, *d_frame = nullptr;
    size_t job_capacity = 0;
    // Domain table (kBatchRows x (n + 1) padded prefixes) and the device
    // rows' unpadded per-job sizes (kDeviceRows x n).
    unsigned long long *d_dom = nullptr, *d_count = nullptr;
    // Sequence-order sort of all jobs' receivers: keys and receiver indices
    // (in, out halves), per-job segment bounds, scratch.
    unsigned long long *d_keys = nullptr;
    uint32_t *d_vals = nullptr;
    int *d_seg = nullptr;  // [2][n] begin, end
    void *d_sort_temp = nullptr;
    size_t sort_temp_bytes = 0, recv_capacity = 0;
    uint64_t recv_total = 0;  // padded receivers of all jobs
    uint32_t levels = 0, max_dirs0 = 0;
    // The job table and frame index of each frame go through two pinned
    // host slots (the table holds the views' current buffers, swapped by
    // history, and the frame's parameters); staged[k] marks the copy that
    // last read slot k.
    void *h_stage[2] = {nullptr, nullptr};
    size_t stage_bytes = 0;
    cudaEvent_t staged[2] = {nullptr, nullptr};
    uint32_t stage_slot = 0;
    int fused_per_sm = 0;                          // resident trace_batch_kernel blocks per SM
    unsigned long long wait_limit_ns = 1000000000ull;  // grid-barrier wait bound
    uint32_t wait_missing = 0;                     // test hook: arrivals that never come
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t captures = 0;
    uint64_t replays = 0;
    uint32_t kernels = 0;
};

static void batch_release_graph(LuxBatch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

static void batch_release_sort(LuxBatch *b) {
    cudaFree(b->d_keys);
    cudaFree(b->d_vals);
    cudaFree(b->d_sort_temp);
    b->d_keys = nullptr;
    b->d_vals = nullptr;
    b->d_sort_temp = nullptr;
    b->sort_temp_bytes = b->recv_capacity = 0;
}

static void batch_release_tables(LuxBatch *b) {
    cudaFree(b->d_jobs);
    cudaFree(b->d_begin);
    cudaFree(b->d_qbegin);
    cudaFree(b->d_dom);
    cudaFree(b->d_count);
    cudaFree(b->d_seg);
    b->d_jobs = nullptr;
    b->d_begin = b->d_qbegin = nullptr;
    b->d_dom = b->d_count = nullptr;
    b->d_seg = nullptr;
    b->job_capacity = 0;
}

extern "C" lux_status lux_batch_create(LuxContext *ctx, LuxBatch **out) {
    if (!ctx || !out) return LUX_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    LuxBatch *b = new (std::nothrow) LuxBatch();
    if (!b) return LUX_ERR_OUT_OF_MEMORY;
    b->ctx = ctx;
    cudaSetDevice(ctx->device);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->fused_per_sm, trace_batch_kernel, 128, 0) != cudaSuccess) {
        cudaGetLastError();
        b->fused_per_sm = 0;
    }
    if (cudaEventCreateWithFlags(&b->staged[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->staged[1], cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc((void **)&b->d_counters, 16) != cudaSuccess || cudaMalloc((void **)&b->d_frame, 16) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(b->d_counters);
        for (int k = 0; k < 2; ++k)
            if (b->staged[k]) cudaEventDestroy(b->staged[k]);
        delete b;
        return lux_fail(ctx, LUX_ERR_OUT_OF_MEMORY, "batch: device allocation failed");
    }
    *out = b;
    return LUX_OK;
}

extern "C" lux_status lux_batch_destroy(LuxBatch *b) {
    if (!b) return LUX_OK;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    batch_release_graph(b);
    batch_release_tables(b);
    batch_release_sort(b);
    for (int k = 0; k < 2; ++k) {
        cudaFreeHost(b->h_stage[k]);
        if (b->staged[k]) cudaEventDestroy(b->staged[k]);
    }
    cudaFree(b->d_counters);
    cudaFree(b->d_frame);
    delete b;
    return LUX_OK;
}

extern "C" lux_status lux_batch_set_graph(LuxBatch *b, uint32_t enable) {
    if (!b) return LUX_ERR_INVALID_ARGUMENT;
    b->use_graph = enable != 0;
    b->built = false;
    return LUX_OK;
}

extern "C" lux_status lux_batch_set_tuning(LuxBatch *b, const LuxTuning *t) {
    if (!b || !t) return LUX_ERR_INVALID_ARGUMENT;
    if (t->closest_blocks_per_sm < 1 || t->closest_blocks_per_sm > 64 || t->shadow_blocks_per_sm < 1 ||
        t->shadow_blocks_per_sm > 64)
        return lux_fail(b->ctx, LUX_ERR_INVALID_ARGUMENT, "batch tuning: blocks per SM must be 1..64");
    if (!tile_valid(t->tile_rays) || t->fused_trace > 1)
        return lux_fail(b->ctx, LUX_ERR_INVALID_ARGUMENT, "batch tuning: tile_rays or fused_trace out of range");
    b->tuning = *t;
    b->built = false;
    return LUX_OK;
}

extern "C" lux_status lux_batch_set_wait(LuxBatch *b, uint64_t limit_ns, uint32_t missing_arrivals) {
    if (!b) return LUX_ERR_INVALID_ARGUMENT;
    if (limit_ns < 1000000ull || limit_ns > 10000000000ull)
        return lux_fail(b->ctx, LUX_ERR_INVALID_ARGUMENT, "batch wait: limit must be 1 ms .. 10 s");
    b->wait_limit_ns = limit_ns;
    b->wait_missing = missing_arrivals;
    b->built = false;
    return LUX_OK;
}

extern "C" lux_status lux_batch_status(LuxBatch *b) {
    if (!b) return LUX_ERR_INVALID_ARGUMENT;
    LuxContext *ctx = b->ctx;
    cudaSetDevice(ctx->device);
    lux_status rc = lux_cuda_check(ctx, (int)cudaStreamSynchronize(ctx->stream), "batch status: synchronize");
    if (rc != LUX_OK) return rc;
    uint32_t abort = 0;
    rc = lux_cuda_check(ctx, (int)cudaMemcpy(&abort, b->d_counters + 3, 4, cudaMemcpyDeviceToHost),
                        "batch status: read");
    if (rc != LUX_OK) return rc;
    if (abort) return lux_fail(ctx, LUX_ERR_TIMEOUT, "batch: a trace-stage grid barrier wait ran out");
    return LUX_OK;
}

extern "C" lux_status lux_batch_info(const LuxBatch *b, LuxBatchInfo *out) {
    if (!b || !out) return LUX_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof *out);
    out->jobs = (uint32_t)b->jobs.size();
    out->graph_captures = b->captures;
    out->graph_launches = b->replays;
    out->interval_rays = b->rays;
    out->kernels_per_frame = b->kernels;
    return LUX_OK;
}

static bool same_jobs(const std::vector<LuxBatchJob> &a, const LuxBatchJob *b, uint32_t n) {
    if (a.size() != n) return false;
    for (uint32_t j = 0; j < n; ++j)
        if (a[j].view != b[j].view || a[j].scene != b[j].scene || a[j].receivers.position != b[j].receivers.position ||
            a[j].receivers.normal != b[j].receivers.normal || a[j].receivers.count != b[j].receivers.count)
            return false;
    return true;
}

// Every kernel of one batched frame, in order, on `st` (captured or direct):
// each per-view pass runs once over all jobs.
static void batch_enqueue(LuxBatch *b, cudaStream_t st) {
    LuxContext *ctx = b->ctx;
    const uint32_t n = (uint32_t)b->jobs.size();
    const int grid = ctx->sm_count * 8;
    cudaMemsetAsync(b->d_counters, 0, 16, st);  // work counters, barrier arrivals, abort word
    batch_clear_kernel<<<grid, 256, 0, st>>>(b->d_jobs, b->d_dom, n);
    if (b->recv_total) {
        const size_t half = b->recv_capacity;
        batch_seed_insert_kernel<<<grid, 256, 0, st>>>(b->d_jobs, b->d_dom, n);
        batch_seed_assign_kernel<<<grid, 256, 0, st>>>(b->d_jobs, b->d_dom, n);
        batch_seed_lookup_kernel<<<grid, 256, 0, st>>>(b->d_jobs, b->d_dom, n, b->d_keys, b->d_vals);
        size_t bytes = b->sort_temp_bytes;
        cub::DeviceSegmentedSort::StableSortPairs(b->d_sort_temp, bytes, b->d_keys, b->d_keys + half, b->d_vals,
                                                  b->d_vals + half, (int)b->recv_total, (int)n, b->d_seg,
                                                  b->d_seg + n, st);
        batch_ordinal_kernel<<<grid, 256, 0, st>>>(b->d_jobs, b->d_dom, n, b->d_vals + half);
    }
    if (b->history) {  // retain: the previous frame's unseen cells stay
        const dim3 g2(std::max(1, grid / (int)std::min(n, 64u)), std::min(n, 65535u));
        batch_retain_count_kernel<<<g2, 256, 0, st>>>(b->d_jobs, n);
        batch_retain_limit_kernel<<<std::min(n, 65535u), kRetainBins, 0, st>>>(b->d_jobs, n);
        batch_retain_insert_kernel<<<g2, 256, 0, st>>>(b->d_jobs, n);
    }
    batch_layout_kernel<<<1, 1024, 0, st>>>(b->d_jobs, n, b->d_dom, b->d_count);
    batch_clear_entries_kernel<<<grid, 256, 0, st>>>(b->d_jobs, b->d_dom, n, b->d_count);
    if (b->total && b->tuning.fused_trace) {
        // One cooperative launch: no more blocks than can be resident.
        const uint32_t per_sm = std::min(b->tuning.closest_blocks_per_sm, (uint32_t)std::max(b->fused_per_sm, 1));
        GridBarrier B{b->d_counters + 2, b->d_counters + 3, b->wait_limit_ns, b->wait_missing};
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(ctx->sm_count * per_sm);
        cfg.blockDim = dim3(128);
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, trace_batch_kernel, (const BatchJob *)b->d_jobs, (const uint32_t *)b->d_begin, n,
                           b->total, (const uint32_t *)b->d_frame, b->d_counters, b->d_qbegin, B,
                           tile_of(b->tuning));
    } else if (b->total) {
        closest_batch_kernel<<<ctx->sm_count * b->tuning.closest_blocks_per_sm, 128, 0, st>>>(
            b->d_jobs, b->d_begin, n, b->total, b->d_frame, b->d_counters, tile_of(b->tuning));
        shade_batch_kernel<<<grid, 128, 0, st>>>(b->d_jobs, b->d_begin, n, b->total, b->d_frame);
        query_prefix_kernel<<<1, 128, 0, st>>>(b->d_jobs, n, b->d_qbegin);
        shadow_batch_kernel<<<ctx->sm_count * b->tuning.shadow_blocks_per_sm, 128, 0, st>>>(
            b->d_jobs, b->d_qbegin, n, b->d_counters + 1, tile_of(b->tuning));
        deposit_batch_kernel<<<grid, 128, 0, st>>>(b->d_jobs, b->d_begin, n, b->total, b->d_frame);
    }
    if (b->levels > 1 || b->history)
        batch_merge_prep_kernel<<<grid, 128, 0, st>>>(b->d_jobs, b->d_dom, n, b->d_count, b->levels);
    // The children passes over each job's list of the records that pass
    // light on (32-bit record indices: every view's records fit them).
    bool listed = LUX_MERGE_COMPACT && b->levels > 1;
    for (const LuxBatchJob &job : b->jobs) listed = listed && job.view->desc.max_entries <= 0xffffffffull;
    if (listed) {
        batch_merge_own_list_kernel<<<grid * 2, 256, 0, st>>>(b->d_jobs, b->d_dom, n, b->d_count);
        batch_list_prefix_kernel<<<1, 32 * LUX_MAX_LEVELS, 0, st>>>(b->d_jobs, b->d_dom, n, b->levels);
        for (int l = (int)b->levels - 2; l >= 0; --l)
            batch_merge_children_list_kernel<<<grid * 512 / LUX_MERGE_THREADS, LUX_MERGE_THREADS, 0, st>>>(
                b->d_jobs, b->d_dom, n, (uint32_t)l);
    } else {
        batch_merge_own_kernel<<<grid * 2, 256, 0, st>>>(b->d_jobs, b->d_dom, n, b->d_count);
        for (int l = (int)b->levels - 2; l >= 0; --l)
            batch_merge_children_kernel<<<grid * 512 / LUX_MERGE_THREADS, LUX_MERGE_THREADS, 0, st>>>(
                b->d_jobs, b->d_dom, n, b->d_count, (uint32_t)l);
    }
    batch_pack_kernel<<<grid, 64, (size_t)b->max_dirs0 * 2 * sizeof(float4), st>>>(b->d_jobs, b->d_dom, n,
                                                                                 b->d_count, b->max_dirs0);
}

// Kernel nodes of a captured graph (the launches one replay makes).
static uint32_t graph_kernels(cudaGraph_t g) {
    size_t count = 0;
    if (cudaGraphGetNodes(g, nullptr, &count) != cudaSuccess) return 0;
    std::vector<cudaGraphNode_t> nodes(count);
    if (cudaGraphGetNodes(g, nodes.data(), &count) != cudaSuccess) return 0;
    uint32_t kernels = 0;
    for (cudaGraphNode_t node : nodes) {
        cudaGraphNodeType type;
        if (cudaGraphNodeGetType(node, &type) == cudaSuccess && type == cudaGraphNodeTypeKernel) ++kernels;
    }
    return kernels;
}

static lux_status batch_build(LuxBatch *b, const LuxBatchJob *jobs, uint32_t n, const LuxSettings &s,
                              std::vector<FrameParams> &params) {
    LuxContext *ctx = b->ctx;
    cudaStream_t st = ctx->stream;
    lux_status rc = lux_cuda_check(ctx, (int)cudaStreamSynchronize(st), "batch: synchronize");
    if (rc != LUX_OK) return rc;
    batch_release_graph(b);
    b->built = false;
    if (n > b->job_capacity) {
        batch_release_tables(b);
        if (cudaMalloc((void **)&b->d_jobs, n * sizeof(BatchJob)) != cudaSuccess ||
            cudaMalloc((void **)&b->d_begin, (n + 1) * 4) != cudaSuccess ||
            cudaMalloc((void **)&b->d_qbegin, (n + 1) * 4) != cudaSuccess ||
            cudaMalloc((void **)&b->d_dom, (size_t)kBatchRows * (n + 1) * 8) != cudaSuccess ||
            cudaMalloc((void **)&b->d_count, (size_t)kDeviceRows * n * 8) != cudaSuccess ||
            cudaMalloc((void **)&b->d_seg, (size_t)2 * n * sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            batch_release_tables(b);
            return lux_fail(ctx, LUX_ERR_OUT_OF_MEMORY, "batch: device allocation failed");
        }
        b->job_capacity = n;
    }
    // Host-sized domain rows and the receivers' sort segments.
    std::vector<unsigned long long> rows((size_t)kRowEntries * (n + 1), 0ull);
    std::vector<int> seg((size_t)2 * n, 0);
    uint32_t levels = 0, max_dirs0 = 1;
    for (uint32_t j = 0; j < n; ++j) {
        const FrameParams &F = params[j];
        const unsigned long long size[kRowEntries] = {(unsigned long long)F.levels * F.dir_capacity,
                                                      (unsigned long long)F.receivers * F.levels, F.receivers};
        for (uint32_t r = 0; r < kRowEntries; ++r)
            rows[(size_t)r * (n + 1) + j + 1] = rows[(size_t)r * (n + 1) + j] + ((size[r] + 31ull) & ~31ull);
        seg[j] = (int)rows[(size_t)kRowRecv * (n + 1) + j];
        seg[n + j] = seg[j] + (int)F.receivers;
        levels = std::max(levels, F.levels);
        max_dirs0 = std::max(max_dirs0, F.dirs[0]);
    }
    const uint64_t recv_total = rows[(size_t)kRowRecv * (n + 1) + n];
    if (recv_total > 0x7fffffe0ull) return lux_fail(ctx, LUX_ERR_CAPACITY, "batch: more than 2^31 receivers");
    if (recv_total > b->recv_capacity) {
        batch_release_sort(b);
        size_t temp = 0;
        cub::DeviceSegmentedSort::StableSortPairs(nullptr, temp, (const unsigned long long *)nullptr,
                                                  (unsigned long long *)nullptr, (const uint32_t *)nullptr,
                                                  (uint32_t *)nullptr, (int)recv_total, (int)n, (const int *)nullptr,
                                                  (const int *)nullptr, st);
        if (cudaMalloc((void **)&b->d_keys, recv_total * 16) != cudaSuccess ||
            cudaMalloc((void **)&b->d_vals, recv_total * 8) != cudaSuccess ||
            cudaMalloc(&b->d_sort_temp, std::max<size_t>(temp, 16)) != cudaSuccess) {
            cudaGetLastError();
            batch_release_sort(b);
            return lux_fail(ctx, LUX_ERR_OUT_OF_MEMORY, "batch: device allocation failed");
        }
        b->recv_capacity = recv_total;
        b->sort_temp_bytes = std::max<size_t>(temp, 16);
    } else {
        size_t temp = 0;
        cub::DeviceSegmentedSort::StableSortPairs(nullptr, temp, (const unsigned long long *)nullptr,
                                                  (unsigned long long *)nullptr, (const uint32_t *)nullptr,
                                                  (uint32_t *)nullptr, (int)recv_total, (int)n, (const int *)nullptr,
                                                  (const int *)nullptr, st);
        if (temp > b->sort_temp_bytes) {
            cudaFree(b->d_sort_temp);
            b->d_sort_temp = nullptr;
            if (cudaMalloc(&b->d_sort_temp, temp) != cudaSuccess) {
                cudaGetLastError();
                batch_release_sort(b);
                return lux_fail(ctx, LUX_ERR_OUT_OF_MEMORY, "batch: device allocation failed");
            }
            b->sort_temp_bytes = temp;
        }
    }
    rc = lux_cuda_check(ctx, (int)cudaMemcpy(b->d_dom, rows.data(), rows.size() * 8, cudaMemcpyHostToDevice),
                        "batch: domain rows");
    if (rc == LUX_OK)
        rc = lux_cuda_check(ctx, (int)cudaMemcpy(b->d_seg, seg.data(), seg.size() * sizeof(int), cudaMemcpyHostToDevice),
                            "batch: sort segments");
    if (rc != LUX_OK) return rc;
    b->recv_total = recv_total;
    b->levels = levels;
    b->max_dirs0 = max_dirs0;
    std::vector<uint32_t> begin(n + 1, 0);
    uint64_t padded = 0, rays = 0;
    for (uint32_t j = 0; j < n; ++j) {
        const FrameParams &F = params[j];
        uint32_t r = F.receivers * F.rays_per_receiver;
        begin[j] = (uint32_t)padded;
        padded += (r + 31u) & ~31u;
        rays += r;
    }
    if (padded > 0xffffffe0ull) return lux_fail(ctx, LUX_ERR_CAPACITY, "batch: more than 2^32 interval rays");
    begin[n] = (uint32_t)padded;
    rc = lux_cuda_check(ctx, (int)cudaMemcpy(b->d_begin, begin.data(), (n + 1) * 4, cudaMemcpyHostToDevice),
                        "batch: ray offsets");
    if (rc != LUX_OK) return rc;
    const size_t stage = n * sizeof(BatchJob) + 16;
    if (stage > b->stage_bytes) {  // the stream is idle: no copy reads the old slots
        for (int k = 0; k < 2; ++k) {
            cudaFreeHost(b->h_stage[k]);
            b->h_stage[k] = nullptr;
        }
        b->stage_bytes = 0;
        if (cudaHostAlloc(&b->h_stage[0], stage, cudaHostAllocDefault) != cudaSuccess ||
            cudaHostAlloc(&b->h_stage[1], stage, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return lux_fail(ctx, LUX_ERR_OUT_OF_MEMORY, "batch: pinned host allocation failed");
        }
        b->stage_bytes = stage;
    }
    b->jobs.assign(jobs, jobs + n);
    b->settings = s;
    b->settings.frame_index = 0;
    b->history = s.history_frames > 0 && (s.temporal_blend > 0.0f || s.transmittance_blend > 0.0f);
    b->params = params;
    b->total = (uint32_t)padded;
    b->rays = rays;
    // The frame is captured once either way: the graph's kernel nodes are
    // the launches a frame makes; without graphs the capture is discarded.
    rc = lux_cuda_check(ctx, (int)cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "batch: capture");
    if (rc != LUX_OK) return rc;
    batch_enqueue(b, st);
    cudaGraph_t g = nullptr;
    rc = lux_cuda_check(ctx, (int)cudaStreamEndCapture(st, &g), "batch: end capture");
    if (rc != LUX_OK) return rc;
    b->graph = g;
    b->kernels = graph_kernels(g);
    if (b->use_graph) {
        rc = lux_cuda_check(ctx, (int)cudaGraphInstantiate(&b->exec, g, 0), "batch: instantiate");
        if (rc != LUX_OK) {
            batch_release_graph(b);
            return rc;
        }
        ++b->captures;
    } else {
        batch_release_graph(b);
    }
    b->built = true;
    return LUX_OK;
}

extern "C" lux_status lux_batch_trace_merge(LuxBatch *b, const LuxBatchJob *jobs, uint32_t n,
                                            const LuxSettings *settings) {
    if (!b || !settings || (n && !jobs)) return LUX_ERR_INVALID_ARGUMENT;
    LuxContext *ctx = b->ctx;
    if (n == 0 || n > 65536) return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "batch: need 1..65536 jobs");
    LuxSettings s = *settings;
    lux_settings_sanitize(&s);
    if (s.layout != LUX_LAYOUT_SPLIT) return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "batch: layout must be Split");
    if (s.multi_bounce) return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "batch: multi_bounce runs per view");
    std::vector<FrameParams> params(n);
    for (uint32_t j = 0; j < n; ++j) {
        const LuxBatchJob &J = jobs[j];
        if (!J.view || !J.scene || J.view->ctx != ctx || J.scene->ctx != ctx)
            return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "batch: job view/scene missing or on another context");
        for (uint32_t k = 0; k < j; ++k)
            if (jobs[k].view == J.view) return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "batch: a view appears twice");
        const LuxReceivers &rc = J.receivers;
        if (rc.count > J.view->desc.max_receivers)
            return lux_fail(ctx, LUX_ERR_CAPACITY, "batch: more receivers than a view's max_receivers");
        if (rc.count && (!rc.position || !rc.normal))
            return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "batch: missing receiver buffers");
        lux_status ps = make_params(J.view, &s, rc.count, params[j]);
        if (ps != LUX_OK) return ps;
        ps = check_nee_slots(ctx, &s, J.scene);
        if (ps != LUX_OK) return ps;
        params[j].lod_enabled = 0;  // batched frames use LOD 0
        if ((uint64_t)rc.count * params[j].rays_per_receiver > J.view->desc.max_rays)
            return lux_fail(ctx, LUX_ERR_CAPACITY, "batch: receivers x rays_per_receiver exceeds a view's max_rays");
    }
    cudaSetDevice(ctx->device);
    LuxSettings key = s;
    key.frame_index = 0;
    // The graph depends on the jobs' sizes and the settings, not on the
    // views' buffers (the job table is copied every frame).
    bool same = b->built && same_jobs(b->jobs, jobs, n) && std::memcmp(&key, &b->settings, sizeof key) == 0;
    if (!same) {
        lux_status rc = batch_build(b, jobs, n, s, params);
        if (rc != LUX_OK) return rc;
    }
    cudaStream_t st = ctx->stream;
    // This frame's job table: each view's history turns over (buffer swap,
    // invalidation boxes) as in an unbatched frame.
    const uint32_t k = b->stage_slot;
    b->stage_slot ^= 1u;
    lux_status rc = lux_cuda_check(ctx, (int)cudaEventSynchronize(b->staged[k]), "batch: stage slot");
    if (rc != LUX_OK) return rc;
    BatchJob *h = static_cast<BatchJob *>(b->h_stage[k]);
    uint32_t *h_frame = reinterpret_cast<uint32_t *>(h + n);
    std::vector<FrameParams> frame_params(n);
    for (uint32_t j = 0; j < n; ++j) {
        FrameParams &F = frame_params[j];
        F = b->params[j];
        F.shade.frame = s.frame_index;
        begin_history(jobs[j].view, F, s);
        BatchJob &J = h[j];
        std::memset(&J, 0, sizeof J);
        J.V = jobs[j].view->dev;
        J.V.sort_keys = nullptr;
        J.V.ray_order = nullptr;
        J.V.query_order = nullptr;
        J.F = F;
        J.S = jobs[j].scene->view;
        J.H = history_device(jobs[j].view);
        J.pos = (const float4 *)jobs[j].receivers.position;
        J.nrm = (const float4 *)jobs[j].receivers.normal;
        J.rays = F.receivers * F.rays_per_receiver;
    }
    *h_frame = s.frame_index;
    rc = lux_cuda_check(ctx, (int)cudaMemcpyAsync(b->d_jobs, h, n * sizeof(BatchJob), cudaMemcpyHostToDevice, st),
                        "batch: job table");
    if (rc == LUX_OK)
        rc = lux_cuda_check(ctx, (int)cudaMemcpyAsync(b->d_frame, h_frame, 4, cudaMemcpyHostToDevice, st),
                            "batch: frame index");
    if (rc == LUX_OK) rc = lux_cuda_check(ctx, (int)cudaEventRecord(b->staged[k], st), "batch: stage event");
    if (rc != LUX_OK) return rc;
    if (b->use_graph) {
        rc = lux_cuda_check(ctx, (int)cudaGraphLaunch(b->exec, st), "batch: graph launch");
        if (rc != LUX_OK) return rc;
        ++b->replays;
    } else {
        batch_enqueue(b, st);
    }
    for (uint32_t j = 0; j < n; ++j) {
        jobs[j].view->last = frame_params[j];
        jobs[j].view->has_frame = true;
        end_history(jobs[j].view, frame_params[j]);
    }
    return lux_cuda_check(ctx, (int)cudaGetLastError(), "batch launch");
}

// ---- FP64 reference irradiance and error reductions --------------------------
// The oracle of the error reports (no reference counterpart): Monte Carlo
// over cosine-weighted hemisphere rays of the same interval radiance the
// cascades resolve (emission seen + one-bounce next-event estimation), each
// ray traced and shaded in FP32 by the library's kernels, the per-point means
// accumulated in FP64.
namespace {

constexpr uint32_t kReferenceRoundRays = 1u << 21;

__global__ void reference_rays_kernel(const float4 *__restrict__ pos, const float4 *__restrict__ nrm, uint32_t count,
                                      uint32_t sample0, uint32_t samples, uint32_t seed, float bias,
                                      LuxRay *__restrict__ rays) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count * samples) return;
    uint32_t p = i / samples, s = sample0 + i % samples;
    float4 p4 = pos[p], n4 = nrm[p];
    f3 P{p4.x, p4.y, p4.z}, N{n4.x, n4.y, n4.z};
    float u1, u2;
    lux::reference_sample(p, s, seed, u1, u2);
    f3 d = lux::cosine_direction(N, u1, u2);
    f3 o = lux::ray_offset(P, N, bias);
    LuxRay r;
    r.origin[0] = o.x;
    r.origin[1] = o.y;
    r.origin[2] = o.z;
    r.tmin = 0.0f;
    r.direction[0] = d.x;
    r.direction[1] = d.y;
    r.direction[2] = d.z;
    r.limit = 1e20f;
    rays[i] = r;
}

// acc[p] += (sum of supported sample radiance, supported samples), in
// sample order.
__global__ void reference_accumulate_kernel(const float4 *__restrict__ radiance, uint32_t count, uint32_t samples,
                                            double4 *__restrict__ acc) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    double4 a = acc[p];
    for (uint32_t s = 0; s < samples; ++s) {
        float4 v = radiance[(size_t)p * samples + s];
        if (v.w < 0.0f) continue;
        a.x += (double)v.x;
        a.y += (double)v.y;
        a.z += (double)v.z;
        a.w += 1.0;
    }
    acc[p] = a;
}

__global__ void reference_finish_kernel(double4 *__restrict__ acc, uint32_t count) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    double4 a = acc[p];
    acc[p] = a.w > 0.0 ? make_double4(a.x / a.w, a.y / a.w, a.z / a.w, a.w) : make_double4(0.0, 0.0, 0.0, 0.0);
}

// out[0] += sum of squared rgb error, out[1] += sum of reference rgb,
// out[2] += points used, out[3] = max |error| (as ordered bits): points with
// estimate alpha > 0 and at least one reference sample.
__global__ void error_stats_kernel(const float4 *__restrict__ est, const double4 *__restrict__ ref, uint32_t count,
                                   double *__restrict__ out) {
    double sq = 0.0, sum = 0.0, used = 0.0, mx = 0.0;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < count; p += gridDim.x * blockDim.x) {
        float4 e = est[p];
        double4 r = ref[p];
        if (!(e.w > 0.0f) || !(r.w > 0.0)) continue;
        double dx = (double)e.x - r.x, dy = (double)e.y - r.y, dz = (double)e.z - r.z;
        sq += dx * dx + dy * dy + dz * dz;
        sum += r.x + r.y + r.z;
        used += 1.0;
        mx = fmax(mx, fmax(fabs(dx), fmax(fabs(dy), fabs(dz))));
    }
    for (int off = 16; off > 0; off >>= 1) {
        sq += __shfl_down_sync(0xffffffffu, sq, off);
        sum += __shfl_down_sync(0xffffffffu, sum, off);
        used += __shfl_down_sync(0xffffffffu, used, off);
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
    }
    if ((threadIdx.x & 31u) == 0u) {
        atomicAdd(&out[0], sq);
        atomicAdd(&out[1], sum);
        atomicAdd(&out[2], used);
        atomicMax((unsigned long long *)&out[3], (unsigned long long)__double_as_longlong(mx));
    }
}

}  // namespace

extern "C" uint32_t lux_reference_round_samples(uint32_t count, uint32_t spp) {
    if (count == 0 || spp == 0) return 0;
    uint32_t r = kReferenceRoundRays / count;
    r = r < 1u ? 1u : r;
    return r < spp ? r : spp;
}

extern "C" lux_status lux_reference_irradiance(LuxContext *ctx, const LuxScene *scene, const LuxSettings *settings,
                                               const float *position, const float *normal, uint32_t count,
                                               uint32_t spp, uint32_t seed, double *out) {
    if (!ctx || !scene || !settings || (count && (!position || !normal || !out))) return LUX_ERR_INVALID_ARGUMENT;
    if (count == 0) return LUX_OK;
    if (spp == 0) return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "reference: spp must be positive");
    LuxSettings s = *settings;
    lux_settings_sanitize(&s);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const uint32_t round = lux_reference_round_samples(count, spp);
    const uint32_t rays = count * round;
    LuxRay *d_rays = nullptr;
    float4 *d_rad = nullptr;
    lux_status rc = lux_cuda_check(ctx, (int)cudaMallocAsync((void **)&d_rays, (size_t)rays * sizeof(LuxRay), st),
                                   "reference: rays");
    if (rc == LUX_OK)
        rc = lux_cuda_check(ctx, (int)cudaMallocAsync((void **)&d_rad, (size_t)rays * sizeof(float4), st),
                            "reference: radiance");
    if (rc == LUX_OK)
        rc = lux_cuda_check(ctx, (int)cudaMemsetAsync(out, 0, (size_t)count * sizeof(double4), st), "reference: clear");
    for (uint32_t k = 0, s0 = 0; rc == LUX_OK && s0 < spp; ++k, s0 += round) {
        uint32_t samples = std::min(round, spp - s0);
        uint32_t n = count * samples;
        reference_rays_kernel<<<(n + 255) / 256, 256, 0, st>>>((const float4 *)position, (const float4 *)normal,
                                                                count, s0, samples, seed, s.normal_bias, d_rays);
        LuxSettings fs = s;
        fs.frame_index = seed + k;
        rc = lux_interval_radiance(ctx, scene, &fs, d_rays, n, (float *)d_rad);
        if (rc != LUX_OK) break;
        reference_accumulate_kernel<<<(count + 127) / 128, 128, 0, st>>>(d_rad, count, samples, (double4 *)out);
    }
    if (rc == LUX_OK) reference_finish_kernel<<<(count + 127) / 128, 128, 0, st>>>((double4 *)out, count);
    if (d_rays) cudaFreeAsync(d_rays, st);
    if (d_rad) cudaFreeAsync(d_rad, st);
    if (rc != LUX_OK) return rc;
    return lux_cuda_check(ctx, (int)cudaGetLastError(), "reference launch");
}

extern "C" lux_status lux_error_stats(LuxContext *ctx, const float *estimate, const double *reference, uint32_t count,
                                      double out[4]) {
    if (!ctx || !out || (count && (!estimate || !reference))) return LUX_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    double *d = nullptr;
    lux_status rc = lux_cuda_check(ctx, (int)cudaMallocAsync((void **)&d, 4 * sizeof(double), st), "error: sums");
    if (rc != LUX_OK) return rc;
    cudaMemsetAsync(d, 0, 4 * sizeof(double), st);
    if (count)
        error_stats_kernel<<<std::min((count + 255) / 256, (uint32_t)ctx->sm_count * 4), 256, 0, st>>>(
            (const float4 *)estimate, (const double4 *)reference, count, d);
    cudaMemcpyAsync(out, d, 4 * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(d, st);
    rc = lux_cuda_check(ctx, (int)cudaStreamSynchronize(st), "error stats");
    if (rc != LUX_OK) return rc;
    return lux_cuda_check(ctx, (int)cudaGetLastError(), "error stats launch");
}
