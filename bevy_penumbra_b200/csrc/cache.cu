// cache.cu - learned radiance cache: multiresolution hash encoding, a fused
// 64-wide MLP on the tcgen05 tensor cores, and Adam.
//
// No reference counterpart (the reference's README defers neural caching).
// The design follows the published real-time neural radiance cache recipe
// (Mueller et al. 2021: hash-grid input encoding, small fully fused MLP,
// relative L2 loss, online training), written for sm_100a:
//
//  * One CTA of 128 threads runs a tile of 128 samples.  Every layer is one
//    tcgen05.mma chain (M = 128 samples, N = 64 or 16 outputs, K = 64 or 16)
//    issued by one thread from shared-memory operands in the canonical
//    K-major no-swizzle layout, accumulating FP32 in tensor memory (TMEM,
//    64 columns).  Thread t of warp w reads accumulator row 32 w + t with
//    tcgen05.ld, so each thread owns one sample's row between layers.
//  * The weights live in shared memory for the kernel's lifetime, packed by
//    the Adam step in the same layout, once as W ([out][in]) for the forward
//    pass and once as W^T for the backward data gradients.
//  * Weight gradients g^T h are summed on the CUDA cores from the same
//    shared tiles (fire-and-forget atomics into an FP32 gradient buffer).
//  * Every wait on the tensor cores is bounded; a wait that gives up sets an
//    error flag, the CTA leaves its loop, and TMEM is freed.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "lux_internal.h"
#include "lux_math.cuh"

namespace {

using bf16 = __nv_bfloat16;

constexpr int kLevelsMax = 16;
constexpr int kIn = 64, kHidden = 64, kOut = 16;
constexpr int kHiddenLayers = 4;
constexpr int kTile = 128;
constexpr uint32_t kTmemCols = 64;       // forward kernel: one [128][64] FP32 accumulator
// Training kernel: the layer accumulator (columns 0-63) and the weight
// gradients of the five layers, each an M = 64 accumulator of dW^T (rows =
// layer inputs, columns = outputs): hidden layer l at columns 64 + 64 l, the
// output layer (16 columns) at 320.
constexpr uint32_t kTrainTmemCols = 512;
constexpr uint32_t kGradCol0 = 64;
constexpr int kWHidden = kHidden * kIn;                       // 4096 per hidden layer
constexpr int kWTotal = kHiddenLayers * kWHidden + kOut * kIn;  // 17408
constexpr int kPackedElems = 2 * kWTotal;                     // W and W^T packed
constexpr uint32_t kWaitLimit = 1u << 22;

// Packed element offset of (n, k) in an [N][K] K-major tile: 8 x 8 core
// matrices of 128 bytes, K-adjacent core matrices N/8 * 128 bytes apart
// (leading byte offset), N-adjacent ones 128 bytes apart (stride byte offset).
__host__ __device__ __forceinline__ uint32_t packed(uint32_t n, uint32_t k, uint32_t N) {
    return ((k >> 3) * (N >> 3) + (n >> 3)) * 64u + (n & 7u) * 8u + (k & 7u);
}

// Offsets (elements) of the packed forward tiles W_l [out][in] and the
// backward tiles W_l^T [in][out].
__host__ __device__ __forceinline__ uint32_t fwd_offset(int l) { return (uint32_t)l * kWHidden; }
__host__ __device__ __forceinline__ uint32_t bwd_offset(int l) { return (uint32_t)kWTotal + (uint32_t)l * kWHidden; }

// ---- PTX wrappers ---------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start address, leading and stride byte
// offsets (16-byte units), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 accumulator,
// both operands K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 16 consecutive FP32 accumulator columns of this thread's row.
__device__ __forceinline__ void tmem_load16(uint32_t addr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_load() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// TMEM allocation by warp 0 (address written to shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t cols = kTmemCols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t addr, uint32_t cols = kTmemCols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(addr), "r"(cols) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(1u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Every thread's view of one tensor-core round: the issuing thread has
// committed, all threads wait (bounded), the answer is CTA-uniform.
__device__ __forceinline__ bool wait_round(uint32_t bar, uint32_t &phase) {
    bool ok = mbar_wait(bar, phase);
    phase ^= 1u;
    return __syncthreads_and(ok) != 0;
}

__device__ __forceinline__ void sync_for_mma() {
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

// One layer: D[128 x N] = A[128 x K] * B[N x K]^T from packed shared tiles.
__device__ __forceinline__ void issue_layer(uint32_t tmem, uint32_t a_addr, uint32_t b_addr, uint32_t N, uint32_t K) {
    const uint32_t a_lbo = (kTile / 8) * 128u, b_lbo = (N / 8) * 128u;
    const uint32_t idesc = idesc_bf16(kTile, N);
    for (uint32_t ks = 0; ks < K / 16u; ++ks)
        mma_bf16(tmem, smem_desc(a_addr + ks * 2u * a_lbo, a_lbo, 128u), smem_desc(b_addr + ks * 2u * b_lbo, b_lbo, 128u),
                 idesc, ks > 0u ? 1u : 0u);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&h);
}

// Writes 64 values as this thread's row of a packed [128][64] tile.
__device__ __forceinline__ void store_row64(bf16 *tile, uint32_t row, const float v[64]) {
#pragma unroll
    for (int kg = 0; kg < 8; ++kg) {
        uint4 q;
        q.x = pack_bf16x2(v[kg * 8 + 0], v[kg * 8 + 1]);
        q.y = pack_bf16x2(v[kg * 8 + 2], v[kg * 8 + 3]);
        q.z = pack_bf16x2(v[kg * 8 + 4], v[kg * 8 + 5]);
        q.w = pack_bf16x2(v[kg * 8 + 6], v[kg * 8 + 7]);
        *reinterpret_cast<uint4 *>(tile + packed(row, (uint32_t)kg * 8u, kTile)) = q;
    }
}

__device__ __forceinline__ float bf16_at(const bf16 *tile, uint32_t row, uint32_t col) {
    return __bfloat162float(tile[packed(row, col, kTile)]);
}

// ---- hash encoding ----------------------------------------------------------

struct GridParams {
    float lo[3], inv_extent[3];
    uint32_t levels, table;  // table = entries per level (power of two)
    uint32_t res[kLevelsMax];
};

__device__ __forceinline__ uint32_t grid_index(const GridParams &G, uint32_t level, uint32_t x, uint32_t y, uint32_t z) {
    uint32_t stride = G.res[level] + 1u;
    unsigned long long dense = (unsigned long long)stride * stride * stride;
    if (dense <= G.table) return x + stride * (y + stride * z);
    return (x * 1u ^ y * 2654435761u ^ z * 805459861u) & (G.table - 1u);
}

struct Corner {
    uint32_t index[8];
    float weight[8];
};

__device__ __forceinline__ void level_corners(const GridParams &G, uint32_t level, const float u[3], Corner &c) {
    float res = (float)G.res[level];
    uint32_t i0[3];
    float f[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float p = u[a] * res;
        float fl = floorf(p);
        fl = fminf(fmaxf(fl, 0.0f), res - 1.0f);
        i0[a] = (uint32_t)fl;
        f[a] = fminf(fmaxf(p - fl, 0.0f), 1.0f);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        uint32_t dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
        c.index[k] = level * G.table + grid_index(G, level, i0[0] + dx, i0[1] + dy, i0[2] + dz);
        c.weight[k] = (dx ? f[0] : 1.0f - f[0]) * (dy ? f[1] : 1.0f - f[1]) * (dz ? f[2] : 1.0f - f[2]);
    }
}

__device__ __forceinline__ void unit_position(const GridParams &G, const LuxCacheSample &s, float u[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) u[a] = fminf(fmaxf((s.position[a] - G.lo[a]) * G.inv_extent[a], 0.0f), 1.0f);
}

// Real spherical harmonics of degree < 4 (16 coefficients) of a unit
// direction, in the usual orthonormal basis.
__device__ __forceinline__ void sh16(float x, float y, float z, float *o) {
    float xx = x * x, yy = y * y, zz = z * z;
    o[0] = 0.28209479f;
    o[1] = -0.48860251f * y;
    o[2] = 0.48860251f * z;
    o[3] = -0.48860251f * x;
    o[4] = 1.09254843f * x * y;
    o[5] = -1.09254843f * y * z;
    o[6] = 0.31539157f * (3.0f * zz - 1.0f);
    o[7] = -1.09254843f * x * z;
    o[8] = 0.54627421f * (xx - yy);
    o[9] = -0.59004359f * y * (3.0f * xx - yy);
    o[10] = 2.89061144f * x * y * z;
    o[11] = -0.45704580f * y * (5.0f * zz - 1.0f);
    o[12] = 0.37317633f * z * (5.0f * zz - 3.0f);
    o[13] = -0.45704580f * x * (5.0f * zz - 1.0f);
    o[14] = 1.44530572f * z * (xx - yy);
    o[15] = -0.59004359f * x * (xx - 3.0f * yy);
}

// The 64 BF16 inputs of one sample: 2 hash features per level (32), the
// direction's 16 spherical-harmonic coefficients, normal, albedo, a
// constant 1 (the first layer's bias), zeros.
// n_dev (optional): a device count that caps n (compacted query lists).
__global__ void encode_kernel(GridParams G, const LuxCacheSample *__restrict__ samples, uint32_t n,
                              const uint32_t *__restrict__ n_dev, const __nv_bfloat162 *__restrict__ table,
                              uint4 *__restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (n_dev) n = min(n, *n_dev);
    if (i >= n) return;
    LuxCacheSample s = samples[i];
    float u[3];
    unit_position(G, s, u);
    float v[kIn];
#pragma unroll
    for (int k = 0; k < kIn; ++k) v[k] = 0.0f;
    // Unrolled over the maximum level count so v[] stays in registers.
#pragma unroll
    for (uint32_t level = 0; level < (uint32_t)kLevelsMax; ++level) {
        if (level >= G.levels) break;
        Corner c;
        level_corners(G, level, u, c);
        float f0 = 0.0f, f1 = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            float2 t = __bfloat1622float2(table[c.index[k]]);
            f0 += c.weight[k] * t.x;
            f1 += c.weight[k] * t.y;
        }
        v[2 * level] = f0;
        v[2 * level + 1] = f1;
    }
    const int base = 2 * kLevelsMax;
    sh16(s.direction[0], s.direction[1], s.direction[2], v + base);
    v[base + 16] = s.normal[0];
    v[base + 17] = s.normal[1];
    v[base + 18] = s.normal[2];
    v[base + 19] = s.albedo[0];
    v[base + 20] = s.albedo[1];
    v[base + 21] = s.albedo[2];
    v[base + 22] = 1.0f;
#pragma unroll
    for (int q = 0; q < kIn / 8; ++q) {
        uint4 w;
        w.x = pack_bf16x2(v[q * 8 + 0], v[q * 8 + 1]);
        w.y = pack_bf16x2(v[q * 8 + 2], v[q * 8 + 3]);
        w.z = pack_bf16x2(v[q * 8 + 4], v[q * 8 + 5]);
        w.w = pack_bf16x2(v[q * 8 + 6], v[q * 8 + 7]);
        out[(size_t)i * (kIn / 8) + q] = w;
    }
}

// Scatter of the input gradient to the hash table (same corners).
__global__ void encode_backward_kernel(GridParams G, const LuxCacheSample *__restrict__ samples, uint32_t n,
                                       const float *__restrict__ dx, float2 *__restrict__ grad) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    LuxCacheSample s = samples[i];
    float u[3];
    unit_position(G, s, u);
    for (uint32_t level = 0; level < G.levels; ++level) {
        float g0 = dx[(size_t)i * 2 * kLevelsMax + 2 * level], g1 = dx[(size_t)i * 2 * kLevelsMax + 2 * level + 1];
        if (g0 == 0.0f && g1 == 0.0f) continue;
        Corner c;
        level_corners(G, level, u, c);
#pragma unroll
        for (int k = 0; k < 8; ++k) atomicAdd(&grad[c.index[k]], make_float2(c.weight[k] * g0, c.weight[k] * g1));
    }
}

// ---- fused MLP ----------------------------------------------------------------

struct SmemForward {
    static constexpr uint32_t kW = 0;                              // packed forward weights
    static constexpr uint32_t kA = 35840;                          // [128][64] activation tile
    static constexpr uint32_t kBar = kA + kTile * kIn * 2;         // mbarrier
    static constexpr uint32_t kSlot = kBar + 8;                    // TMEM address
    static constexpr uint32_t kBytes = kSlot + 8;
};

// Inference: out[row] = MLP(x[row]) (rgb; w = 1).  clamp: rgb >= 0.
__global__ void __launch_bounds__(kTile) mlp_forward_kernel(const uint4 *__restrict__ x, uint32_t n,
                                                             const uint32_t *__restrict__ n_dev,
                                                             const uint4 *__restrict__ weights, float4 *__restrict__ out,
                                                             int clamp, uint32_t *__restrict__ error) {
    if (n_dev) n = min(n, *n_dev);
    extern __shared__ __align__(1024) unsigned char smem[];
    bf16 *W = reinterpret_cast<bf16 *>(smem + SmemForward::kW);
    bf16 *A = reinterpret_cast<bf16 *>(smem + SmemForward::kA);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + SmemForward::kBar);
    uint32_t *slot = reinterpret_cast<uint32_t *>(smem + SmemForward::kSlot);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    if (warp == 0) tmem_alloc(slot);
    if (tid == 0) mbar_init(bar);
    for (uint32_t i = tid; i < kWTotal / 8; i += kTile) reinterpret_cast<uint4 *>(W)[i] = weights[i];
    sync_for_mma();
    const uint32_t tmem = *slot;
    const uint32_t lane_addr = tmem + ((warp * 32u) << 16);
    const uint32_t bar_addr = smem_u32(bar), a_addr = smem_u32(A), w_addr = smem_u32(W);
    uint32_t phase = 0;
    bool ok = true;
    for (uint32_t tile = blockIdx.x; ok && tile * kTile < n; tile += gridDim.x) {
        uint32_t row = tile * kTile + tid;
#pragma unroll
        for (int kg = 0; kg < 8; ++kg) {
            uint4 q = row < n ? x[(size_t)row * 8 + kg] : make_uint4(0, 0, 0, 0);
            *reinterpret_cast<uint4 *>(A + packed(tid, (uint32_t)kg * 8u, kTile)) = q;
        }
        for (int l = 0; l <= kHiddenLayers && ok; ++l) {
            sync_for_mma();
            const uint32_t N = l < kHiddenLayers ? kHidden : kOut;
            if (tid == 0) {
                issue_layer(tmem, a_addr, w_addr + fwd_offset(l) * 2u, N, kIn);
                mma_commit(bar_addr);
            }
            ok = wait_round(bar_addr, phase);
            if (!ok) break;
            tc_fence_after();
            if (l < kHiddenLayers) {
                float v[64];
                tmem_load16(lane_addr + 0, v);
                tmem_load16(lane_addr + 16, v + 16);
                tmem_load16(lane_addr + 32, v + 32);
                tmem_load16(lane_addr + 48, v + 48);
                tmem_wait_load();
#pragma unroll
                for (int k = 0; k < 64; ++k) v[k] = fmaxf(v[k], 0.0f);
                store_row64(A, tid, v);
            } else {
                float v[16];
                tmem_load16(lane_addr, v);
                tmem_wait_load();
                if (row < n) {
                    float r = v[0], g = v[1], b = v[2];
                    if (clamp) {
                        r = fmaxf(r, 0.0f);
                        g = fmaxf(g, 0.0f);
                        b = fmaxf(b, 0.0f);
                    }
                    out[row] = make_float4(r, g, b, 1.0f);
                }
            }
        }
    }
    if (!ok && tid == 0) atomicOr(error, 1u);
    if (!ok) mbar_wait(bar_addr, phase ^ 1u);  // let an in-flight chain finish before freeing TMEM
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_free(tmem);
    }
}

static_assert(kPackedElems * 2 == 69632, "packed weights fill the first 68 KiB of shared memory");

struct SmemTrain {
    static constexpr uint32_t kWf = 0;                           // W then W^T tiles (kPackedElems)
    static constexpr uint32_t kH = 69632;                        // 5 x [128][64] activation tiles
    static constexpr uint32_t kHBytes = kTile * kIn * 2;         // 16384
    static constexpr uint32_t kG = kH + 5 * kHBytes;             // [128][64] layer gradient
    static constexpr uint32_t kD = kG + kHBytes;                 // [128][16] output gradient
    static constexpr uint32_t kBar = kD + kTile * kOut * 2;
    static constexpr uint32_t kSlot = kBar + 8;
    static constexpr uint32_t kRed = kSlot + 8;                  // 4 warp partial losses
    static constexpr uint32_t kBytes = kRed + 16;
};

// Weight gradient of one layer on the tensor cores: dW^T[i][o] += sum_b
// h[b][i] g[b][o] over the tile's 128 samples, an M = 64 (inputs) x N (64 or
// 16 outputs) x K = 128 (samples) chain.  Both operands are the activation
// and gradient tiles as they are, read MN-major: in the packed [128][*] tiles
// the feature index is contiguous inside an 8 x 8 core matrix, core matrices
// along the features are kTile / 8 x 128 bytes apart (stride byte offset) and
// along the samples 128 bytes apart (leading byte offset).  The accumulator
// stays in TMEM across the CTA's tiles.
__device__ __forceinline__ void issue_weight_grad(uint32_t tmem_col, uint32_t h_addr, uint32_t g_addr, uint32_t N,
                                                  bool accumulate) {
    const uint32_t lbo = 128u, sbo = (kTile / 8) * 128u;
    const uint32_t idesc = idesc_bf16(64u, N) | (1u << 15) | (1u << 16);  // A and B MN-major
    for (uint32_t ks = 0; ks < (uint32_t)kTile / 16u; ++ks)
        mma_bf16(tmem_col, smem_desc(h_addr + ks * 2u * lbo, lbo, sbo), smem_desc(g_addr + ks * 2u * lbo, lbo, sbo),
                 idesc, (accumulate || ks > 0u) ? 1u : 0u);
}

// Adds one layer's TMEM weight gradient to the FP32 gradient buffer.  The
// M = 64 accumulator keeps row r in TMEM lane 32 (r / 16) + r % 16, so lanes
// 0-15 of warp w hold rows 16 w .. 16 w + 15 (the layer inputs i).
template <int kCols>
__device__ __forceinline__ void flush_weight_grad(uint32_t lane_addr, uint32_t warp, uint32_t lane,
                                                  float *__restrict__ grad) {
    const uint32_t i = warp * 16u + lane;
#pragma unroll
    for (int c0 = 0; c0 < kCols; c0 += 16) {
        float v[16];
        tmem_load16(lane_addr + (uint32_t)c0, v);
        tmem_wait_load();
        if (lane < 16u) {
#pragma unroll
            for (int c = 0; c < 16; ++c)
                if (v[c] != 0.0f) atomicAdd(&grad[(uint32_t)(c0 + c) * kIn + i], v[c]);
        }
    }
}

// One training pass over `n` encoded samples: forward, relative L2 loss,
// backward data gradients and weight gradients on the tensor cores; dx =
// gradient of the hash features (first 32 inputs).
__global__ void __launch_bounds__(kTile) mlp_train_kernel(const uint4 *__restrict__ x, const float4 *__restrict__ target,
                                                           const LuxCacheSample *__restrict__ samples, uint32_t n,
                                                           float scale, const uint4 *__restrict__ weights,
                                                           float *__restrict__ grad_w, float *__restrict__ dx,
                                                           float *__restrict__ loss, uint32_t *__restrict__ error) {
    extern __shared__ __align__(1024) unsigned char smem[];
    bf16 *Wf = reinterpret_cast<bf16 *>(smem + SmemTrain::kWf);
    bf16 *H = reinterpret_cast<bf16 *>(smem + SmemTrain::kH);
    bf16 *G = reinterpret_cast<bf16 *>(smem + SmemTrain::kG);
    bf16 *D = reinterpret_cast<bf16 *>(smem + SmemTrain::kD);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + SmemTrain::kBar);
    uint32_t *slot = reinterpret_cast<uint32_t *>(smem + SmemTrain::kSlot);
    float *red = reinterpret_cast<float *>(smem + SmemTrain::kRed);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    if (warp == 0) tmem_alloc(slot, kTrainTmemCols);
    if (tid == 0) mbar_init(bar);
    for (uint32_t i = tid; i < kPackedElems / 8; i += kTile) reinterpret_cast<uint4 *>(Wf)[i] = weights[i];
    sync_for_mma();
    const uint32_t tmem = *slot;
    const uint32_t lane_addr = tmem + ((warp * 32u) << 16);
    const uint32_t bar_addr = smem_u32(bar);
    const uint32_t w_addr = smem_u32(Wf), h_addr = smem_u32(H), g_addr = smem_u32(G), d_addr = smem_u32(D);
    const uint32_t h_elems = kTile * kIn;
    uint32_t phase = 0;
    bool ok = true, grads = false;  // grads: the TMEM weight gradients hold this CTA's sums
    float loss_sum = 0.0f;
    for (uint32_t tile = blockIdx.x; ok && tile * kTile < n; tile += gridDim.x) {
        const uint32_t row = tile * kTile + tid;
#pragma unroll
        for (int kg = 0; kg < 8; ++kg) {
            uint4 q = row < n ? x[(size_t)row * 8 + kg] : make_uint4(0, 0, 0, 0);
            *reinterpret_cast<uint4 *>(H + packed(tid, (uint32_t)kg * 8u, kTile)) = q;
        }
        // Forward: h_{l+1} = relu(h_l W_l^T), y = h_4 W_4^T.
        float y[16];
        for (int l = 0; l <= kHiddenLayers && ok; ++l) {
            sync_for_mma();
            const uint32_t N = l < kHiddenLayers ? kHidden : kOut;
            if (tid == 0) {
                issue_layer(tmem, h_addr + (uint32_t)l * h_elems * 2u, w_addr + fwd_offset(l) * 2u, N, kIn);
                mma_commit(bar_addr);
            }
            ok = wait_round(bar_addr, phase);
            if (!ok) break;
            tc_fence_after();
            if (l < kHiddenLayers) {
                float v[64];
                tmem_load16(lane_addr + 0, v);
                tmem_load16(lane_addr + 16, v + 16);
                tmem_load16(lane_addr + 32, v + 32);
                tmem_load16(lane_addr + 48, v + 48);
                tmem_wait_load();
#pragma unroll
                for (int k = 0; k < 64; ++k) v[k] = fmaxf(v[k], 0.0f);
                store_row64(H + (uint32_t)(l + 1) * h_elems, tid, v);
            } else {
                tmem_load16(lane_addr, y);
                tmem_wait_load();
            }
        }
        if (!ok) break;
        // Relative L2 loss and its gradient (weighted; rows past n weigh 0).
        float gout[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) gout[c] = 0.0f;
        if (row < n) {
            float w = samples[row].weight;
            float4 t = target[row];
            float tt[3] = {t.x, t.y, t.z};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                float d = y[c] - tt[c];
                float denom = y[c] * y[c] + 0.01f;
                loss_sum += w * d * d / denom;
                gout[c] = w * 2.0f * d / denom * scale;
            }
        }
#pragma unroll
        for (int kg = 0; kg < 2; ++kg) {
            uint4 q;
            q.x = pack_bf16x2(gout[kg * 8 + 0], gout[kg * 8 + 1]);
            q.y = pack_bf16x2(gout[kg * 8 + 2], gout[kg * 8 + 3]);
            q.z = pack_bf16x2(gout[kg * 8 + 4], gout[kg * 8 + 5]);
            q.w = pack_bf16x2(gout[kg * 8 + 6], gout[kg * 8 + 7]);
            *reinterpret_cast<uint4 *>(D + packed(tid, (uint32_t)kg * 8u, kTile)) = q;
        }
        // Backward, layer 4 down to 0: dh_l = g_l W_l (from the packed W_l^T)
        // and dW_l^T += h_l^T g_l, both on the tensor cores in one round.
        for (int l = kHiddenLayers; l >= 0 && ok; --l) {
            sync_for_mma();
            const bool out_layer = l == kHiddenLayers;
            if (tid == 0) {
                const uint32_t grad_tile = out_layer ? d_addr : g_addr;
                issue_layer(tmem, grad_tile, w_addr + bwd_offset(l) * 2u, kIn,
                            out_layer ? (uint32_t)kOut : (uint32_t)kHidden);
                issue_weight_grad(tmem + kGradCol0 + (uint32_t)l * 64u, h_addr + (uint32_t)l * h_elems * 2u, grad_tile,
                                  out_layer ? (uint32_t)kOut : (uint32_t)kHidden, grads);
                mma_commit(bar_addr);
            }
            const bf16 *h = H + (uint32_t)l * h_elems;
            ok = wait_round(bar_addr, phase);  // both chains done: G may be overwritten
            if (!ok) break;
            tc_fence_after();
            float v[64];
            tmem_load16(lane_addr + 0, v);
            tmem_load16(lane_addr + 16, v + 16);
            tmem_load16(lane_addr + 32, v + 32);
            tmem_load16(lane_addr + 48, v + 48);
            tmem_wait_load();
            if (l > 0) {
#pragma unroll
                for (int k = 0; k < 64; ++k) v[k] = bf16_at(h, tid, (uint32_t)k) > 0.0f ? v[k] : 0.0f;
                store_row64(G, tid, v);
            } else if (row < n) {
#pragma unroll
                for (int k = 0; k < 2 * kLevelsMax; ++k) dx[(size_t)row * 2 * kLevelsMax + k] = v[k];
            }
        }
        grads = grads || ok;
    }
    // This CTA's weight gradients, once, from TMEM.
    if (ok && grads) {
        tc_fence_after();
        for (int l = 0; l < kHiddenLayers; ++l)
            flush_weight_grad<kHidden>(lane_addr + kGradCol0 + (uint32_t)l * 64u, warp, tid & 31u,
                                       grad_w + fwd_offset(l));
        flush_weight_grad<kOut>(lane_addr + kGradCol0 + (uint32_t)kHiddenLayers * 64u, warp, tid & 31u,
                                grad_w + fwd_offset(kHiddenLayers));
    }
    for (int off = 16; off > 0; off >>= 1) loss_sum += __shfl_down_sync(0xffffffffu, loss_sum, off);
    if ((tid & 31u) == 0u) red[warp] = loss_sum;
    if (!ok && tid == 0) atomicOr(error, 1u);
    if (!ok) mbar_wait(bar_addr, phase ^ 1u);
    tc_fence_before();
    __syncthreads();
    if (tid == 0) atomicAdd(loss, red[0] + red[1] + red[2] + red[3]);
    if (warp == 0) {
        tc_fence_after();
        tmem_free(tmem, kTrainTmemCols);
    }
}

// ---- Adam ---------------------------------------------------------------------

struct AdamParams {
    float lr, beta1, beta2, eps, correction1, correction2;
};

// Adam on four consecutive parameters per thread (the hash table: n is a
// multiple of 4), with the BF16 copy written as one 8-byte store.  Sparse
// ("lazy") Adam: a parameter this step's samples did not reach (zero
// gradient) keeps its value and moments, so a step reads only the gradients
// of the untouched entries -- a batch reaches a quarter of a fine level's
// entries at most.  A parameter's first update is the dense step's.
//
// The same launch also takes the Adam step of the MLP weights (thread e of
// the grid: weight e, dense Adam, skipping weights whose gradient and first
// moment are both zero: never touched) and writes each weight's BF16 copy into the forward (W) and
// backward (W^T) tile layouts, as pack_weights_kernel does: one launch per
// training step instead of three.
__global__ void adam4_kernel(AdamParams P, float4 *__restrict__ param, float4 *__restrict__ grad,
                             float4 *__restrict__ m, float4 *__restrict__ v, size_t n4, uint2 *__restrict__ out,
                             float *__restrict__ w, float *__restrict__ wg, float *__restrict__ wm,
                             float *__restrict__ wv, bf16 *__restrict__ w_packed) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (w && e < (uint32_t)kWTotal) {
        float p = w[e];
        const float g = wg[e];
        float mi = wm[e], vi = wv[e];
        if (!(g == 0.0f && mi == 0.0f)) {
            wg[e] = 0.0f;
            mi = P.beta1 * mi + (1.0f - P.beta1) * g;
            vi = P.beta2 * vi + (1.0f - P.beta2) * g * g;
            wm[e] = mi;
            wv[e] = vi;
            p = p - P.lr * (mi / P.correction1) / (sqrtf(vi / P.correction2) + P.eps);
            w[e] = p;
        }
        const uint32_t l = e < (uint32_t)(kHiddenLayers * kWHidden) ? e / kWHidden : (uint32_t)kHiddenLayers;
        const uint32_t local = e - l * kWHidden;
        const uint32_t o = local / kIn, i = local % kIn;
        const uint32_t N = l < (uint32_t)kHiddenLayers ? kHidden : kOut;
        const bf16 b = __float2bfloat16_rn(p);
        w_packed[fwd_offset((int)l) + packed(o, i, N)] = b;
        w_packed[bwd_offset((int)l) + packed(i, o, kIn)] = b;
    }
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x) {
        float4 g = grad[i];
        if (g.x == 0.0f && g.y == 0.0f && g.z == 0.0f && g.w == 0.0f) continue;  // not reached this step
        grad[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        float4 mi = m[i], vi = v[i], p = param[i];
        float gs[4] = {g.x, g.y, g.z, g.w}, ms[4] = {mi.x, mi.y, mi.z, mi.w}, vs[4] = {vi.x, vi.y, vi.z, vi.w};
        float ps[4] = {p.x, p.y, p.z, p.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (gs[k] == 0.0f) continue;
            ms[k] = P.beta1 * ms[k] + (1.0f - P.beta1) * gs[k];
            vs[k] = P.beta2 * vs[k] + (1.0f - P.beta2) * gs[k] * gs[k];
            ps[k] = ps[k] - P.lr * (ms[k] / P.correction1) / (sqrtf(vs[k] / P.correction2) + P.eps);
        }
        m[i] = make_float4(ms[0], ms[1], ms[2], ms[3]);
        v[i] = make_float4(vs[0], vs[1], vs[2], vs[3]);
        param[i] = make_float4(ps[0], ps[1], ps[2], ps[3]);
        out[i] = make_uint2(pack_bf16x2(ps[0], ps[1]), pack_bf16x2(ps[2], ps[3]));
    }
}

// Packs the FP32 master weights into the forward (W) and backward (W^T)
// shared-memory tile layouts.
__global__ void pack_weights_kernel(const float *__restrict__ w, bf16 *__restrict__ out) {
    uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (uint32_t)kWTotal) return;
    uint32_t l = e < (uint32_t)(kHiddenLayers * kWHidden) ? e / kWHidden : (uint32_t)kHiddenLayers;
    uint32_t local = e - l * kWHidden;
    uint32_t o = local / kIn, i = local % kIn;
    uint32_t N = l < (uint32_t)kHiddenLayers ? kHidden : kOut;
    bf16 b = __float2bfloat16_rn(w[e]);
    out[fwd_offset((int)l) + packed(o, i, N)] = b;
    out[bwd_offset((int)l) + packed(i, o, kIn)] = b;
}

__global__ void init_uniform_kernel(float *__restrict__ p, size_t n, float scale, uint32_t seed, bf16 *__restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t h = lux::transport_hash((uint32_t)i * 0x9E3779B9u ^ lux::transport_hash(seed + (uint32_t)(i >> 32)));
        float u = (float)(h >> 8) / 16777216.0f;
        float val = (2.0f * u - 1.0f) * scale;
        p[i] = val;
        if (out) out[i] = __float2bfloat16_rn(val);
    }
}

}  // namespace

struct LuxCache {
    LuxContext *ctx = nullptr;
    LuxCacheDesc desc{};
    GridParams grid{};
    size_t table_params = 0;  // levels * table * 2
    float *table_master = nullptr, *table_grad = nullptr, *table_m = nullptr, *table_v = nullptr;
    bf16 *table = nullptr;
    float *w_master = nullptr, *w_grad = nullptr, *w_m = nullptr, *w_v = nullptr;
    bf16 *w_packed = nullptr;
    uint4 *x = nullptr;       // encoded inputs, capacity rows
    float *dx = nullptr;      // batch rows x 32
    uint32_t capacity = 0;
    float *loss = nullptr;    // device scalar
    uint32_t *error = nullptr;
    uint64_t steps = 0, samples = 0;
};

namespace {

void cache_free(LuxCache *c) {
    void *ptrs[] = {c->table_master, c->table_grad, c->table_m, c->table_v, c->table, c->w_master, c->w_grad,
                    c->w_m,          c->w_v,        c->w_packed, c->x,      c->dx,    c->loss,     c->error};
    for (void *p : ptrs)
        if (p) cudaFree(p);
}

lux_status ensure_rows(LuxCache *c, uint32_t rows) {
    if (rows <= c->capacity) return LUX_OK;
    cudaStreamSynchronize(c->ctx->stream);
    if (c->x) cudaFree(c->x);
    c->x = nullptr;
    c->capacity = 0;
    if (cudaMalloc((void **)&c->x, (size_t)rows * kIn * 2) != cudaSuccess) {
        cudaGetLastError();
        return lux_fail(c->ctx, LUX_ERR_OUT_OF_MEMORY, "cache: encoding buffer allocation failed");
    }
    c->capacity = rows;
    return LUX_OK;
}

void set_grid(LuxCache *c, const float lo[3], const float hi[3]) {
    GridParams &G = c->grid;
    for (int a = 0; a < 3; ++a) {
        float ext = hi[a] - lo[a];
        G.lo[a] = lo[a];
        G.inv_extent[a] = ext > 0.0f ? 1.0f / ext : 1.0f;
    }
}

constexpr uint32_t kForwardSmem = SmemForward::kBytes;
constexpr uint32_t kTrainSmem = SmemTrain::kBytes;

}  // namespace

LuxContext *lux_cache_context(const LuxCache *c) { return c ? c->ctx : nullptr; }

extern "C" void lux_cache_desc_default(LuxCacheDesc *d) {
    if (!d) return;
    std::memset(d, 0, sizeof *d);
    d->levels = 16;
    d->log2_table = 19;
    d->base_resolution = 16;
    d->growth = 1.5f;
    d->learning_rate = 1e-3f;
    d->batch = 16384;
    d->seed = 1;
}

extern "C" lux_status lux_cache_create(LuxContext *ctx, const LuxCacheDesc *desc_in, LuxCache **out) {
    if (!ctx || !out) return LUX_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    LuxCacheDesc d;
    if (desc_in)
        d = *desc_in;
    else
        lux_cache_desc_default(&d);
    if (d.levels < 1 || d.levels > (uint32_t)kLevelsMax || d.log2_table < 8 || d.log2_table > 24 ||
        d.base_resolution < 2 || !(d.growth >= 1.0f && d.growth <= 4.0f) || d.batch < kTile ||
        d.batch > (1u << 22) || !(d.learning_rate > 0.0f))
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "cache: descriptor out of range");
    LuxCache *c = new (std::nothrow) LuxCache();
    if (!c) return LUX_ERR_OUT_OF_MEMORY;
    c->ctx = ctx;
    c->desc = d;
    GridParams &G = c->grid;
    G.levels = d.levels;
    G.table = 1u << d.log2_table;
    for (uint32_t l = 0; l < (uint32_t)kLevelsMax; ++l)
        G.res[l] = (uint32_t)std::floor((double)d.base_resolution * std::pow((double)d.growth, (double)l));
    float lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
    set_grid(c, lo, hi);
    c->table_params = (size_t)d.levels * G.table * 2;
    cudaSetDevice(ctx->device);
    size_t tp = c->table_params;
    bool ok = cudaMalloc((void **)&c->table_master, tp * 4) == cudaSuccess &&
              cudaMalloc((void **)&c->table_grad, tp * 4) == cudaSuccess &&
              cudaMalloc((void **)&c->table_m, tp * 4) == cudaSuccess &&
              cudaMalloc((void **)&c->table_v, tp * 4) == cudaSuccess &&
              cudaMalloc((void **)&c->table, tp * 2) == cudaSuccess &&
              cudaMalloc((void **)&c->w_master, kWTotal * 4) == cudaSuccess &&
              cudaMalloc((void **)&c->w_grad, kWTotal * 4) == cudaSuccess &&
              cudaMalloc((void **)&c->w_m, kWTotal * 4) == cudaSuccess &&
              cudaMalloc((void **)&c->w_v, kWTotal * 4) == cudaSuccess &&
              cudaMalloc((void **)&c->w_packed, kPackedElems * 2) == cudaSuccess &&
              cudaMalloc((void **)&c->dx, (size_t)d.batch * 2 * kLevelsMax * 4) == cudaSuccess &&
              cudaMalloc((void **)&c->loss, 16) == cudaSuccess && cudaMalloc((void **)&c->error, 16) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        cache_free(c);
        delete c;
        return lux_fail(ctx, LUX_ERR_OUT_OF_MEMORY, "cache: device allocation failed");
    }
    cudaStream_t st = ctx->stream;
    cudaMemsetAsync(c->table_grad, 0, tp * 4, st);
    cudaMemsetAsync(c->table_m, 0, tp * 4, st);
    cudaMemsetAsync(c->table_v, 0, tp * 4, st);
    cudaMemsetAsync(c->w_grad, 0, kWTotal * 4, st);
    cudaMemsetAsync(c->w_m, 0, kWTotal * 4, st);
    cudaMemsetAsync(c->w_v, 0, kWTotal * 4, st);
    cudaMemsetAsync(c->w_packed, 0, kPackedElems * 2, st);
    cudaMemsetAsync(c->error, 0, 16, st);
    const int grid = ctx->sm_count * 8;
    init_uniform_kernel<<<grid, 256, 0, st>>>(c->table_master, tp, 1e-4f, d.seed, c->table);
    // Hidden layers: uniform +-sqrt(6 / fan_in) (ReLU); output layer a tenth.
    init_uniform_kernel<<<grid, 256, 0, st>>>(c->w_master, (size_t)kHiddenLayers * kWHidden,
                                              std::sqrt(6.0f / kIn), d.seed ^ 0x5bd1e995u, nullptr);
    init_uniform_kernel<<<grid, 256, 0, st>>>(c->w_master + kHiddenLayers * kWHidden, (size_t)kOut * kIn,
                                              0.1f * std::sqrt(6.0f / kIn), d.seed ^ 0x27d4eb2fu, nullptr);
    pack_weights_kernel<<<(kWTotal + 255) / 256, 256, 0, st>>>(c->w_master, c->w_packed);
    cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kForwardSmem);
    cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem);
    lux_status rc = lux_cuda_check(ctx, (int)cudaStreamSynchronize(st), "cache: initialise");
    if (rc != LUX_OK) {
        cache_free(c);
        delete c;
        return rc;
    }
    *out = c;
    return LUX_OK;
}

extern "C" lux_status lux_cache_destroy(LuxCache *c) {
    if (!c) return LUX_OK;
    cudaSetDevice(c->ctx->device);
    cudaStreamSynchronize(c->ctx->stream);
    cache_free(c);
    delete c;
    return LUX_OK;
}

extern "C" lux_status lux_cache_set_bounds(LuxCache *c, const float lo[3], const float hi[3]) {
    if (!c || !lo || !hi) return LUX_ERR_INVALID_ARGUMENT;
    for (int a = 0; a < 3; ++a)
        if (!std::isfinite(lo[a]) || !std::isfinite(hi[a]) || !(hi[a] > lo[a]))
            return lux_fail(c->ctx, LUX_ERR_INVALID_ARGUMENT, "cache: bounds must be finite with hi > lo");
    set_grid(c, lo, hi);
    return LUX_OK;
}

static lux_status cache_forward(LuxCache *c, const uint4 *x, uint32_t count, const uint32_t *count_dev, float *out,
                                int clamp) {
    LuxContext *ctx = c->ctx;
    uint32_t tiles = (count + kTile - 1) / kTile;
    uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)ctx->sm_count * 2u);
    mlp_forward_kernel<<<grid, kTile, kForwardSmem, ctx->stream>>>(x, count, count_dev, (const uint4 *)c->w_packed,
                                                                   (float4 *)out, clamp, c->error);
    return lux_cuda_check(ctx, (int)cudaGetLastError(), "cache: forward launch");
}

extern "C" lux_status lux_cache_encode(LuxCache *c, const LuxCacheSample *samples, uint32_t count, uint16_t *out) {
    if (!c || (count && (!samples || !out))) return LUX_ERR_INVALID_ARGUMENT;
    if (count == 0) return LUX_OK;
    cudaSetDevice(c->ctx->device);
    encode_kernel<<<(count + 127) / 128, 128, 0, c->ctx->stream>>>(
        c->grid, samples, count, nullptr, (const __nv_bfloat162 *)c->table, (uint4 *)out);
    return lux_cuda_check(c->ctx, (int)cudaGetLastError(), "cache: encode launch");
}

extern "C" lux_status lux_cache_forward(LuxCache *c, const uint16_t *encoded, uint32_t count, float *out) {
    if (!c || (count && (!encoded || !out))) return LUX_ERR_INVALID_ARGUMENT;
    if (count == 0) return LUX_OK;
    cudaSetDevice(c->ctx->device);
    return cache_forward(c, (const uint4 *)encoded, count, nullptr, out, 0);
}

extern "C" lux_status lux_cache_query(LuxCache *c, const LuxCacheSample *queries, uint32_t count, float *out) {
    if (!c || (count && (!queries || !out))) return LUX_ERR_INVALID_ARGUMENT;
    if (count == 0) return LUX_OK;
    cudaSetDevice(c->ctx->device);
    lux_status rc = ensure_rows(c, count);
    if (rc != LUX_OK) return rc;
    encode_kernel<<<(count + 127) / 128, 128, 0, c->ctx->stream>>>(c->grid, queries, count, nullptr,
                                                                   (const __nv_bfloat162 *)c->table, c->x);
    return cache_forward(c, c->x, count, nullptr, out, 1);
}

lux_status lux_cache_query_device_count(LuxCache *c, const LuxCacheSample *queries, const uint32_t *count,
                                        uint32_t max_count, float *out) {
    if (!c || !queries || !count || !out) return LUX_ERR_INVALID_ARGUMENT;
    if (max_count == 0) return LUX_OK;
    lux_status rc = ensure_rows(c, max_count);
    if (rc != LUX_OK) return rc;
    encode_kernel<<<(max_count + 127) / 128, 128, 0, c->ctx->stream>>>(c->grid, queries, max_count, count,
                                                                       (const __nv_bfloat162 *)c->table, c->x);
    return cache_forward(c, c->x, max_count, count, out, 1);
}

extern "C" lux_status lux_cache_train(LuxCache *c, const LuxCacheSample *samples, const float *targets, uint32_t count) {
    if (!c || (count && (!samples || !targets))) return LUX_ERR_INVALID_ARGUMENT;
    if (count == 0) return LUX_OK;
    LuxContext *ctx = c->ctx;
    cudaSetDevice(ctx->device);
    const uint32_t batch = c->desc.batch;
    lux_status rc = ensure_rows(c, batch);
    if (rc != LUX_OK) return rc;
    cudaStream_t st = ctx->stream;
    const int grid = ctx->sm_count * 8;
    for (uint32_t s0 = 0; s0 < count; s0 += batch) {
        uint32_t nb = std::min(batch, count - s0);
        const LuxCacheSample *sb = samples + s0;
        encode_kernel<<<(nb + 127) / 128, 128, 0, st>>>(c->grid, sb, nb, nullptr, (const __nv_bfloat162 *)c->table,
                                                        c->x);
        cudaMemsetAsync(c->loss, 0, 4, st);
        uint32_t tiles = (nb + kTile - 1) / kTile;
        mlp_train_kernel<<<std::min<uint32_t>(tiles, (uint32_t)ctx->sm_count), kTile, kTrainSmem, st>>>(
            c->x, (const float4 *)targets + s0, sb, nb, 1.0f / (3.0f * (float)nb), (const uint4 *)c->w_packed,
            c->w_grad, c->dx, c->loss, c->error);
        encode_backward_kernel<<<(nb + 127) / 128, 128, 0, st>>>(c->grid, sb, nb, c->dx, (float2 *)c->table_grad);
        ++c->steps;
        AdamParams P;
        P.lr = c->desc.learning_rate;
        P.beta1 = 0.9f;
        P.beta2 = 0.99f;
        P.eps = 1e-10f;
        P.correction1 = 1.0f - (float)std::pow(0.9, (double)c->steps);
        P.correction2 = 1.0f - (float)std::pow(0.99, (double)c->steps);
        adam4_kernel<<<std::max(grid, (kWTotal + 255) / 256), 256, 0, st>>>(
            P, (float4 *)c->table_master, (float4 *)c->table_grad, (float4 *)c->table_m, (float4 *)c->table_v,
            c->table_params / 4, (uint2 *)c->table, c->w_master, c->w_grad, c->w_m, c->w_v, c->w_packed);
        c->samples += nb;
        rc = lux_cuda_check(ctx, (int)cudaGetLastError(), "cache: train launch");
        if (rc != LUX_OK) return rc;
    }
    return LUX_OK;
}

extern "C" lux_status lux_cache_stats(LuxCache *c, LuxCacheStats *out) {
    if (!c || !out) return LUX_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->ctx->device);
    lux_status rc = lux_cuda_check(c->ctx, (int)cudaStreamSynchronize(c->ctx->stream), "cache: stats");
    if (rc != LUX_OK) return rc;
    float loss = 0.0f;
    uint32_t err = 0;
    cudaMemcpy(&loss, c->loss, 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(&err, c->error, 4, cudaMemcpyDeviceToHost);
    std::memset(out, 0, sizeof *out);
    out->steps = c->steps;
    out->samples = c->samples;
    uint64_t last = c->samples == 0 ? 0 : ((c->samples - 1) % c->desc.batch) + 1;
    out->last_loss = last ? loss / (3.0f * (float)last) : 0.0f;
    out->error_flags = err;
    return lux_cuda_check(c->ctx, (int)cudaGetLastError(), "cache: stats copy");
}

// One training pass without the Adam step (tests): the FP32 weight and
// hash-table gradients of `count` <= batch samples, copied to host memory and
// cleared on the device.
extern "C" lux_status lux_cache_gradients(LuxCache *c, const LuxCacheSample *samples, const float *targets,
                                          uint32_t count, float *grad_weights, float *grad_table) {
    if (!c || !samples || !targets || !grad_weights || !grad_table) return LUX_ERR_INVALID_ARGUMENT;
    if (count == 0 || count > c->desc.batch)
        return lux_fail(c->ctx, LUX_ERR_INVALID_ARGUMENT, "cache: gradients take 1..batch samples");
    LuxContext *ctx = c->ctx;
    cudaSetDevice(ctx->device);
    lux_status rc = ensure_rows(c, c->desc.batch);
    if (rc != LUX_OK) return rc;
    cudaStream_t st = ctx->stream;
    encode_kernel<<<(count + 127) / 128, 128, 0, st>>>(c->grid, samples, count, nullptr,
                                                       (const __nv_bfloat162 *)c->table, c->x);
    cudaMemsetAsync(c->loss, 0, 4, st);
    uint32_t tiles = (count + kTile - 1) / kTile;
    mlp_train_kernel<<<std::min<uint32_t>(tiles, (uint32_t)ctx->sm_count), kTile, kTrainSmem, st>>>(
        c->x, (const float4 *)targets, samples, count, 1.0f / (3.0f * (float)count), (const uint4 *)c->w_packed,
        c->w_grad, c->dx, c->loss, c->error);
    encode_backward_kernel<<<(count + 127) / 128, 128, 0, st>>>(c->grid, samples, count, c->dx,
                                                                (float2 *)c->table_grad);
    rc = lux_cuda_check(ctx, (int)cudaStreamSynchronize(st), "cache: gradients");
    if (rc != LUX_OK) return rc;
    bool ok = cudaMemcpy(grad_weights, c->w_grad, kWTotal * 4, cudaMemcpyDeviceToHost) == cudaSuccess &&
              cudaMemcpy(grad_table, c->table_grad, c->table_params * 4, cudaMemcpyDeviceToHost) == cudaSuccess;
    cudaMemsetAsync(c->w_grad, 0, kWTotal * 4, st);
    cudaMemsetAsync(c->table_grad, 0, c->table_params * 4, st);
    if (!ok) return lux_cuda_check(ctx, (int)cudaGetLastError(), "cache: gradient copy");
    return lux_cuda_check(ctx, (int)cudaStreamSynchronize(st), "cache: gradient clear");
}

// The FP32 master hash table (levels x 2^log2_table x 2 features) in host memory.
extern "C" lux_status lux_cache_read_table(LuxCache *c, float *out) {
    if (!c || !out) return LUX_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->ctx->device);
    lux_status rc = lux_cuda_check(c->ctx, (int)cudaStreamSynchronize(c->ctx->stream), "cache: table");
    if (rc != LUX_OK) return rc;
    return lux_cuda_check(c->ctx, (int)cudaMemcpy(out, c->table_master, c->table_params * 4, cudaMemcpyDeviceToHost),
                          "cache: table copy");
}

extern "C" lux_status lux_cache_read_weights(LuxCache *c, float *out) {
    if (!c || !out) return LUX_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->ctx->device);
    lux_status rc = lux_cuda_check(c->ctx, (int)cudaStreamSynchronize(c->ctx->stream), "cache: weights");
    if (rc != LUX_OK) return rc;
    return lux_cuda_check(c->ctx, (int)cudaMemcpy(out, c->w_master, kWTotal * 4, cudaMemcpyDeviceToHost),
                          "cache: weights copy");
}
