// rate.cu - the device's measured read rate, the denominator of the
// traversal roofline.  The BVH nodes, triangles and instances of a scene stay
// in L2 while the cascade rays are traced, so the traversal kernels are bound
// by the L2 read rate rather than by HBM; this launch measures that rate (a
// buffer well inside L2) or the HBM read rate (a buffer well above it) with
// the same 16-byte loads the node tests issue.
#include <cuda_runtime.h>

#include <algorithm>

#include "lux_internal.h"

namespace {

constexpr int kRateThreads = 512;
constexpr int kRateBlocksPerSm = 4;

// Every pass reads the whole buffer once, grid-strided, four independent
// 16-byte loads in flight per thread.  The loads bypass L1 (ld.global.cg), so
// a buffer that fits in L2 is served by L2 on every pass.  The XOR of every
// word is kept and compared with a constant so no load is dead.
__global__ void __launch_bounds__(kRateThreads, kRateBlocksPerSm)
    read_rate_kernel(const uint4 *__restrict__ buf, unsigned long long n, uint32_t passes, uint32_t *sink) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    const unsigned long long start = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t acc = 0;
    for (uint32_t p = 0; p < passes; ++p) {
        unsigned long long i = start;
        for (; i + 3ull * stride < n; i += 4ull * stride) {
            uint4 a = __ldcg(buf + i), b = __ldcg(buf + i + stride);
            uint4 c = __ldcg(buf + i + 2ull * stride), d = __ldcg(buf + i + 3ull * stride);
            acc ^= (a.x ^ a.y ^ a.z ^ a.w) ^ (b.x ^ b.y ^ b.z ^ b.w) ^ (c.x ^ c.y ^ c.z ^ c.w) ^
                   (d.x ^ d.y ^ d.z ^ d.w);
        }
        for (; i < n; i += stride) {
            uint4 a = __ldcg(buf + i);
            acc ^= a.x ^ a.y ^ a.z ^ a.w;
        }
    }
    if (acc == 0x9e3779b9u) atomicAdd(sink, 1u);
}

}  // namespace

extern "C" lux_status lux_measure_read_rate(LuxContext *ctx, uint64_t bytes, uint32_t passes, double *gb_per_s) {
    if (!ctx || !gb_per_s) return LUX_ERR_INVALID_ARGUMENT;
    *gb_per_s = 0.0;
    if (bytes < (1ull << 20) || bytes % 16u != 0u || bytes > (64ull << 30))
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "measure_read_rate: bytes must be a multiple of 16 in [1 MiB, 64 GiB]");
    if (passes == 0u || passes > 4096u)
        return lux_fail(ctx, LUX_ERR_INVALID_ARGUMENT, "measure_read_rate: passes must be in [1, 4096]");
    lux_status s = lux_cuda_check(ctx, (int)cudaSetDevice(ctx->device), "measure_read_rate set device");
    if (s != LUX_OK) return s;
    void *buf = nullptr;
    uint32_t *sink = nullptr;
    cudaEvent_t begin = nullptr, end = nullptr;
    const cudaStream_t st = ctx->stream;
    const int grid = std::max(ctx->sm_count, 1) * kRateBlocksPerSm;
    const unsigned long long n = bytes / 16u;
    float best = 0.0f;
    s = lux_cuda_check(ctx, (int)cudaMalloc(&buf, bytes), "measure_read_rate buffer");
    if (s == LUX_OK) s = lux_cuda_check(ctx, (int)cudaMalloc((void **)&sink, sizeof(uint32_t)), "measure_read_rate sink");
    if (s == LUX_OK) s = lux_cuda_check(ctx, (int)cudaEventCreate(&begin), "measure_read_rate event");
    if (s == LUX_OK) s = lux_cuda_check(ctx, (int)cudaEventCreate(&end), "measure_read_rate event");
    if (s == LUX_OK) s = lux_cuda_check(ctx, (int)cudaMemsetAsync(buf, 0x5a, bytes, st), "measure_read_rate fill");
    if (s == LUX_OK) s = lux_cuda_check(ctx, (int)cudaMemsetAsync(sink, 0, sizeof(uint32_t), st), "measure_read_rate fill");
    // One warm-up launch (brings the buffer into L2 when it fits), then the
    // shortest of five timed launches.
    for (int trial = 0; trial < 6 && s == LUX_OK; ++trial) {
        if (trial > 0) s = lux_cuda_check(ctx, (int)cudaEventRecord(begin, st), "measure_read_rate record");
        if (s != LUX_OK) break;
        read_rate_kernel<<<grid, kRateThreads, 0, st>>>(static_cast<const uint4 *>(buf), n, passes, sink);
        s = lux_cuda_check(ctx, (int)cudaGetLastError(), "measure_read_rate launch");
        if (s != LUX_OK || trial == 0) continue;
        s = lux_cuda_check(ctx, (int)cudaEventRecord(end, st), "measure_read_rate record");
        if (s == LUX_OK) s = lux_cuda_check(ctx, (int)cudaEventSynchronize(end), "measure_read_rate wait");
        float ms = 0.0f;
        if (s == LUX_OK) s = lux_cuda_check(ctx, (int)cudaEventElapsedTime(&ms, begin, end), "measure_read_rate time");
        if (s == LUX_OK && ms > 0.0f && (best == 0.0f || ms < best)) best = ms;
    }
    if (s == LUX_OK) s = lux_cuda_check(ctx, (int)cudaStreamSynchronize(st), "measure_read_rate synchronize");
    if (begin) cudaEventDestroy(begin);
    if (end) cudaEventDestroy(end);
    if (sink) cudaFree(sink);
    if (buf) cudaFree(buf);
    if (s != LUX_OK) return s;
    if (!(best > 0.0f)) return lux_fail(ctx, LUX_ERR_INTERNAL, "measure_read_rate: no timed launch");
    *gb_per_s = (double)bytes * (double)passes / ((double)best * 1e-3) / 1e9;
    return LUX_OK;
}
