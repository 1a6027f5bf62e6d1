// membench.cu -- read-bandwidth probes of the memory levels the trace kernel
// is served from, for its roofline: the device's L2 (a buffer that fits in
// it, read with ld.global.cg, which caches in L2 only) and its L1 (a small
// region per block, read with ld.global.nc, the read-only path the trace
// kernel uses for BVH records and triangles).  HBM copy bandwidth is measured
// elsewhere; these two have no vendor figure to take.
//
// Each probe reads its buffer `passes` times after one untimed pass, between
// CUDA events on one stream, and reports bytes read / elapsed time.  The
// loads feed an XOR that is stored only when it equals a value no buffer
// produces (the buffers are zero-filled), so the compiler keeps every load
// and nothing is written.
#include <cstdint>

#include <cuda_runtime.h>

#include "common.h"

namespace
{
constexpr int kThreads = 256;

__device__ __forceinline__ uint4 ld_cg(const uint4* p)
{
    uint4 v;
    asm volatile("ld.global.cg.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}

// Grid-stride read of n_vec 16-byte words, four independent loads in flight
// per thread per iteration.
__global__ void __launch_bounds__(kThreads) l2_read_kernel(const uint4* __restrict__ p, size_t n_vec, int passes,
                                                          unsigned* __restrict__ sink)
{
    unsigned acc = 0;
    const size_t stride = (size_t)gridDim.x * kThreads;
    const size_t first = (size_t)blockIdx.x * kThreads + threadIdx.x;
    for (int k = 0; k < passes; ++k)
    {
        size_t i = first;
        for (; i + 3 * stride < n_vec; i += 4 * stride)
        {
            const uint4 a = ld_cg(p + i), b = ld_cg(p + i + stride), c = ld_cg(p + i + 2 * stride),
                        d = ld_cg(p + i + 3 * stride);
            acc ^= a.x ^ a.y ^ a.z ^ a.w ^ b.x ^ b.y ^ b.z ^ b.w ^ c.x ^ c.y ^ c.z ^ c.w ^ d.x ^ d.y ^ d.z ^ d.w;
        }
        for (; i < n_vec; i += stride)
        {
            const uint4 a = ld_cg(p + i);
            acc ^= a.x ^ a.y ^ a.z ^ a.w;
        }
    }
    if (acc == 0x9e3779b9u) *sink = acc;
}

// Every block reads the same region of region_vec 16-byte words `passes`
// times through the read-only (L1) path; after the first pass it is
// resident in each SM's L1.
__global__ void __launch_bounds__(kThreads) l1_read_kernel(const uint4* __restrict__ p, int region_vec, int passes,
                                                          unsigned* __restrict__ sink)
{
    unsigned acc = 0;
    for (int k = 0; k < passes; ++k)
    {
#pragma unroll 4
        for (int i = threadIdx.x; i < region_vec; i += kThreads)
        {
            const uint4 a = __ldg(p + i);
            acc ^= a.x ^ a.y ^ a.z ^ a.w;
        }
    }
    if (acc == 0x9e3779b9u) *sink = acc;
}
}  // namespace

extern "C" int lg_measure_read_bandwidth(int device, int level, int64_t bytes, int passes, double* gbs)
{
    if (!gbs || passes < 1 || bytes < 4096 || (level != 1 && level != 2))
        return lg::set_error(LG_ERR_INVALID, "lg_measure_read_bandwidth: level 1 or 2, bytes >= 4096, passes >= 1");
    if (level == 1 && bytes > 48 * 1024)
        return lg::set_error(LG_ERR_INVALID, "lg_measure_read_bandwidth: the L1 region is at most 48 KB");
    int prev = 0;
    LG_TRY_CUDA(cudaGetDevice(&prev));
    LG_TRY_CUDA(cudaSetDevice(device));
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const size_t n_vec = (size_t)bytes / sizeof(uint4);
    void* buf = nullptr;
    unsigned* sink = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = LG_OK;
    float ms = 0.0f;
    cudaError_t e = cudaMalloc(&buf, n_vec * sizeof(uint4));
    if (e == cudaSuccess) e = cudaMalloc(&sink, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaMemsetAsync(buf, 0, n_vec * sizeof(uint4), st);
    // L2: 8 resident blocks per SM keep enough loads in flight; L1: one wave of
    // blocks, 4 per SM, each reading the whole region.
    const int blocks = (level == 2 ? 8 : 4) * (sms > 0 ? sms : 148);
    for (int run = 0; run < 2 && e == cudaSuccess; ++run)
    {
        const int p = run == 0 ? 1 : passes;  // untimed warm-up pass, then the timed passes
        if (run == 1) e = cudaEventRecord(e0, st);
        if (e != cudaSuccess) break;
        if (level == 2) l2_read_kernel<<<blocks, kThreads, 0, st>>>((const uint4*)buf, n_vec, p, sink);
        else l1_read_kernel<<<blocks, kThreads, 0, st>>>((const uint4*)buf, (int)n_vec, p, sink);
        e = cudaGetLastError();
        if (e == cudaSuccess && run == 1) e = cudaEventRecord(e1, st);
    }
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess) rc = lg::set_error(LG_ERR_CUDA, "lg_measure_read_bandwidth: %s", cudaGetErrorString(e));
    else
    {
        const double read = (double)n_vec * sizeof(uint4) * passes * (level == 1 ? (double)blocks : 1.0);
        *gbs = read / (ms * 1e-3) / 1e9;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    cudaFree(sink);
    cudaFree(buf);
    cudaSetDevice(prev);
    return rc;
}
