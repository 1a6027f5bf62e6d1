// unet_resample.cu -- bilinear 2x upsampling between decoder levels of the
// HDR denoiser variant, and its adjoint for training.
//
// Upsampling follows F.interpolate(scale_factor=2, mode="bilinear",
// align_corners=False): output index d of an axis of input size n reads
// source coordinate max((d + 0.5) / 2 - 0.5, 0), i.e.
//   d = 2i     -> 0.25 * in[i-1] + 0.75 * in[i]      (in[0] alone for i = 0)
//   d = 2i + 1 -> 0.75 * in[i]   + 0.25 * in[i+1]    (in[n-1] alone for i = n-1)
// separably in y and x, in FP32 from the BF16 inputs, rounded once to BF16.
// The adjoint spreads each output gradient back with the same weights; per
// axis, input i collects outputs 2i-1 (0.25, i >= 1), 2i (0.75; 1 at i = 0),
// 2i+1 (0.75; 1 at i = n-1) and 2i+2 (0.25, i <= n-2).  Both kernels move
// 8 channels (16 bytes) per load/store in the channel-blocked layout and are
// bandwidth-bound elementwise passes.
#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "tc_ptx.cuh"
#include "unet_conv.cuh"

namespace lg
{
namespace
{
__device__ __forceinline__ void unpack(uint4 u, float* v)
{
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        const float2 f = __bfloat1622float2(h[i]);
        v[2 * i] = f.x;
        v[2 * i + 1] = f.y;
    }
}
__device__ __forceinline__ uint4 pack(const float* v)
{
    uint4 u;
    uint32_t* w = reinterpret_cast<uint32_t*>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        __nv_bfloat162 b = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
        w[i] = *reinterpret_cast<uint32_t*>(&b);
    }
    return u;
}
__device__ __forceinline__ const uint4* at(const __nv_bfloat16* base, int C, int H, int W, int n, int b, int y, int x)
{
    return reinterpret_cast<const uint4*>(base + ((((size_t)n * (C >> 3) + b) * H + y) * W + x) * 8);
}

// Source rows (i0, i1) and the weight of i1 for output index d of an axis of size n.
__device__ __forceinline__ void src_axis(int d, int n, int& i0, int& i1, float& l1)
{
    const int i = d >> 1;
    if (d & 1)
    {
        i0 = i;
        i1 = i + 1 < n ? i + 1 : i;
        l1 = 0.25f;
    }
    else if (i == 0)
    {
        i0 = i1 = 0;
        l1 = 0.0f;
    }
    else
    {
        i0 = i - 1;
        i1 = i;
        l1 = 0.75f;
    }
}

// Grid (ceil(w / 128), 2h, N * C/8), 128 threads: a thread writes the output
// pixel pair (2i, 2i+1) of row Y, 8 channels, from the source columns
// i-1, i, i+1 of the two source rows (6 loads for 2 outputs, one 32-byte
// store); 32-bit index math from the grid, no divisions.
__global__ void __launch_bounds__(128) up2_kernel(const __nv_bfloat16* __restrict__ in, int N, int C, int h, int w,
                                                  __nv_bfloat16* __restrict__ out, int out_C, int coff)
{
    const int i = blockIdx.x * 128 + threadIdx.x;
    if (i >= w) return;
    const int H = 2 * h, W = 2 * w, CB = C >> 3;
    const int Y = blockIdx.y;
    const int n = blockIdx.z / CB, b = blockIdx.z % CB;
    int y0, y1;
    float ly;
    src_axis(Y, h, y0, y1, ly);
    const float hy = 1.0f - ly;
    // output 2i reads columns (i-1, i) with weight 0.75 on i (column 0 alone at i = 0);
    // output 2i+1 reads (i, i+1) with weight 0.25 on i+1 (column w-1 alone at the end)
    int xa0, xa1, xb0, xb1;
    float la, lb;
    src_axis(2 * i, w, xa0, xa1, la);
    src_axis(2 * i + 1, w, xb0, xb1, lb);
    const float ha = 1.0f - la, hb = 1.0f - lb;
    float p0[8], q0[8], p1[8], q1[8], r0[8], r1[8], o[8], o2[8];
    unpack(__ldg(at(in, C, h, w, n, b, y0, xa0)), p0);  // row y0: columns xa0 (= i-1 or 0), i, xb1 (= i+1 or w-1)
    unpack(__ldg(at(in, C, h, w, n, b, y0, xa1)), q0);
    unpack(__ldg(at(in, C, h, w, n, b, y0, xb1)), r0);
    unpack(__ldg(at(in, C, h, w, n, b, y1, xa0)), p1);
    unpack(__ldg(at(in, C, h, w, n, b, y1, xa1)), q1);
    unpack(__ldg(at(in, C, h, w, n, b, y1, xb1)), r1);
    // xa1 == xb0 == i: the pair's shared column
#pragma unroll
    for (int k = 0; k < 8; ++k)
    {
        o[k] = hy * (ha * p0[k] + la * q0[k]) + ly * (ha * p1[k] + la * q1[k]);
        o2[k] = hy * (hb * q0[k] + lb * r0[k]) + ly * (hb * q1[k] + lb * r1[k]);
    }
    // 2i is even and W = 2w, so the pair starts on a 32-byte boundary
    tc::st_global_v8(out + ((((size_t)n * (out_C >> 3) + (coff >> 3) + b) * H + Y) * W + 2 * i) * 8, pack(o), pack(o2));
}

// Outputs of one axis feeding input i (size n): up to 4 indices and weights.
__device__ __forceinline__ int taps_axis(int i, int n, int* idx, float* wt)
{
    int k = 0;
    if (i >= 1) { idx[k] = 2 * i - 1; wt[k++] = 0.25f; }
    idx[k] = 2 * i;
    wt[k++] = i == 0 ? 1.0f : 0.75f;
    idx[k] = 2 * i + 1;
    wt[k++] = i == n - 1 ? 1.0f : 0.75f;
    if (i <= n - 2) { idx[k] = 2 * i + 2; wt[k++] = 0.25f; }
    return k;
}

// Grid (ceil(w / 128), h, N * C/8), 128 threads: one low-resolution pixel
// (8 channels) per thread.
__global__ void __launch_bounds__(128) up2_adjoint_kernel(const __nv_bfloat16* __restrict__ g_hi, int N, int C, int h,
                                                          int w, const __nv_bfloat16* __restrict__ ref, float slope,
                                                          __nv_bfloat16* __restrict__ g_lo)
{
    const int x = blockIdx.x * 128 + threadIdx.x;
    if (x >= w) return;
    const int H = 2 * h, W = 2 * w, CB = C >> 3;
    const int y = blockIdx.y;
    const int n = blockIdx.z / CB, b = blockIdx.z % CB;
    int iy[4], ix[4];
    float wy[4], wx[4];
    const int ny = taps_axis(y, h, iy, wy), nx = taps_axis(x, w, ix, wx);
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int p = 0; p < ny; ++p)
        for (int q = 0; q < nx; ++q)
        {
            float g[8];
            unpack(__ldg(at(g_hi, C, H, W, n, b, iy[p], ix[q])), g);
            const float wgt = wy[p] * wx[q];
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[k] = fmaf(wgt, g[k], acc[k]);
        }
    float r[8];
    unpack(__ldg(at(ref, C, h, w, n, b, y, x)), r);
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] *= r[k] > 0.0f ? 1.0f : slope;
    *reinterpret_cast<uint4*>(g_lo + ((((size_t)n * CB + b) * h + y) * w + x) * 8) = pack(acc);
}
}  // namespace

cudaError_t bilinear_up2(const __nv_bfloat16* in, int N, int C, int h, int w, __nv_bfloat16* out, int out_C,
                         int coff, cudaStream_t stream)
{
    if (N <= 0 || C <= 0 || h <= 0 || w <= 0 || (C % 8) || (coff % 8) || coff + C > out_C) return cudaErrorInvalidValue;
    if (2 * h > 65535 || (long long)N * (C >> 3) > 65535) return cudaErrorInvalidValue;
    const dim3 grid((unsigned)((w + 127) / 128), (unsigned)(2 * h), (unsigned)(N * (C >> 3)));
    up2_kernel<<<grid, 128, 0, stream>>>(in, N, C, h, w, out, out_C, coff);
    return cudaGetLastError();
}

cudaError_t bilinear_up2_adjoint(const __nv_bfloat16* g_hi, int N, int C, int h, int w, const __nv_bfloat16* ref,
                                 float slope, __nv_bfloat16* g_lo, cudaStream_t stream)
{
    if (N <= 0 || C <= 0 || h <= 0 || w <= 0 || (C % 8)) return cudaErrorInvalidValue;
    if (h > 65535 || (long long)N * (C >> 3) > 65535) return cudaErrorInvalidValue;
    const dim3 grid((unsigned)((w + 127) / 128), (unsigned)h, (unsigned)(N * (C >> 3)));
    up2_adjoint_kernel<<<grid, 128, 0, stream>>>(g_hi, N, C, h, w, ref, slope, g_lo);
    return cudaGetLastError();
}
}  // namespace lg
