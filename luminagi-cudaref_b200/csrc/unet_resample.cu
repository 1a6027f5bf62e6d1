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

__global__ void up2_kernel(const __nv_bfloat16* __restrict__ in, int N, int C, int h, int w,
                           __nv_bfloat16* __restrict__ out, int out_C, int coff)
{
    const int H = 2 * h, W = 2 * w, CB = C >> 3;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // over N * CB * H * W
    if (i >= (long long)N * CB * H * W) return;
    const int X = (int)(i % W);
    const int Y = (int)((i / W) % H);
    const int b = (int)((i / ((long long)W * H)) % CB);
    const int n = (int)(i / ((long long)W * H * CB));
    int y0, y1, x0, x1;
    float ly, lx;
    src_axis(Y, h, y0, y1, ly);
    src_axis(X, w, x0, x1, lx);
    float a[8], bb[8], c[8], d[8], o[8];
    unpack(__ldg(at(in, C, h, w, n, b, y0, x0)), a);
    unpack(__ldg(at(in, C, h, w, n, b, y0, x1)), bb);
    unpack(__ldg(at(in, C, h, w, n, b, y1, x0)), c);
    unpack(__ldg(at(in, C, h, w, n, b, y1, x1)), d);
    const float hy = 1.0f - ly, hx = 1.0f - lx;
#pragma unroll
    for (int k = 0; k < 8; ++k) o[k] = hy * (hx * a[k] + lx * bb[k]) + ly * (hx * c[k] + lx * d[k]);
    *reinterpret_cast<uint4*>(out + ((((size_t)n * (out_C >> 3) + (coff >> 3) + b) * H + Y) * W + X) * 8) = pack(o);
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

__global__ void up2_adjoint_kernel(const __nv_bfloat16* __restrict__ g_hi, int N, int C, int h, int w,
                                   const __nv_bfloat16* __restrict__ ref, float slope,
                                   __nv_bfloat16* __restrict__ g_lo)
{
    const int H = 2 * h, W = 2 * w, CB = C >> 3;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // over N * CB * h * w
    if (i >= (long long)N * CB * h * w) return;
    const int x = (int)(i % w);
    const int y = (int)((i / w) % h);
    const int b = (int)((i / ((long long)w * h)) % CB);
    const int n = (int)(i / ((long long)w * h * CB));
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
    const long long total = (long long)N * (C >> 3) * (2 * h) * (2 * w);
    up2_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(in, N, C, h, w, out, out_C, coff);
    return cudaGetLastError();
}

cudaError_t bilinear_up2_adjoint(const __nv_bfloat16* g_hi, int N, int C, int h, int w, const __nv_bfloat16* ref,
                                 float slope, __nv_bfloat16* g_lo, cudaStream_t stream)
{
    if (N <= 0 || C <= 0 || h <= 0 || w <= 0 || (C % 8)) return cudaErrorInvalidValue;
    const long long total = (long long)N * (C >> 3) * h * w;
    up2_adjoint_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(g_hi, N, C, h, w, ref, slope, g_lo);
    return cudaGetLastError();
}
}  // namespace lg
