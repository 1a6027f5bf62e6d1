// imgops.cu -- image plumbing between the renderer and the denoiser, on the device.
//
//   lg_rgb8_to_f32:  8-bit HWC frames -> FP32 NCHW in [0,1] (u8 / 255, as the
//                    reference's training and denoise scripts read PNGs,
//                    ml/train.py:102-103, tools/denoise.py:34)
//   lg_f32_to_rgb8:  FP32 NCHW -> 8-bit HWC with clip(v,0,1)*255 + 0.5 truncated
//                    (tools/denoise.py:51)
//   lg_accum_to_f32 / lg_f32_tonemap_rgb8: the HDR denoiser's linear input from
//                    the accumulator, and its output tonemapped as tonemap_kernel does
//   lg_gather_crops: square crops of several FP32 NCHW images into one batch
//                    (ml/train.py:104-110 random crops)
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "common.h"

namespace
{
// The four conversions below run one thread per pixel, grid (ceil(H*W / 256),
// n): the pixel's three HWC values and its three NCHW plane entries, with no
// 64-bit divisions in the index math.
__global__ void rgb8_to_f32_kernel(const uint8_t* __restrict__ in, long long HW, float* __restrict__ out)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= HW) return;
    const long long img = blockIdx.y;
#pragma unroll
    for (int c = 0; c < 3; ++c) out[(img * 3 + c) * HW + p] = (float)in[(img * HW + p) * 3 + c] / 255.0f;
}

__global__ void f32_to_rgb8_kernel(const float* __restrict__ in, long long HW, uint8_t* __restrict__ out)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= HW) return;
    const long long img = blockIdx.y;
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
        const float v = fminf(fmaxf(in[(img * 3 + c) * HW + p], 0.0f), 1.0f);
        out[(img * HW + p) * 3 + c] = (uint8_t)(v * 255.0f + 0.5f);
    }
}

// accum (HWC sums over spp) * inv_spp -> FP32 NCHW linear radiance.
__global__ void accum_to_f32_kernel(const float* __restrict__ acc, long long HW, float inv_spp, float* __restrict__ out)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= HW) return;
    const long long img = blockIdx.y;
#pragma unroll
    for (int c = 0; c < 3; ++c) out[(img * 3 + c) * HW + p] = acc[(img * HW + p) * 3 + c] * inv_spp;
}

// FP32 NCHW linear radiance -> HWC u8 with tonemap_kernel's formula.
__global__ void f32_tonemap_kernel(const float* __restrict__ in, long long HW, uint8_t* __restrict__ out)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= HW) return;
    const long long img = blockIdx.y;
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
        const float v = sqrtf(fmaxf(0.0f, fminf(in[(img * 3 + c) * HW + p], 1.0f)));
        out[(img * HW + p) * 3 + c] = (uint8_t)(v * 255.0f);
    }
}

// Grid of the per-pixel conversions.
dim3 px_grid(long long HW, int n) { return dim3((unsigned)((HW + 255) / 256), (unsigned)n); }

struct Crop
{
    int img, y, x;
};

__global__ void gather_kernel(const float* __restrict__ imgs, int H, int W, const Crop* __restrict__ crops, int n,
                              int cs, float* __restrict__ out)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // over n*3*cs*cs
    const long long per = 3LL * cs * cs;
    if (i >= n * per) return;
    const int k = (int)(i / per);
    const long long r = i % per;
    const int c = (int)(r / ((long long)cs * cs));
    const int yy = (int)((r / cs) % cs), xx = (int)(r % cs);
    const Crop cr = crops[k];
    out[i] = imgs[(((long long)cr.img * 3 + c) * H + cr.y + yy) * W + cr.x + xx];
}
}  // namespace

extern "C" {

int lg_rgb8_to_f32(const uint8_t* d_rgb, int n, int h, int w, float* d_out, void* stream)
{
    if (!d_rgb || !d_out || n < 0 || h <= 0 || w <= 0) return lg::set_error(LG_ERR_INVALID, "bad argument");
    if (n == 0) return LG_OK;
    if (n > 65535) return lg::set_error(LG_ERR_INVALID, "at most 65535 images per call");
    rgb8_to_f32_kernel<<<px_grid((long long)h * w, n), 256, 0, (cudaStream_t)stream>>>(d_rgb, (long long)h * w, d_out);
    LG_TRY_CUDA(cudaGetLastError());
    return LG_OK;
}

int lg_f32_to_rgb8(const float* d_in, int n, int h, int w, uint8_t* d_rgb, void* stream)
{
    if (!d_rgb || !d_in || n < 0 || h <= 0 || w <= 0) return lg::set_error(LG_ERR_INVALID, "bad argument");
    if (n == 0) return LG_OK;
    if (n > 65535) return lg::set_error(LG_ERR_INVALID, "at most 65535 images per call");
    f32_to_rgb8_kernel<<<px_grid((long long)h * w, n), 256, 0, (cudaStream_t)stream>>>(d_in, (long long)h * w, d_rgb);
    LG_TRY_CUDA(cudaGetLastError());
    return LG_OK;
}

int lg_accum_to_f32(const float* d_accum, int n, int h, int w, float inv_spp, float* d_out, void* stream)
{
    if (!d_accum || !d_out || n < 0 || h <= 0 || w <= 0) return lg::set_error(LG_ERR_INVALID, "bad argument");
    if (n == 0) return LG_OK;
    if (n > 65535) return lg::set_error(LG_ERR_INVALID, "at most 65535 images per call");
    accum_to_f32_kernel<<<px_grid((long long)h * w, n), 256, 0, (cudaStream_t)stream>>>(d_accum, (long long)h * w,
                                                                                        inv_spp, d_out);
    LG_TRY_CUDA(cudaGetLastError());
    return LG_OK;
}

int lg_f32_tonemap_rgb8(const float* d_in, int n, int h, int w, uint8_t* d_rgb, void* stream)
{
    if (!d_rgb || !d_in || n < 0 || h <= 0 || w <= 0) return lg::set_error(LG_ERR_INVALID, "bad argument");
    if (n == 0) return LG_OK;
    if (n > 65535) return lg::set_error(LG_ERR_INVALID, "at most 65535 images per call");
    f32_tonemap_kernel<<<px_grid((long long)h * w, n), 256, 0, (cudaStream_t)stream>>>(d_in, (long long)h * w, d_rgb);
    LG_TRY_CUDA(cudaGetLastError());
    return LG_OK;
}

int lg_gather_crops(const float* d_images, int n_images, int h, int w, const int32_t* img_idx, const int32_t* ys,
                    const int32_t* xs, int n_crops, int crop, float* d_out, void* stream)
{
    if (!d_images || !d_out || !img_idx || !ys || !xs || n_crops < 0 || crop <= 0)
        return lg::set_error(LG_ERR_INVALID, "bad argument");
    std::vector<Crop> cr((size_t)n_crops);
    for (int k = 0; k < n_crops; ++k)
    {
        if (img_idx[k] < 0 || img_idx[k] >= n_images || ys[k] < 0 || xs[k] < 0 || ys[k] + crop > h || xs[k] + crop > w)
            return lg::set_error(LG_ERR_INVALID, "crop %d out of range", k);
        cr[(size_t)k] = Crop{img_idx[k], ys[k], xs[k]};
    }
    if (n_crops == 0) return LG_OK;
    Crop* d_cr = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    LG_TRY_CUDA(cudaMallocAsync((void**)&d_cr, cr.size() * sizeof(Crop), st));
    cudaError_t e = cudaMemcpyAsync(d_cr, cr.data(), cr.size() * sizeof(Crop), cudaMemcpyHostToDevice, st);
    const long long total = (long long)n_crops * 3 * crop * crop;
    if (e == cudaSuccess)
    {
        gather_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(d_images, h, w, d_cr, n_crops, crop, d_out);
        e = cudaGetLastError();
    }
    cudaFreeAsync(d_cr, st);
    if (e != cudaSuccess) return lg::set_error(LG_ERR_CUDA, "gather_crops: %s", cudaGetErrorString(e));
    if (!stream) LG_TRY_CUDA(cudaStreamSynchronize(st));
    return LG_OK;
}

}  // extern "C"
