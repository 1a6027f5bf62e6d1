// unet_wgrad.cuh -- weight and bias gradients of the 3x3 convolution.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace lg
{
struct WgradArgs
{
    int N, H, W;
    int Cout;       // channels of dZ (multiple of 32)
    int Cin;        // channels of the blocked input X (multiple of 16)
    int Cin_real;   // channels that have weights (<= Cin)
    int rows_per_cta;  // set by the launcher: row groups (of the K-step's rows) per CTA
    float* dw;      // [Cout][Cin_real][3][3], added to
    int* err;
    // Scratch of conv3x3_wgrad_partial_floats() floats: each CTA stores its
    // partial sums there and one pass adds them to dw in a fixed order, so the
    // gradient does not depend on the order the CTAs finish in.
    float* partial;
};

// Floats of WgradArgs::partial the launch for this layer shape needs.
size_t conv3x3_wgrad_partial_floats(int N, int H, int Cout, int Cin, int Cin_real, int sm_count);
// dW += sum over pixels of dZ (x) shifted X; both blocked BF16 at N x C x H x W.
cudaError_t conv3x3_wgrad(const __nv_bfloat16* dz, const __nv_bfloat16* x, const WgradArgs& a, int sm_count,
                          cudaStream_t stream);
// Floats of scratch conv_bias_grad_many needs for C channels in all.
size_t conv_bias_grad_partial_floats(int C);
// One layer's bias gradient in a batched launch: db[c] += sum over the N x HW pixels of dz (blocked BF16).
struct BiasGradJob
{
    const __nv_bfloat16* dz;
    float* db;
    int N, C, HW;
};
constexpr int kMaxBiasJobs = 16;
// Up to kMaxBiasJobs layers in two launches, each channel's sum in a fixed order: kBiasBlocks block partials,
// each over a fixed pixel stride and its warps in order, then the partials in block order; partial holds
// conv_bias_grad_partial_floats(sum of C) floats.
cudaError_t conv_bias_grad_many(const BiasGradJob* jobs, int n, float* partial, cudaStream_t stream);
}  // namespace lg
