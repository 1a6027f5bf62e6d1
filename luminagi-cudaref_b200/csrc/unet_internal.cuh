// unet_internal.cuh -- the denoiser object shared by unet.cu (forward, C ABI)
// and unet_train.cu (backward, Adam).
#pragma once
#include <cstddef>
#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.h"
#include "unet_conv.cuh"

namespace lg
{
struct LayerDef
{
    int cin_real, cin, cout;
};
// 14 convs in state_dict order; cin is the padded channel count the kernel reads.
constexpr LayerDef kLayers[14] = {
    {3, 16, 32},    {32, 32, 32},   {32, 32, 64},   {64, 64, 64},   {64, 64, 128},  {128, 128, 128}, {128, 128, 256},
    {256, 256, 256}, {384, 384, 128}, {128, 128, 128}, {192, 192, 64}, {64, 64, 64},  {96, 96, 32},   {32, 32, 32}};

struct Buf
{
    void* p = nullptr;
    size_t bytes = 0;
    int ensure(size_t b)
    {
        if (b <= bytes) return LG_OK;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) return set_error(LG_ERR_NOMEM, "cudaMalloc(%zu): %s", b, cudaGetErrorString(e));
        bytes = b;
        return LG_OK;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
};
}  // namespace lg


struct lg_unet
{
    using Buf = lg::Buf;
    int device = 0;
    int in_ch = 3;  // input channels: 3 (colour) or 12 (colour + albedo, normal, position)
    float slope = 0.1f;
    bool bilinear = false;  // decoder upsampling: nearest (reference) or bilinear
    bool log_hdr = false;   // log1p input, log-space residual, expm1 output (HDR variant)
    cudaStream_t stream = nullptr;
    // parameters (FP32, state_dict order) and packed BF16 weights
    Buf params;     // all FP32 params contiguous
    Buf packed[14];
    size_t w_off[14], b_off[14], tail_w_off, tail_b_off, n_params;
    bool packed_ok = false;
    // activations, sized for (N, H, W)
    int aN = 0, aH = 0, aW = 0;
    Buf x0, t1, cat1, p1, t2, cat2, p2, t3, cat3, p3, t4, t5, t6, t7, u1, xin, yout, err;
    Buf lo7, lo9, lo11;  // bilinear mode: low-resolution outputs of the convs before each upsampling
    // Inference with nearest upsampling: u3a, u2a and u1a read the upsampled half of their input as the
    // lower level's output upsampled along x only (uh3, uh2, uh1) and fold their row taps per output-row
    // parity (packed_fold); fold_up = false keeps the 2x2-copied concat halves.
    bool fold_up = true;
    Buf packed_fold[14];
    bool packed_fold_ok = false;  // reset whenever the plain weights are repacked
    Buf uh1, uh2, uh3;
    // training state
    int sm_count = 148;
    Buf grads, adam_m, adam_v, loss;
    Buf packed_dg[17];   // input-gradient weights (see unet_train.cu)
    bool packed_dg_ok = false;
    long long adam_t = 0;
    int gN = 0, gH = 0, gW = 0;
    Buf dz[14], gs1, gs2, gs3, tgt;
    Buf gup;  // bilinear mode: full-resolution gradient of an upsampled concat half
    Buf wpart, bpart, tpart;  // per-CTA partial weight / bias / tail gradients, summed in a fixed order
    // tile shapes (lg::ConvTile; zero = the default heuristic) of the 14 convs and
    // the 16 input-gradient convs, as chosen by lg_unet_autotune
    lg::ConvTile tile[14] = {}, tile_dg[16] = {};
    // autotuning: events recorded around one conv of the forward (probe_layer)
    // or of the backward (probe_dgrad); -1 = none
    int probe_layer = -1, probe_dgrad = -1;
    cudaEvent_t probe_ev0 = nullptr, probe_ev1 = nullptr;
    cudaEvent_t order_ev = nullptr;  // lg_unet_train_step_async: orders the caller's stream and the network's
};

namespace lg
{
// Real input channels of conv `i`: the first takes the network input (padded
// to kLayers[0].cin = 16 channels in the blocked layout), the rest are fixed.
inline int layer_cin_real(const lg_unet* u, int i) { return i == 0 ? u->in_ch : kLayers[i].cin_real; }
// keep_u1: also store u1b's activation (the tail's input), which the
// backward pass reads; inference leaves it out (96 MB at 1728x864).
int unet_forward_device(lg_unet* u, const float* d_x, int N, int H, int W, float* d_y, bool keep_u1 = true);
int unet_pack_all(lg_unet* u);
}  // namespace lg

