// unet_train.cu -- backward pass and Adam for the denoiser (reference
// ml/train.py:184-201: L1 loss, loss.backward(), Adam step).
//
// Gradients flow as BF16 tensors in the channel-blocked layout; every GEMM
// accumulates in FP32 and parameters and their gradients stay FP32.
//   * L1 + clamp + tail: one per-pixel kernel (mean |pred - target|, clamp
//     passes the gradient where 0 <= x + tail <= 1, 1x1 tail weight/bias
//     gradients, and the gradient into u1's second conv times act').
//   * Input gradients: the forward tcgen05 convolution with flipped,
//     transposed weights; its epilogue applies act' of the producer's output
//     (kEpiBwdMask), sums the 2x2 children of an upsampled tensor
//     (kEpiBwdSumPool), keeps the skip-connection part (kEpiBwdStore), or routes
//     a pooled gradient to the window maximum and adds the skip part
//     (kEpiBwdUnpool).  Concat inputs are split into their two sources.
//   * Weight gradients: unet_wgrad.cu; bias gradients: a channel reduction.
//   * Adam (betas 0.9/0.999, eps 1e-8, no weight decay, bias-corrected, as
//     torch.optim.Adam) on the FP32 master parameters, then re-packing to BF16.
#include <cmath>
#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "unet_internal.cuh"
#include "unet_wgrad.cuh"

using namespace lg;

namespace
{
typedef __nv_bfloat16 bf;

// Input-gradient convolutions: (forward layer, input-channel slice, epilogue).
struct DgradDef
{
    int layer, ci_lo, ci_cnt, epi;
};
constexpr DgradDef kDgrad[16] = {
    {13, 0, 32, kEpiBwdMask},     {12, 0, 64, kEpiBwdSumPool}, {12, 64, 32, kEpiBwdStore}, {11, 0, 64, kEpiBwdMask},
    {10, 0, 128, kEpiBwdSumPool}, {10, 128, 64, kEpiBwdStore}, {9, 0, 128, kEpiBwdMask},   {8, 0, 256, kEpiBwdSumPool},
    {8, 256, 128, kEpiBwdStore},  {7, 0, 256, kEpiBwdMask},    {6, 0, 128, kEpiBwdUnpool}, {5, 0, 128, kEpiBwdMask},
    {4, 0, 64, kEpiBwdUnpool},    {3, 0, 64, kEpiBwdMask},     {2, 0, 32, kEpiBwdUnpool},  {1, 0, 32, kEpiBwdMask}};

__device__ __forceinline__ float dact(float y, float slope) { return y > 0.0f ? 1.0f : slope; }

// One thread per pixel.  u1: blocked BF16 (32 ch); x, target, pred: FP32 NCHW.
__global__ void tail_backward_kernel(const bf* __restrict__ u1, const float* __restrict__ x, int xC, int log_hdr,
                                     const float* __restrict__ target, const float* __restrict__ tw,
                                     const float* __restrict__ tb, int N, int H, int W, float slope, float inv_numel,
                                     bf* __restrict__ dz, float* __restrict__ partial)
{
    __shared__ float red[8][100];
    const int HW = H * W;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float gtw[96], gtb[3], l = 0.0f;
#pragma unroll
    for (int i = 0; i < 96; ++i) gtw[i] = 0.0f;
    gtb[0] = gtb[1] = gtb[2] = 0.0f;
    if (p < (long long)N * HW)
    {
        const int n = (int)(p / HW), q = (int)(p % HW);
        float v[32];
#pragma unroll
        for (int b = 0; b < 4; ++b)
        {
            const uint4 u = __ldg(reinterpret_cast<const uint4*>(u1 + (((size_t)n * 4 + b) * HW + q) * 8));
            const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
            for (int i = 0; i < 4; ++i)
            {
                const float2 f = __bfloat1622float2(h[i]);
                v[8 * b + 2 * i] = f.x;
                v[8 * b + 2 * i + 1] = f.y;
            }
        }
        float gpre[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            float acc = __ldg(&tb[k]);  // same order as the forward epilogue
#pragma unroll
            for (int c = 0; c < 32; ++c) acc = fmaf(__ldg(&tw[k * 32 + c]), v[c], acc);
            const size_t pi = ((size_t)n * 3 + k) * HW + q;
            const float xv = x[((size_t)n * xC + k) * HW + q];
            // reference: L1(clamp(x + t, 0, 1), target); HDR variant: L1(max(log1p(x) + t, 0), log1p(target))
            const float pre = (log_hdr ? log1pf(xv) : xv) + acc;
            const float pred = log_hdr ? fmaxf(pre, 0.0f) : fminf(fmaxf(pre, 0.0f), 1.0f);
            const float diff = pred - (log_hdr ? log1pf(target[pi]) : target[pi]);
            l += fabsf(diff);
            const float g = (diff > 0.0f ? 1.0f : (diff < 0.0f ? -1.0f : 0.0f)) * inv_numel;
            gpre[k] = (pre >= 0.0f && (log_hdr || pre <= 1.0f)) ? g : 0.0f;
            gtb[k] = gpre[k];
        }
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int c = 0; c < 32; ++c) gtw[k * 32 + c] = gpre[k] * v[c];
        float d[32];
#pragma unroll
        for (int c = 0; c < 32; ++c)
            d[c] = (__ldg(&tw[c]) * gpre[0] + __ldg(&tw[32 + c]) * gpre[1] + __ldg(&tw[64 + c]) * gpre[2]) *
                   dact(v[c], slope);
#pragma unroll
        for (int b = 0; b < 4; ++b)
        {
            __nv_bfloat162 h[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(d[8 * b + 2 * i], d[8 * b + 2 * i + 1]);
            *reinterpret_cast<uint4*>(dz + (((size_t)n * 4 + b) * HW + q) * 8) = *reinterpret_cast<uint4*>(h);
        }
    }
    // block reduction of the 96 + 3 + 1 partial sums
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    auto wsum = [](float t) {
        for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        return t;
    };
#pragma unroll 4
    for (int i = 0; i < 96; ++i)
    {
        const float t = wsum(gtw[i]);
        if (lane == 0) red[warp][i] = t;
    }
    for (int k = 0; k < 3; ++k)
    {
        const float t = wsum(gtb[k]);
        if (lane == 0) red[warp][96 + k] = t;
    }
    const float lt = wsum(l);
    if (lane == 0) red[warp][99] = lt;
    __syncthreads();
    if (threadIdx.x < 100)
    {
        float t = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w][threadIdx.x];
        partial[(size_t)blockIdx.x * 100 + threadIdx.x] = t;  // this block's 96 + 3 + 1 sums
    }
}

// The blocks' partial sums of tail_backward_kernel added in block order:
// 96 tail-weight and 3 tail-bias gradients (added to) and the loss sum (set).
__global__ void tail_reduce_kernel(const float* __restrict__ partial, int blocks, float* __restrict__ dtw,
                                   float* __restrict__ dtb, float* __restrict__ loss)
{
    const int i = threadIdx.x;
    if (i >= 100) return;
    float t = 0.0f;
    for (int b = 0; b < blocks; ++b) t += partial[(size_t)b * 100 + i];
    if (i < 96) dtw[i] += t;
    else if (i < 99) dtb[i - 96] += t;
    else *loss = t;
}

// torch.optim.Adam: m <- b1 m + (1-b1) g; v <- b2 v + (1-b2) g^2;
// p <- p - (lr / (1 - b1^t)) * m / (sqrt(v) / sqrt(1 - b2^t) + eps).
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps, float bc1,
                            float bc2_sqrt)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = m[i] + (1.0f - b1) * (gi - m[i]);
    const float vi = v[i] * b2 + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float denom = sqrtf(vi) / bc2_sqrt + eps;
    p[i] -= (lr / bc1) * mi / denom;
}

int ensure_train(lg_unet* u, int N, int H, int W)
{
    const size_t np = u->n_params;
    LG_TRY(u->grads.ensure(np * sizeof(float)));
    if (!u->adam_m.p)
    {
        LG_TRY(u->adam_m.ensure(np * sizeof(float)));
        LG_TRY(u->adam_v.ensure(np * sizeof(float)));
        LG_TRY_CUDA(cudaMemsetAsync(u->adam_m.p, 0, np * sizeof(float), u->stream));
        LG_TRY_CUDA(cudaMemsetAsync(u->adam_v.p, 0, np * sizeof(float), u->stream));
    }
    LG_TRY(u->loss.ensure(sizeof(float)));
    if (u->gN == N && u->gH == H && u->gW == W) return LG_OK;
    const size_t px = (size_t)N * H * W, b2 = sizeof(bf);
    const size_t lvl[4] = {px, px / 4, px / 16, px / 64};
    const int lv[14] = {0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 0, 0};  // output level of each layer
    for (int i = 0; i < 14; ++i) LG_TRY(u->dz[i].ensure(lvl[lv[i]] * kLayers[i].cout * b2));
    LG_TRY(u->gs1.ensure(px * 32 * b2));
    LG_TRY(u->gs2.ensure(px / 4 * 64 * b2));
    LG_TRY(u->gs3.ensure(px / 16 * 128 * b2));
    if (u->bilinear) LG_TRY(u->gup.ensure(px * 64 * b2));  // largest upsampled half: 64 ch at full size
    u->gN = N;
    u->gH = H;
    u->gW = W;
    return LG_OK;
}

// The 16 input-gradient convs' packed weights, in one launch.
int pack_dgrad(lg_unet* u)
{
    if (u->packed_dg_ok) return LG_OK;
    ConvPackJob jobs[16];
    for (int k = 0; k < 16; ++k)
    {
        const DgradDef& d = kDgrad[k];
        const LayerDef& L = kLayers[d.layer];
        LG_TRY(u->packed_dg[k].ensure(conv_packed_elems(L.cout, d.ci_cnt) * sizeof(bf)));
        jobs[k] = conv_pack_job_dgrad((const float*)u->params.p + u->w_off[d.layer], L.cout,
                                      layer_cin_real(u, d.layer), d.ci_lo, d.ci_cnt, (bf*)u->packed_dg[k].p,
                                      u->tile_dg[k]);
    }
    LG_TRY_CUDA(conv_pack_many(jobs, 16, u->stream));
    u->packed_dg_ok = true;
    return LG_OK;
}

// Forward (activations kept), L1 loss and every parameter gradient into u->grads.
int loss_and_grads(lg_unet* u, const float* d_x, const float* d_t, int N, int H, int W, float* loss_host)
{
    LG_TRY(ensure_train(u, N, H, W));
    LG_TRY(u->yout.ensure((size_t)N * 3 * H * W * sizeof(float)));
    LG_TRY(unet_forward_device(u, d_x, N, H, W, (float*)u->yout.p));
    LG_TRY(pack_dgrad(u));
    cudaStream_t st = u->stream;
    float* G = (float*)u->grads.p;
    const float* P = (const float*)u->params.p;
    LG_TRY_CUDA(cudaMemsetAsync(G, 0, u->n_params * sizeof(float), st));
    LG_TRY_CUDA(cudaMemsetAsync(u->loss.p, 0, sizeof(float), st));
    const long long npx = (long long)N * H * W;
    const float inv_numel = 1.0f / (float)(npx * 3);
    const int tail_blocks = (int)((npx + 255) / 256);
    LG_TRY(u->tpart.ensure((size_t)tail_blocks * 100 * sizeof(float)));
    tail_backward_kernel<<<(unsigned)tail_blocks, 256, 0, st>>>(
        (const bf*)u->u1.p, d_x, u->in_ch, u->log_hdr ? 1 : 0, d_t, P + u->tail_w_off, P + u->tail_b_off, N, H, W, u->slope, inv_numel,
        (bf*)u->dz[13].p, (float*)u->tpart.p);
    LG_TRY_CUDA(cudaGetLastError());
    tail_reduce_kernel<<<1, 128, 0, st>>>((const float*)u->tpart.p, tail_blocks, G + u->tail_w_off,
                                          G + u->tail_b_off, (float*)u->loss.p);
    LG_TRY_CUDA(cudaGetLastError());

    const int hs[4] = {H, H / 2, H / 4, H / 8}, ws[4] = {W, W / 2, W / 4, W / 8};
    const int lv_out[14] = {0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 0, 0};
    // forward inputs of each layer (blocked BF16)
    const void* in_of[14] = {u->x0.p, u->t1.p, u->p1.p, u->t2.p, u->p2.p, u->t3.p, u->p3.p,
                             u->t4.p, u->cat3.p, u->t5.p, u->cat2.p, u->t6.p, u->cat1.p, u->t7.p};
    auto wgrad = [&](int L) -> int {
        const int lv = lv_out[L];
        WgradArgs a{};
        a.N = N;
        a.H = hs[lv];
        a.W = ws[lv];
        a.Cout = kLayers[L].cout;
        a.Cin = kLayers[L].cin;
        a.Cin_real = layer_cin_real(u, L);
        a.dw = G + u->w_off[L];
        a.err = (int*)u->err.p;
        LG_TRY(u->wpart.ensure(conv3x3_wgrad_partial_floats(N, a.H, a.Cout, a.Cin, a.Cin_real, u->sm_count) *
                               sizeof(float)));
        a.partial = (float*)u->wpart.p;
        LG_TRY_CUDA(conv3x3_wgrad((const bf*)u->dz[L].p, (const bf*)in_of[L], a, u->sm_count, st));
        return LG_OK;
    };
    auto dgrad = [&](int k, void* out, int out_c, const void* ref, int ref_c, int ref_coff, const void* skip,
                     int skip_c, int epi = -1) -> int {
        const DgradDef& d = kDgrad[k];
        const int lv = lv_out[d.layer];  // the backward conv runs at the forward layer's resolution
        ConvArgs a{};
        a.N = N;
        a.H = hs[lv];
        a.W = ws[lv];
        a.Cin = kLayers[d.layer].cout;
        a.Cout = d.ci_cnt;
        a.wpack = (const bf*)u->packed_dg[k].p;
        a.slope = u->slope;
        a.epilogue = epi >= 0 ? epi : d.epi;
        a.out = (bf*)out;
        a.out_C = out_c;
        a.out_coff = 0;
        a.ref = (const bf*)ref;
        a.ref_C = ref_c;
        a.ref_coff = ref_coff;
        a.skip = (const bf*)skip;
        a.skip_C = skip_c;
        a.skip_coff = 0;
        a.err = (int*)u->err.p;
        a.tile = u->tile_dg[k];
        const bool probe = k == u->probe_dgrad;
        if (probe) LG_TRY_CUDA(cudaEventRecord(u->probe_ev0, st));
        LG_TRY_CUDA(conv3x3_forward((const bf*)u->dz[d.layer].p, a, st));
        if (probe) LG_TRY_CUDA(cudaEventRecord(u->probe_ev1, st));
        return LG_OK;
    };
    // decoder, from the output back
    LG_TRY(wgrad(13));
    LG_TRY(dgrad(0, u->dz[12].p, 32, u->t7.p, 32, 0, nullptr, 0));
    LG_TRY(wgrad(12));
    // Gradient of an upsampled concat half back to the low-resolution conv
    // output: the 2x2 sum of nearest upsampling fused in the epilogue, or
    // (bilinear) the full-resolution gradient stored and passed through the
    // upsampling's adjoint, each times act' of the stored output.
    auto up_grad = [&](int k, int layer, void* cat, int cat_c, const Buf& lo, int c, int h, int w) -> int {
        if (!u->bilinear) return dgrad(k, u->dz[layer].p, c, cat, cat_c, 0, nullptr, 0);
        LG_TRY(dgrad(k, u->gup.p, c, nullptr, 0, 0, nullptr, 0, kEpiBwdStore));
        LG_TRY_CUDA(bilinear_up2_adjoint((const bf*)u->gup.p, N, c, h, w, (const bf*)lo.p, u->slope,
                                         (bf*)u->dz[layer].p, st));
        return LG_OK;
    };
    LG_TRY(up_grad(1, 11, u->cat1.p, 96, u->lo11, 64, H / 2, W / 2));
    LG_TRY(dgrad(2, u->gs1.p, 32, nullptr, 0, 0, nullptr, 0));
    LG_TRY(wgrad(11));
    LG_TRY(dgrad(3, u->dz[10].p, 64, u->t6.p, 64, 0, nullptr, 0));
    LG_TRY(wgrad(10));
    LG_TRY(up_grad(4, 9, u->cat2.p, 192, u->lo9, 128, H / 4, W / 4));
    LG_TRY(dgrad(5, u->gs2.p, 64, nullptr, 0, 0, nullptr, 0));
    LG_TRY(wgrad(9));
    LG_TRY(dgrad(6, u->dz[8].p, 128, u->t5.p, 128, 0, nullptr, 0));
    LG_TRY(wgrad(8));
    LG_TRY(up_grad(7, 7, u->cat3.p, 384, u->lo7, 256, H / 8, W / 8));
    LG_TRY(dgrad(8, u->gs3.p, 128, nullptr, 0, 0, nullptr, 0));
    // encoder
    LG_TRY(wgrad(7));
    LG_TRY(dgrad(9, u->dz[6].p, 256, u->t4.p, 256, 0, nullptr, 0));
    LG_TRY(wgrad(6));
    LG_TRY(dgrad(10, u->dz[5].p, 128, u->cat3.p, 384, 256, u->gs3.p, 128));
    LG_TRY(wgrad(5));
    LG_TRY(dgrad(11, u->dz[4].p, 128, u->t3.p, 128, 0, nullptr, 0));
    LG_TRY(wgrad(4));
    LG_TRY(dgrad(12, u->dz[3].p, 64, u->cat2.p, 192, 128, u->gs2.p, 64));
    LG_TRY(wgrad(3));
    LG_TRY(dgrad(13, u->dz[2].p, 64, u->t2.p, 64, 0, nullptr, 0));
    LG_TRY(wgrad(2));
    LG_TRY(dgrad(14, u->dz[1].p, 32, u->cat1.p, 96, 64, u->gs1.p, 32));
    LG_TRY(wgrad(1));
    LG_TRY(dgrad(15, u->dz[0].p, 32, u->t1.p, 32, 0, nullptr, 0));
    LG_TRY(wgrad(0));
    // every layer's bias gradient from its kept dZ, in one batched pass (the same sums as one pass per layer)
    BiasGradJob bj[14];
    int bias_c = 0;
    for (int L = 0; L < 14; ++L)
    {
        const int lv = lv_out[L];
        bj[L] = BiasGradJob{(const bf*)u->dz[L].p, G + u->b_off[L], N, kLayers[L].cout, hs[lv] * ws[lv]};
        bias_c += kLayers[L].cout;
    }
    LG_TRY(u->bpart.ensure(conv_bias_grad_partial_floats(bias_c) * sizeof(float)));
    LG_TRY_CUDA(conv_bias_grad_many(bj, 14, (float*)u->bpart.p, st));
    if (loss_host)
    {
        float s = 0.0f;
        LG_TRY_CUDA(cudaMemcpyAsync(&s, u->loss.p, sizeof(float), cudaMemcpyDeviceToHost, st));
        LG_TRY_CUDA(cudaStreamSynchronize(st));
        *loss_host = s * inv_numel;
    }
    return LG_OK;
}

int adam_step(lg_unet* u, float lr)
{
    u->adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float bc1 = 1.0f - (float)std::pow(0.9, (double)u->adam_t);
    const float bc2 = 1.0f - (float)std::pow(0.999, (double)u->adam_t);
    const size_t n = u->n_params;
    adam_kernel<<<(unsigned)((n + 255) / 256), 256, 0, u->stream>>>((float*)u->params.p, (const float*)u->grads.p,
                                                                    (float*)u->adam_m.p, (float*)u->adam_v.p, n, lr, b1,
                                                                    b2, eps, bc1, sqrtf(bc2));
    LG_TRY_CUDA(cudaGetLastError());
    u->packed_ok = false;
    u->packed_dg_ok = false;
    LG_TRY(unet_pack_all(u));
    return LG_OK;
}

// *dst += *sum * scale (one thread): the batch loss into a caller's device accumulator.
__global__ void loss_add_kernel(const float* __restrict__ sum, float scale, float* __restrict__ dst)
{
    *dst += *sum * scale;
}

int check_err(lg_unet* u)
{
    int err = 0;
    LG_TRY_CUDA(cudaMemcpyAsync(&err, u->err.p, sizeof(int), cudaMemcpyDeviceToHost, u->stream));
    LG_TRY_CUDA(cudaStreamSynchronize(u->stream));
    if (err) return set_error(LG_ERR_DEVICE, "a tensor-core kernel reported wait timeout %d", err);
    return LG_OK;
}
}  // namespace

extern "C" {

int lg_unet_train_step(lg_unet* u, const float* d_x, const float* d_target, int n, int h, int w, float lr,
                       float* loss_out)
{
    if (!u || !d_x || !d_target) return set_error(LG_ERR_INVALID, "NULL argument");
    float loss = 0.0f;
    LG_TRY(loss_and_grads(u, d_x, d_target, n, h, w, loss_out ? &loss : nullptr));
    LG_TRY(adam_step(u, lr));
    LG_TRY(check_err(u));
    if (loss_out) *loss_out = loss;
    return LG_OK;
}

int lg_unet_train_step_async(lg_unet* u, const float* d_x, const float* d_target, int n, int h, int w, float lr,
                             float* d_loss_sum, void* stream)
{
    if (!u || !d_x || !d_target) return set_error(LG_ERR_INVALID, "NULL argument");
    if (!u->order_ev) LG_TRY_CUDA(cudaEventCreateWithFlags(&u->order_ev, cudaEventDisableTiming));
    cudaEvent_t ev = u->order_ev;
    LG_TRY_CUDA(cudaEventRecord(ev, (cudaStream_t)stream));
    LG_TRY_CUDA(cudaStreamWaitEvent(u->stream, ev, 0));
    int rc = loss_and_grads(u, d_x, d_target, n, h, w, nullptr);
    if (rc == LG_OK && d_loss_sum)
    {
        // u->loss holds the summed |difference| of this batch; the mean times n
        const float inv_numel = 1.0f / (float)((long long)n * h * w * 3);  // as loss_and_grads scales it
        loss_add_kernel<<<1, 1, 0, u->stream>>>((const float*)u->loss.p, inv_numel * (float)n, d_loss_sum);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = set_error(LG_ERR_CUDA, "loss: %s", cudaGetErrorString(e));
    }
    if (rc == LG_OK) rc = adam_step(u, lr);
    // later work on the caller's stream waits for this step (also after an error, for what was queued)
    const cudaError_t e1 = cudaEventRecord(ev, u->stream);
    const cudaError_t e2 = e1 == cudaSuccess ? cudaStreamWaitEvent((cudaStream_t)stream, ev, 0) : e1;
    if (rc == LG_OK && e2 != cudaSuccess) rc = set_error(LG_ERR_CUDA, "stream order: %s", cudaGetErrorString(e2));
    return rc;
}

int lg_unet_sync(lg_unet* u)
{
    if (!u) return set_error(LG_ERR_INVALID, "NULL argument");
    return check_err(u);
}

int lg_unet_loss_grad(lg_unet* u, const float* d_x, const float* d_target, int n, int h, int w, float* grads_host,
                      float* loss_out)
{
    if (!u || !d_x || !d_target) return set_error(LG_ERR_INVALID, "NULL argument");
    float loss = 0.0f;
    LG_TRY(loss_and_grads(u, d_x, d_target, n, h, w, &loss));
    if (grads_host)
        LG_TRY_CUDA(cudaMemcpyAsync(grads_host, u->grads.p, u->n_params * sizeof(float), cudaMemcpyDeviceToHost,
                                    u->stream));
    LG_TRY(check_err(u));
    if (loss_out) *loss_out = loss;
    return LG_OK;
}

int lg_unet_adam_apply(lg_unet* u, float lr)
{
    if (!u) return set_error(LG_ERR_INVALID, "NULL argument");
    if (!u->grads.p || !u->adam_m.p) return set_error(LG_ERR_INVALID, "no gradients yet: call lg_unet_loss_grad first");
    LG_TRY(adam_step(u, lr));
    return check_err(u);
}

int lg_unet_autotune(lg_unet* u, int n, int h, int w, int flags, int32_t* tiles_out)
{
    if (!u || n <= 0 || h <= 0 || w <= 0 || (h % 8) || (w % 8)) return set_error(LG_ERR_INVALID, "bad argument");
    if (!u->probe_ev0)
    {
        LG_TRY_CUDA(cudaEventCreate(&u->probe_ev0));
        LG_TRY_CUDA(cudaEventCreate(&u->probe_ev1));
    }
    // Inputs of the real shapes (values do not change the timing): x in [0,1), target 0.
    const size_t xin = (size_t)n * u->in_ch * h * w, xout = (size_t)n * 3 * h * w;
    Buf x, t, y;
    LG_TRY(x.ensure(xin * sizeof(float)));
    LG_TRY(t.ensure(xout * sizeof(float)));
    LG_TRY(y.ensure(xout * sizeof(float)));
    LG_TRY_CUDA(cudaMemsetAsync(x.p, 0, xin * sizeof(float), u->stream));
    LG_TRY_CUDA(cudaMemsetAsync(t.p, 0, xout * sizeof(float), u->stream));
    auto time_probe = [&](bool backward, float& best) -> int {
        best = 1e30f;
        for (int rep = 0; rep < 3; ++rep)
        {
            if (backward) LG_TRY(loss_and_grads(u, (const float*)x.p, (const float*)t.p, n, h, w, nullptr));
            else LG_TRY(unet_forward_device(u, (const float*)x.p, n, h, w, (float*)y.p, false));
            LG_TRY_CUDA(cudaStreamSynchronize(u->stream));
            float ms = 0.0f;
            LG_TRY_CUDA(cudaEventElapsedTime(&ms, u->probe_ev0, u->probe_ev1));
            if (rep > 0 && ms < best) best = ms;  // the first run warms the new shape
        }
        return LG_OK;
    };
    int rc = LG_OK;
    const int n_sets = (flags & LG_UNET_TUNE_BACKWARD) ? 2 : 1;
    for (int set = 0; set < n_sets && rc == LG_OK; ++set)
    {
        const bool bwd = set == 1;
        const int count = bwd ? 16 : 14;
        for (int i = 0; i < count && rc == LG_OK; ++i)
        {
            const int cin = bwd ? kLayers[kDgrad[i].layer].cout : kLayers[i].cin;
            const int cout = bwd ? kDgrad[i].ci_cnt : kLayers[i].cout;
            ConvTile cand[32];
            const int nc = conv_tile_candidates(cin, cout, cand, 32);
            ConvTile& slot = bwd ? u->tile_dg[i] : u->tile[i];
            ConvTile best = conv_default_tile(cin, cout);
            float best_ms = 1e30f;
            (bwd ? u->probe_dgrad : u->probe_layer) = i;
            for (int c = 0; c < nc && rc == LG_OK; ++c)
            {
                slot = cand[c];
                u->packed_ok = false;
                u->packed_dg_ok = false;
                float ms = 0.0f;
                rc = time_probe(bwd, ms);
                if (rc == LG_OK && ms < best_ms)
                {
                    best_ms = ms;
                    best = cand[c];
                }
            }
            slot = best;
            u->probe_layer = u->probe_dgrad = -1;
        }
    }
    u->probe_layer = u->probe_dgrad = -1;
    u->packed_ok = false;
    u->packed_dg_ok = false;
    // Autotuning ran training passes: leave the optimiser state and gradients as they were.
    if (u->adam_m.p)
    {
        cudaMemsetAsync(u->adam_m.p, 0, u->n_params * sizeof(float), u->stream);
        cudaMemsetAsync(u->adam_v.p, 0, u->n_params * sizeof(float), u->stream);
    }
    u->adam_t = 0;
    if (rc == LG_OK) rc = unet_pack_all(u);
    if (rc == LG_OK && tiles_out)
        for (int i = 0; i < 30; ++i)
        {
            const ConvTile& tt = i < 14 ? u->tile[i] : u->tile_dg[i - 14];
            const int cin = i < 14 ? kLayers[i].cin : kLayers[kDgrad[i - 14].layer].cout;
            const int cout = i < 14 ? kLayers[i].cout : kDgrad[i - 14].ci_cnt;
            const ConvTile r = tt.bn ? tt : conv_default_tile(cin, cout);
            tiles_out[4 * i] = r.bn;
            tiles_out[4 * i + 1] = r.kc;
            tiles_out[4 * i + 2] = r.stages;
            tiles_out[4 * i + 3] = r.persist;
        }
    x.release();
    t.release();
    y.release();
    if (rc == LG_OK) LG_TRY_CUDA(cudaStreamSynchronize(u->stream));
    return rc;
}

int lg_unet_set_fold_upsampling(lg_unet* u, int on)
{
    if (!u) return set_error(LG_ERR_INVALID, "NULL argument");
    u->fold_up = on != 0;
    u->packed_fold_ok = false;  // which layers fold has changed
    return LG_OK;
}

int lg_unet_set_tiles(lg_unet* u, const int32_t* tiles)
{
    if (!u || !tiles) return set_error(LG_ERR_INVALID, "NULL argument");
    ConvTile fwd[14], bwd[16];
    for (int i = 0; i < 30; ++i)
    {
        const int p4 = tiles[4 * i + 3];
        if (p4 < 0 || p4 > 7) return set_error(LG_ERR_INVALID, "conv %d: kernel choice %d is not 0..7", i, p4);
        ConvTile t{tiles[4 * i], tiles[4 * i + 1], tiles[4 * i + 2], p4};
        const bool back = i >= 14;
        const int cin = back ? kLayers[kDgrad[i - 14].layer].cout : kLayers[i].cin;
        const int cout = back ? kDgrad[i - 14].ci_cnt : kLayers[i].cout;
        bool ok = false;
        if (t.bn == 0)  // the default shape, on the kernel the fourth value selects
        {
            const int persist = t.persist;
            t = conv_default_tile(cin, cout);
            t.persist = persist;
            ok = persist < 2;  // the resident-weights kernels are compiled for some shapes only
        }
        ConvTile cand[32];
        const int nc = conv_tile_candidates(cin, cout, cand, 32);
        for (int c = 0; c < nc && !ok; ++c)
            ok = cand[c].bn == t.bn && cand[c].kc == t.kc && cand[c].stages == t.stages && cand[c].persist == t.persist;
        if (!ok)
            return set_error(LG_ERR_INVALID, "conv %d: (%d, %d, %d, %d) is not a compiled tile for %d -> %d channels", i,
                             t.bn, t.kc, t.stages, t.persist, cin, cout);
        (back ? bwd[i - 14] : fwd[i]) = t;
    }
    for (int i = 0; i < 14; ++i) u->tile[i] = fwd[i];
    for (int i = 0; i < 16; ++i) u->tile_dg[i] = bwd[i];
    u->packed_ok = false;
    u->packed_dg_ok = false;
    LG_TRY(unet_pack_all(u));
    LG_TRY_CUDA(cudaStreamSynchronize(u->stream));
    return LG_OK;
}

int lg_unet_adam_reset(lg_unet* u)
{
    if (!u) return set_error(LG_ERR_INVALID, "NULL argument");
    u->adam_t = 0;
    if (u->adam_m.p)
    {
        LG_TRY_CUDA(cudaMemsetAsync(u->adam_m.p, 0, u->n_params * sizeof(float), u->stream));
        LG_TRY_CUDA(cudaMemsetAsync(u->adam_v.p, 0, u->n_params * sizeof(float), u->stream));
    }
    return LG_OK;
}

}  // extern "C"
