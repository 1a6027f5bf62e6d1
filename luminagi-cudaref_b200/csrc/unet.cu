// unet.cu -- the denoiser network (reference ml/train.py:37-75) on the
// tcgen05 convolution, and its C ABI (lg_unet_*).
//
// Architecture (base 32, 3- or 12-channel input): d1(in->32) d2(32->64) d3(64->128)
// d4(128->256) at full, 1/2, 1/4, 1/8 resolution, each two 3x3 convs with an
// activation, 2x2 max-pool between levels; u3(384->128) u2(192->64)
// u1(96->32) on cat(up(deeper), skip) with nearest 2x upsampling; a 1x1 tail
// to RGB; out = clamp(x[:, :3] + tail, 0, 1).  The 12-channel variant
// (train.py --gbuffer) stacks colour, albedo, normal and position images.  Activation LeakyReLU(0.1) as in the
// reference (ReLU selectable).  Parameters are kept in FP32 in the reference's
// state_dict order (d1.net.0.weight, d1.net.0.bias, d1.net.2.weight, ...,
// tail.weight, tail.bias) and packed to BF16 for the kernels.
//
// Fusion: the concat buffers are written in place by their producers -- the
// skip half by the encoder's second conv (which also writes the pooled tensor
// for the next level), the upsampled half by the decoder level below (which
// writes each pixel 2x2 times) -- and u1's second conv computes the tail,
// residual and clamp in its epilogue.
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.h"
#include "unet_conv.cuh"

#include "unet_internal.cuh"

using namespace lg;

namespace
{
size_t layout_params(lg_unet* u)
{
    size_t off = 0;
    for (int i = 0; i < 14; ++i)
    {
        u->w_off[i] = off;
        off += (size_t)kLayers[i].cout * layer_cin_real(u, i) * 9;
        u->b_off[i] = off;
        off += (size_t)kLayers[i].cout;
    }
    u->tail_w_off = off;
    off += 3 * 32;
    u->tail_b_off = off;
    off += 3;
    return off;
}

int ensure_acts(lg_unet* u, int N, int H, int W)
{
    if (u->aN == N && u->aH == H && u->aW == W) return LG_OK;
    const size_t px = (size_t)N * H * W, b2 = sizeof(__nv_bfloat16);
    LG_TRY(u->x0.ensure(px * 16 * b2));
    // channels past in_ch stay zero: the input conversion writes only the blocks that hold input channels
    LG_TRY_CUDA(cudaMemsetAsync(u->x0.p, 0, px * 16 * b2, u->stream));
    LG_TRY(u->t1.ensure(px * 32 * b2));
    LG_TRY(u->cat1.ensure(px * 96 * b2));
    LG_TRY(u->p1.ensure(px / 4 * 32 * b2));
    LG_TRY(u->t2.ensure(px / 4 * 64 * b2));
    LG_TRY(u->cat2.ensure(px / 4 * 192 * b2));
    LG_TRY(u->p2.ensure(px / 16 * 64 * b2));
    LG_TRY(u->t3.ensure(px / 16 * 128 * b2));
    LG_TRY(u->cat3.ensure(px / 16 * 384 * b2));
    LG_TRY(u->p3.ensure(px / 64 * 128 * b2));
    LG_TRY(u->t4.ensure(px / 64 * 256 * b2));
    LG_TRY(u->t5.ensure(px / 16 * 128 * b2));
    LG_TRY(u->t6.ensure(px / 4 * 64 * b2));
    LG_TRY(u->t7.ensure(px * 32 * b2));
    LG_TRY(u->u1.ensure(px * 32 * b2));
    if (u->bilinear)
    {
        LG_TRY(u->lo7.ensure(px / 64 * 256 * b2));
        LG_TRY(u->lo9.ensure(px / 16 * 128 * b2));
        LG_TRY(u->lo11.ensure(px / 4 * 64 * b2));
    }
    LG_TRY(u->err.ensure(sizeof(int)));
    u->aN = N;
    u->aH = H;
    u->aW = W;
    return LG_OK;
}

// Upsampled channels at the front of decoder conv i's input (u3a, u2a, u1a: cat(up, skip)); 0 otherwise.
int up_channels(int i) { return (i == 8 || i == 10 || i == 12) ? kLayers[i].cin - kLayers[i].cout : 0; }

// Whether decoder conv i runs its folded-upsampling form in inference: nearest upsampling and a tile that has one.
bool folds(const lg_unet* u, int i)
{
    return u->fold_up && !u->bilinear && up_channels(i) > 0 &&
           conv_tile_folds(u->tile[i], kLayers[i].cin, kLayers[i].cout, up_channels(i));
}

// The 14 convs' packed weights, in one launch (they are repacked after every Adam step).
int pack_all_impl(lg_unet* u)
{
    if (u->packed_ok) return LG_OK;
    ConvPackJob jobs[14];
    for (int i = 0; i < 14; ++i)
    {
        const LayerDef& L = kLayers[i];
        LG_TRY(u->packed[i].ensure(conv_packed_elems(L.cin, L.cout) * sizeof(__nv_bfloat16)));
        jobs[i] = conv_pack_job((const float*)u->params.p + u->w_off[i], L.cout, layer_cin_real(u, i), L.cin,
                                (__nv_bfloat16*)u->packed[i].p, u->tile[i]);
    }
    LG_TRY_CUDA(conv_pack_many(jobs, 14, u->stream));
    u->packed_ok = true;
    u->packed_fold_ok = false;
    return LG_OK;
}

// The folded-upsampling weights of u3a/u2a/u1a, packed on the first inference pass that needs them.
int pack_fold_impl(lg_unet* u)
{
    if (u->packed_fold_ok) return LG_OK;
    for (int i = 0; i < 14; ++i)
    {
        if (!folds(u, i)) continue;
        const LayerDef& L = kLayers[i];
        const int uc = up_channels(i);
        LG_TRY(u->packed_fold[i].ensure(conv_packed_elems_folded(L.cin, L.cout, uc) * sizeof(__nv_bfloat16)));
        LG_TRY_CUDA(conv_pack_weights_folded((const float*)u->params.p + u->w_off[i], L.cout, L.cin, uc,
                                             (__nv_bfloat16*)u->packed_fold[i].p, u->stream, u->tile[i]));
    }
    u->packed_fold_ok = true;
    return LG_OK;
}

ConvArgs base_args(lg_unet* u, int layer, int N, int H, int W)
{
    ConvArgs a{};
    a.N = N;
    a.H = H;
    a.W = W;
    a.Cin = kLayers[layer].cin;
    a.Cout = kLayers[layer].cout;
    a.wpack = (const __nv_bfloat16*)u->packed[layer].p;
    a.bias = (const float*)u->params.p + u->b_off[layer];
    a.slope = u->slope;
    a.epilogue = kEpiStore;
    a.err = (int*)u->err.p;
    a.tile = u->tile[layer];
    return a;
}

typedef __nv_bfloat16 bf;

// Runs the network on a device FP32 NCHW input (N x in_ch x H x W) into d_y (N x 3 x H x W).
int forward_device_impl(lg_unet* u, const float* d_x, int N, int H, int W, float* d_y, bool keep_u1)
{
    if (N <= 0 || H <= 0 || W <= 0 || (H % 8) || (W % 8))
        return set_error(LG_ERR_INVALID, "UNet input must be N>0 and H, W multiples of 8 (got %dx%d)", H, W);
    LG_TRY(pack_all_impl(u));
    LG_TRY(ensure_acts(u, N, H, W));
    cudaStream_t st = u->stream;
    LG_TRY_CUDA(cudaMemsetAsync(u->err.p, 0, sizeof(int), st));
    LG_TRY_CUDA(to_blocked_bf16(d_x, N, u->in_ch, H, W, (bf*)u->x0.p, 16, st, u->log_hdr, true));
    const int H2 = H / 2, W2 = W / 2, H4 = H / 4, W4 = W / 4, H8 = H / 8, W8 = W / 8;
    // inference with nearest upsampling: u3a, u2a, u1a fold their upsampled inputs where their tiles allow
    const bool fold = !keep_u1;
    if (fold) LG_TRY(pack_fold_impl(u));
    auto run = [&](int layer, const void* in, int h, int w, int epi, void* out, int out_c, int out_coff, void* out2,
                   int out2_c, int out2_coff, const void* up_h = nullptr, int x_only = 0) -> int {
        ConvArgs a = base_args(u, layer, N, h, w);
        a.up_x_only = x_only;
        if (up_h)
        {
            a.up_h = (const bf*)up_h;
            a.up_C = up_channels(layer);
            a.wpack = (const bf*)u->packed_fold[layer].p;
        }
        a.epilogue = epi;
        a.out = (bf*)out;
        a.out_C = out_c;
        a.out_coff = out_coff;
        a.out2 = (bf*)out2;
        a.out2_C = out2_c;
        a.out2_coff = out2_coff;
        if (epi == kEpiTail)
        {
            a.tail_w = (const float*)u->params.p + u->tail_w_off;
            a.tail_b = (const float*)u->params.p + u->tail_b_off;
            a.resid = d_x;
            a.resid_C = u->in_ch;  // residual on x[:, :3]
            a.log_hdr = u->log_hdr ? 1 : 0;
            a.final_out = d_y;
        }
        const bool probe = layer == u->probe_layer;
        if (probe) LG_TRY_CUDA(cudaEventRecord(u->probe_ev0, st));
        LG_TRY_CUDA(conv3x3_forward((const bf*)in, a, st));
        if (probe) LG_TRY_CUDA(cudaEventRecord(u->probe_ev1, st));
        return LG_OK;
    };
    // encoder
    LG_TRY(run(0, u->x0.p, H, W, kEpiStore, u->t1.p, 32, 0, nullptr, 0, 0));
    LG_TRY(run(1, u->t1.p, H, W, kEpiStore, u->cat1.p, 96, 64, u->p1.p, 32, 0));
    LG_TRY(run(2, u->p1.p, H2, W2, kEpiStore, u->t2.p, 64, 0, nullptr, 0, 0));
    LG_TRY(run(3, u->t2.p, H2, W2, kEpiStore, u->cat2.p, 192, 128, u->p2.p, 64, 0));
    LG_TRY(run(4, u->p2.p, H4, W4, kEpiStore, u->t3.p, 128, 0, nullptr, 0, 0));
    LG_TRY(run(5, u->t3.p, H4, W4, kEpiStore, u->cat3.p, 384, 256, u->p3.p, 128, 0));
    LG_TRY(run(6, u->p3.p, H8, W8, kEpiStore, u->t4.p, 256, 0, nullptr, 0, 0));
    // The conv before each upsampling writes its output 2x upsampled into the
    // first channels of the next level's concat buffer: nearest copies in its
    // epilogue, or (bilinear) a stored low-resolution result and a resampling pass.
    // With folding, the conv before the upsampling writes its output upsampled along x only (uh, h x 2w) and
    // the next level's first conv reads it there instead of the concat buffer's upsampled half.
    const size_t px = (size_t)N * H * W;
    if (fold && folds(u, 8)) LG_TRY(u->uh3.ensure(px / 32 * 256 * sizeof(bf)));
    if (fold && folds(u, 10)) LG_TRY(u->uh2.ensure(px / 8 * 128 * sizeof(bf)));
    if (fold && folds(u, 12)) LG_TRY(u->uh1.ensure(px / 2 * 64 * sizeof(bf)));
    auto up = [&](int layer, const void* in, int h, int w, Buf& lo, int c, void* cat, int cat_c, Buf& uh) -> int {
        if (fold && folds(u, layer + 1))
            return run(layer, in, h, w, kEpiUpsample, uh.p, c, 0, nullptr, 0, 0, nullptr, 1);
        if (!u->bilinear) return run(layer, in, h, w, kEpiUpsample, cat, cat_c, 0, nullptr, 0, 0);
        LG_TRY(run(layer, in, h, w, kEpiStore, lo.p, c, 0, nullptr, 0, 0));
        LG_TRY_CUDA(bilinear_up2((const bf*)lo.p, N, c, h, w, (bf*)cat, cat_c, 0, st));
        return LG_OK;
    };
    LG_TRY(up(7, u->t4.p, H8, W8, u->lo7, 256, u->cat3.p, 384, u->uh3));
    // decoder
    auto uh_of = [&](int layer, Buf& uh) -> const void* { return fold && folds(u, layer) ? uh.p : nullptr; };
    LG_TRY(run(8, u->cat3.p, H4, W4, kEpiStore, u->t5.p, 128, 0, nullptr, 0, 0, uh_of(8, u->uh3)));
    LG_TRY(up(9, u->t5.p, H4, W4, u->lo9, 128, u->cat2.p, 192, u->uh2));
    LG_TRY(run(10, u->cat2.p, H2, W2, kEpiStore, u->t6.p, 64, 0, nullptr, 0, 0, uh_of(10, u->uh2)));
    LG_TRY(up(11, u->t6.p, H2, W2, u->lo11, 64, u->cat1.p, 96, u->uh1));
    LG_TRY(run(12, u->cat1.p, H, W, kEpiStore, u->t7.p, 32, 0, nullptr, 0, 0, uh_of(12, u->uh1)));
    LG_TRY(run(13, u->t7.p, H, W, kEpiTail, keep_u1 ? u->u1.p : nullptr, 32, 0, nullptr, 0, 0));
    return LG_OK;
}
}  // namespace

namespace lg
{
int unet_forward_device(lg_unet* u, const float* d_x, int N, int H, int W, float* d_y, bool keep_u1)
{
    return forward_device_impl(u, d_x, N, H, W, d_y, keep_u1);
}
int unet_pack_all(lg_unet* u) { return pack_all_impl(u); }
}  // namespace lg

extern "C" {

int lg_unet_create(int base, int in_ch, int act_mode, lg_unet** out)
{
    if (!out) return set_error(LG_ERR_INVALID, "NULL argument");
    *out = nullptr;
    if (base != 32 || in_ch < 3 || in_ch > kLayers[0].cin)
        return set_error(LG_ERR_INVALID, "UNet(base=%d, in_ch=%d): base must be 32 and in_ch in [3, %d]", base, in_ch,
                         kLayers[0].cin);
    if (act_mode & ~(LG_UNET_RELU | LG_UNET_BILINEAR | LG_UNET_LOG_HDR))
        return set_error(LG_ERR_INVALID, "unknown UNet mode bits 0x%x", act_mode);
    lg_unet* u = new (std::nothrow) lg_unet();
    if (!u) return set_error(LG_ERR_NOMEM, "out of memory");
    cudaGetDevice(&u->device);
    cudaDeviceGetAttribute(&u->sm_count, cudaDevAttrMultiProcessorCount, u->device);
    u->slope = (act_mode & LG_UNET_RELU) ? 0.0f : 0.1f;
    u->bilinear = (act_mode & LG_UNET_BILINEAR) != 0;
    u->log_hdr = (act_mode & LG_UNET_LOG_HDR) != 0;
    u->in_ch = in_ch;
    u->n_params = layout_params(u);
    // Forward tiles: lg_unet_autotune's choice at batch 8, 1728x864 on B200 (7.05 ms, against 8.92 ms before the
    // packed-row-tap kernels and 9.75 ms with the per-shape heuristic); the input-gradient convs keep the
    // heuristic until tuned.
    static const ConvTile kTunedFwd[14] = {{32, 16, 4, 5}, {32, 32, 3, 4}, {64, 32, 2, 4}, {64, 32, 2, 4},
                                           {64, 32, 2, 6}, {64, 32, 2, 6}, {64, 32, 2, 6}, {64, 32, 2, 6},
                                           {64, 32, 2, 6}, {64, 32, 2, 6}, {64, 32, 2, 6}, {64, 32, 2, 4},
                                           {32, 32, 2, 7}, {32, 32, 3, 4}};
    for (int i = 0; i < 14; ++i) u->tile[i] = kTunedFwd[i];
    cudaError_t e = cudaStreamCreateWithFlags(&u->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess)
    {
        delete u;
        return set_error(LG_ERR_CUDA, "stream: %s", cudaGetErrorString(e));
    }
    int rc = u->params.ensure(u->n_params * sizeof(float));
    if (rc != LG_OK)
    {
        lg_unet_destroy(u);
        return rc;
    }
    cudaMemsetAsync(u->params.p, 0, u->n_params * sizeof(float), u->stream);
    *out = u;
    return LG_OK;
}

void lg_unet_destroy(lg_unet* u)
{
    if (!u) return;
    if (u->stream) cudaStreamSynchronize(u->stream);
    u->params.release();
    for (auto& b : u->packed) b.release();
    for (Buf* b : {&u->x0, &u->t1, &u->cat1, &u->p1, &u->t2, &u->cat2, &u->p2, &u->t3, &u->cat3, &u->p3, &u->t4,
                   &u->t5, &u->t6, &u->t7, &u->u1, &u->xin, &u->yout, &u->err, &u->grads, &u->adam_m, &u->adam_v,
                   &u->loss, &u->gs1, &u->gs2, &u->gs3, &u->tgt, &u->lo7, &u->lo9, &u->lo11, &u->gup, &u->wpart, &u->bpart, &u->tpart,
                   &u->uh1, &u->uh2, &u->uh3})
        b->release();
    for (auto& b : u->packed_fold) b.release();
    for (auto& b : u->packed_dg) b.release();
    for (auto& b : u->dz) b.release();
    if (u->probe_ev0) cudaEventDestroy(u->probe_ev0);
    if (u->probe_ev1) cudaEventDestroy(u->probe_ev1);
    if (u->order_ev) cudaEventDestroy(u->order_ev);
    if (u->stream) cudaStreamDestroy(u->stream);
    delete u;
}

int64_t lg_unet_num_params(const lg_unet* u) { return u ? (int64_t)u->n_params : 0; }

int lg_unet_set_params(lg_unet* u, const float* host_params, int64_t n)
{
    if (!u || !host_params) return set_error(LG_ERR_INVALID, "NULL argument");
    if ((size_t)n != u->n_params)
        return set_error(LG_ERR_INVALID, "expected %zu parameters, got %lld", u->n_params, (long long)n);
    LG_TRY_CUDA(cudaMemcpyAsync(u->params.p, host_params, u->n_params * sizeof(float), cudaMemcpyHostToDevice,
                                u->stream));
    u->packed_ok = false;
    u->packed_dg_ok = false;
    LG_TRY(pack_all_impl(u));
    LG_TRY_CUDA(cudaStreamSynchronize(u->stream));
    return LG_OK;
}

int lg_unet_get_params(lg_unet* u, float* host_params, int64_t n)
{
    if (!u || !host_params) return set_error(LG_ERR_INVALID, "NULL argument");
    if ((size_t)n != u->n_params)
        return set_error(LG_ERR_INVALID, "expected %zu parameters, got %lld", u->n_params, (long long)n);
    LG_TRY_CUDA(cudaMemcpyAsync(host_params, u->params.p, u->n_params * sizeof(float), cudaMemcpyDeviceToHost,
                                u->stream));
    LG_TRY_CUDA(cudaStreamSynchronize(u->stream));
    return LG_OK;
}

int lg_unet_forward_device(lg_unet* u, const float* d_x, int n, int h, int w, float* d_y, void* stream)
{
    if (!u || !d_x || !d_y) return set_error(LG_ERR_INVALID, "NULL argument");
    if (stream)
    {
        cudaEvent_t ev;
        LG_TRY_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        cudaEventRecord(ev, (cudaStream_t)stream);
        cudaStreamWaitEvent(u->stream, ev, 0);
        cudaEventDestroy(ev);
    }
    LG_TRY(forward_device_impl(u, d_x, n, h, w, d_y, false));
    if (stream)
    {
        cudaEvent_t ev;
        LG_TRY_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        cudaEventRecord(ev, u->stream);
        cudaStreamWaitEvent((cudaStream_t)stream, ev, 0);
        cudaEventDestroy(ev);
        return LG_OK;
    }
    LG_TRY_CUDA(cudaStreamSynchronize(u->stream));
    int err = 0;
    LG_TRY_CUDA(cudaMemcpy(&err, u->err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return set_error(LG_ERR_DEVICE, "convolution kernel reported wait timeout %d", err);
    return LG_OK;
}

int lg_unet_wait_selftest(lg_unet* u, int64_t limit_ns)
{
    if (!u) return set_error(LG_ERR_INVALID, "NULL argument");
    if (limit_ns < 1000 || limit_ns > 2000000000ll)
        return set_error(LG_ERR_INVALID, "wait limit must be 1 us .. 2 s (got %lld ns)", (long long)limit_ns);
    LG_TRY(u->err.ensure(sizeof(int)));
    LG_TRY_CUDA(cudaMemsetAsync(u->err.p, 0, sizeof(int), u->stream));
    LG_TRY_CUDA(launch_wait_probe((int*)u->err.p, (unsigned long long)limit_ns, u->stream));
    LG_TRY_CUDA(cudaStreamSynchronize(u->stream));
    int err = 0;
    LG_TRY_CUDA(cudaMemcpy(&err, u->err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return set_error(LG_ERR_DEVICE, "convolution kernel reported wait timeout %d", err);
    return LG_OK;
}

int lg_unet_forward(lg_unet* u, const float* x, int n, int h, int w, float* y)
{
    if (!u || !x || !y) return set_error(LG_ERR_INVALID, "NULL argument");
    const size_t bytes = (size_t)n * 3 * h * w * sizeof(float);
    const size_t in_bytes = (size_t)n * u->in_ch * h * w * sizeof(float);
    LG_TRY(u->xin.ensure(in_bytes));
    LG_TRY(u->yout.ensure(bytes));
    LG_TRY_CUDA(cudaMemcpyAsync(u->xin.p, x, in_bytes, cudaMemcpyHostToDevice, u->stream));
    LG_TRY(forward_device_impl(u, (const float*)u->xin.p, n, h, w, (float*)u->yout.p, false));
    LG_TRY_CUDA(cudaMemcpyAsync(y, u->yout.p, bytes, cudaMemcpyDeviceToHost, u->stream));
    LG_TRY_CUDA(cudaStreamSynchronize(u->stream));
    int err = 0;
    LG_TRY_CUDA(cudaMemcpy(&err, u->err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return set_error(LG_ERR_DEVICE, "convolution kernel reported wait timeout %d", err);
    return LG_OK;
}

// One convolution layer on device buffers (blocked BF16 in/out, FP32 PyTorch-
// layout weights); used to test the kernel layer by layer.
int lg_conv3x3_device(const void* d_in, int n, int cin, int h, int w, const float* d_w, int cin_real,
                      const float* d_b, int cout, float slope, int epilogue, void* d_out, int out_c, int out_coff,
                      void* d_out2, int out2_c, int out2_coff, void* stream)
{
    if (!d_in || !d_w || !d_b || !d_out) return set_error(LG_ERR_INVALID, "NULL argument");
    if (epilogue != kEpiStore && epilogue != kEpiUpsample)
        return set_error(LG_ERR_INVALID, "epilogue must be 0 (store/pool) or 1 (upsample)");
    cudaStream_t st = (cudaStream_t)stream;
    __nv_bfloat16* packed = nullptr;
    LG_TRY_CUDA(cudaMallocAsync((void**)&packed, conv_packed_elems(cin, cout) * sizeof(__nv_bfloat16), st));
    cudaError_t e = conv_pack_weights(d_w, cout, cin_real, cin, packed, st);
    ConvArgs a{};
    a.N = n; a.H = h; a.W = w; a.Cin = cin; a.Cout = cout; a.wpack = packed; a.bias = d_b; a.slope = slope;
    a.epilogue = epilogue; a.out = (__nv_bfloat16*)d_out; a.out_C = out_c; a.out_coff = out_coff;
    a.out2 = (__nv_bfloat16*)d_out2; a.out2_C = out2_c; a.out2_coff = out2_coff;
    if (e == cudaSuccess) e = conv3x3_forward((const __nv_bfloat16*)d_in, a, st);
    cudaFreeAsync(packed, st);
    if (e != cudaSuccess) return set_error(LG_ERR_CUDA, "conv3x3: %s", cudaGetErrorString(e));
    LG_TRY_CUDA(cudaStreamSynchronize(st));
    return LG_OK;
}

int lg_to_blocked_bf16(const float* d_x, int n, int c, int h, int w, void* d_out, int cpad, void* stream)
{
    if (cpad % 8 || cpad < c) return set_error(LG_ERR_INVALID, "cpad must be a multiple of 8 >= c");
    LG_TRY_CUDA(to_blocked_bf16(d_x, n, c, h, w, (__nv_bfloat16*)d_out, cpad, (cudaStream_t)stream));
    return LG_OK;
}

int lg_from_blocked_bf16(const void* d_in, int n, int c, int h, int w, float* d_out, void* stream)
{
    if (c % 8) return set_error(LG_ERR_INVALID, "c must be a multiple of 8");
    LG_TRY_CUDA(from_blocked_bf16((const __nv_bfloat16*)d_in, n, c, h, w, d_out, (cudaStream_t)stream));
    return LG_OK;
}

}  // extern "C"
