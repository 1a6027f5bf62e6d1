// unet_conv.cuh -- 3x3 "same" convolution on tcgen05 tensor cores.
//
// Activations live in device memory as BF16 in a channel-blocked layout:
// element (n, c, y, x) of a C-channel H x W tensor is at
//     (((n * C/8 + c/8) * H + y) * W + x) * 8 + c % 8
// i.e. planes of 8 channels, 16 bytes per pixel.  A 5-D TMA box of that
// tensor lands in shared memory exactly in the MMA's no-swizzle K-major
// layout, and a one-pixel shift of a 3x3 tap is a 16-byte shift of the MMA
// descriptor, so each input tile is loaded once for all nine taps.
#pragma once
#include <cstddef>
#include <cstdint>

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace lg
{
enum ConvEpilogue : int
{
    kEpiStore = 0,     // act(acc + bias) -> out (and, if out2, 2x2 max-pooled -> out2)
    kEpiUpsample = 1,  // act(acc + bias) -> out at 2x resolution (nearest, 4 copies; 2 along x with up_x_only)
    kEpiTail = 2,      // act(acc + bias) -> out (optional); 1x1 conv to 3 + residual + clamp -> final (FP32 NCHW)
                       // (log_hdr: residual on log1p(input), out = expm1(max(y, 0)))
    // Backward (input-gradient) epilogues; no bias is added.
    kEpiBwdMask = 3,     // out = acc * act'(ref) at the same position
    kEpiBwdSumPool = 4,  // acc at 2x resolution -> 2x2 sum -> * act'(ref at 1x) -> out (1x)
    kEpiBwdStore = 5,    // out = acc
    kEpiBwdUnpool = 6,   // acc = d(pooled); route to the max of ref's 2x2 window, add skip, * act'(ref) -> out (2x)
};

// Tile shape of one convolution: BN output channels per CTA, KC input
// channels per K-block, STAGES pipeline stages, and which kernel runs it.  Packed weights depend on
// (BN, KC), so a layer packs and launches with the same tile.  bn == 0 means
// the default heuristic (conv_default_tile).
struct ConvTile
{
    int bn, kc, stages;
    int persist;  // 0: one tile per CTA; 1: the persistent, warp-specialised kernel; 2: persistent with the
                  // weights resident in shared memory; 3: as 2 with 4-row tiles (same packing, same results)
};
ConvTile conv_default_tile(int Cin, int Cout);
// The compiled tile shapes valid for a layer (Cout % bn == 0, Cin % kc == 0);
// returns how many were written to out (at most max).
int conv_tile_candidates(int Cin, int Cout, ConvTile* out, int max);

struct ConvArgs
{
    int N, H, W;         // spatial size of input and output
    int Cin;             // input channels (the tensor map's channel count; multiple of 16)
    int Cout;            // output channels of the layer
    const __nv_bfloat16* wpack;  // packed weights (conv_pack_weights)
    const float* bias;           // [Cout]
    float slope;                 // activation: x > 0 ? x : slope * x (0.1 LeakyReLU, 0 ReLU)
    int epilogue;                // ConvEpilogue
    __nv_bfloat16* out;          // blocked output (may be null for kEpiTail)
    int out_C, out_coff;         // channel count of `out` and first channel written
    __nv_bfloat16* out2;         // pooled output (kEpiStore, may be null)
    int out2_C, out2_coff;
    const float* tail_w;         // [3][Cout] (kEpiTail, Cout == 32)
    const float* tail_b;         // [3]
    const float* resid;          // FP32 NCHW input image (kEpiTail), channels 0..2 used, resid_C channels
    int resid_C;
    int log_hdr;                 // kEpiTail: the HDR variant's log-space residual and expm1 output
    float* final_out;            // FP32 NCHW [N][3][H][W]
    int* err;                    // set non-zero by a kernel that hit a wait limit
    // backward epilogues
    const __nv_bfloat16* ref;    // forward activation whose act' masks the gradient
    int ref_C, ref_coff;
    const __nv_bfloat16* skip;   // kEpiBwdUnpool: gradient arriving through the skip connection (2x res)
    int skip_C, skip_coff;
    ConvTile tile;               // {0, 0, 0}: default; must match the tile the weights were packed with
    int a_chunked;               // set by the launcher: the A map is the 8-pixel-run view (W % 8 == 0)
    // Folded upsampling (inference form of a decoder conv whose input is cat([up2(lo), skip]) with nearest
    // 2x upsampling): with up_C > 0 the first up_C input channels are read from up_h, the low-resolution
    // tensor upsampled along x only (blocked, N x up_C x H/2 x W), and the row taps are folded per output-row
    // parity (conv_pack_weights_folded); the skip channels are read from `in` (channels up_C..Cin-1).
    const __nv_bfloat16* up_h;
    int up_C;
    int up_x_only;               // kEpiUpsample: write the 2x-along-x copy only (out is N x out_C x H x 2W)
};

// Bytes of packed weights for a layer (BF16).
size_t conv_packed_elems(int Cin, int Cout);
// The same for the folded-upsampling form (ConvArgs::up_C): the up_C upsampled channels carry four
// folded row taps per column tap instead of three.
size_t conv_packed_elems_folded(int Cin, int Cout, int up_C);
// Whether a tile has a folded-upsampling form (the packed-row-tap kernels with streamed weights, BN <= 64).
bool conv_tile_folds(ConvTile tile, int Cin, int Cout, int up_C);
// Packs w[Cout][Cin][3][3] for the folded form: per output block the skip channels' K-blocks (row taps
// packed into N, as conv_pack_weights with the same tile) and then the upsampled channels' K-blocks with the
// row taps summed per output-row parity: [dx][KC/8][ky2 | ky1+ky2 | ky0+ky1 | ky0][BN][8], the four
// output rows 2h-1 .. 2h+2 that low-resolution row h reaches.
cudaError_t conv_pack_weights_folded(const float* d_w, int Cout, int Cin, int up_C, __nv_bfloat16* d_packed,
                                     cudaStream_t stream, ConvTile tile);
// Packs PyTorch-layout FP32 weights w[Cout][Cin_real][3][3] into the layout
// the kernel streams (input channels beyond Cin_real are zero).
cudaError_t conv_pack_weights(const float* d_w, int Cout, int Cin_real, int Cin, __nv_bfloat16* d_packed,
                              cudaStream_t stream, ConvTile tile = ConvTile{0, 0, 0});

// One layer's packing in a batched launch (conv_pack_many): the arguments of conv_pack_weights (dgrad = 0), or
// (dgrad = 1) a forward conv's input-gradient weights w'[ci][co][ky][kx] = w[co][ci][2-ky][2-kx] for ci in
// [ci_lo, ci_lo+ci_cnt), packed as a convolution with Cin' = Cout input and ci_cnt output channels; resolved to
// the tile's (BN, KC) and layout.
struct ConvPackJob
{
    const float* w;
    __nv_bfloat16* out;
    size_t elems;
    int Cout, Cin_real, Cin, bn, kc, dyp, dgrad, ci_lo, ci_cnt;
};
constexpr int kMaxPackJobs = 16;
ConvPackJob conv_pack_job(const float* d_w, int Cout, int Cin_real, int Cin, __nv_bfloat16* d_packed, ConvTile tile);
ConvPackJob conv_pack_job_dgrad(const float* d_w, int Cout, int Cin_real, int ci_lo, int ci_cnt,
                                __nv_bfloat16* d_packed, ConvTile tile);
// Packs up to kMaxPackJobs layers in one launch (forward jobs: the same bits as one conv_pack_weights call each).
cudaError_t conv_pack_many(const ConvPackJob* jobs, int n, cudaStream_t stream);

// Launches the convolution reading `in` (blocked BF16, N x Cin x H x W).
cudaError_t conv3x3_forward(const __nv_bfloat16* in, const ConvArgs& a, cudaStream_t stream);

// The bounded wait of the convolution kernels (tc::mbar_wait) on an mbarrier
// that nothing arrives at: after limit_ns the probe stores 3 in *err, as a
// convolution kernel whose wait ran out stores its code, and returns.  It
// issues no TMA copy or MMA, so nothing is left in flight; the context stays
// usable.  Exercises the error path (device flag -> host status) on demand.
cudaError_t launch_wait_probe(int* err, unsigned long long limit_ns, cudaStream_t stream);

// FP32 NCHW (C channels) -> blocked BF16 with Cpad channels (zero padded);
// log1p_in applies log1p to every value first (the HDR variant's input).
// skip_zero_blocks: leave the 8-channel blocks past channel C untouched (the
// caller keeps them zero).
cudaError_t to_blocked_bf16(const float* x, int N, int C, int H, int W, __nv_bfloat16* out, int Cpad,
                            cudaStream_t stream, bool log1p_in = false, bool skip_zero_blocks = false);

// Bilinear 2x upsampling (F.interpolate(scale_factor=2, mode="bilinear",
// align_corners=False)) of a blocked BF16 tensor N x C x h x w into channels
// [coff, coff + C) of a blocked tensor N x out_C x 2h x 2w.
cudaError_t bilinear_up2(const __nv_bfloat16* in, int N, int C, int h, int w, __nv_bfloat16* out, int out_C,
                         int coff, cudaStream_t stream);
// Its adjoint, masked by the activation derivative: g_lo = up2^T(g_hi) *
// act'(ref), where g_hi is N x C x 2h x 2w and ref, g_lo are N x C x h x w
// (all blocked BF16).
cudaError_t bilinear_up2_adjoint(const __nv_bfloat16* g_hi, int N, int C, int h, int w, const __nv_bfloat16* ref,
                                 float slope, __nv_bfloat16* g_lo, cudaStream_t stream);
// Blocked BF16 (C channels) -> FP32 NCHW.
cudaError_t from_blocked_bf16(const __nv_bfloat16* in, int N, int C, int H, int W, float* out, cudaStream_t stream);
}  // namespace lg
