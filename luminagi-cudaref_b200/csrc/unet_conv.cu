// unet_conv.cu -- 3x3 convolution as an implicit GEMM on tcgen05 (see unet_conv.cuh).
//
// One CTA computes a 2-row x 128-pixel output tile for BN output channels:
//   M = 128 pixels (one MMA per output row), N = BN, K = 9 taps x Cin.
// Per K-block of KC input channels, thread 0
//   * loads the input halo (4 rows x 130 pixels x KC channels) with one 5-D
//     TMA box (out-of-range rows/columns are zero-filled: the conv padding),
//   * bulk-copies the packed weights of the 9 taps (9 x KC x BN),
//   * issues 9 taps x KC/16 K-steps x 2 rows tcgen05.mma (M=128, N=BN, K=16)
//     into two TMEM accumulators; tap (dy,dx) is the same smem tile read at
//     pixel offset (row+dy)*130 + dx, i.e. 16-byte steps of the descriptor,
//   * commits each stage to an mbarrier that frees it for the next K-block.
// The 4 warps then read their 32 TMEM lanes (= pixels) and apply bias and
// activation, writing BF16 in the blocked layout, plus the fused extras:
// 2x2 max-pool (both rows are in the tile; x pairs are adjacent lanes),
// nearest 2x upsample into a concat buffer, or the UNet tail (1x1 conv to
// RGB + residual + clamp).  Operands are BF16, accumulation FP32.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <mutex>

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.h"
#include "tc_ptx.cuh"
#include "unet_conv.cuh"

namespace lg
{
namespace
{
constexpr int kTileX = 128;  // output pixels per row (= MMA M)
constexpr int kHaloX = kTileX + 2;
constexpr int kRows = 2;     // output rows per CTA
constexpr int kHaloY = kRows + 2;
constexpr int kThreads = 128;

typedef ConvTile TileCfg;

// Default tile shape per layer: BN = min(Cout, 128), KC = 32 input channels
// per K-block (16 when Cin is not a multiple of 32), stages to fill ~100 KB
// for narrow layers or ~210 KB for wide ones, on the persistent kernel.  The
// autotuner (lg_unet_autotune) may pick another compiled shape or kernel.
TileCfg pick_cfg(int Cin, int Cout)
{
    TileCfg c{};
    c.bn = Cout < 128 ? Cout : 128;
    c.kc = (Cin % 32 == 0) ? 32 : 16;
    if (c.bn == 32) c.stages = c.kc == 16 ? 4 : 2;
    else if (c.bn == 64) c.stages = 3;
    else c.stages = 2;
    c.persist = 1;  // persistent kernel: 1.3-1.4x the one-tile-per-CTA kernel on the UNet layers
    return c;
}

// Pixels per halo row of an A tile in shared memory: 130 when the TMA box
// starts at x0 - 1 pixel by pixel (16-byte box rows), 144 when it is loaded
// as 18 runs of 8 pixels (128-byte box rows) from x0 - 8 (chunked view).
constexpr int kChunkX = kTileX + 16;
template <int BN, int KC, int ROWS = kRows, int AX = kHaloX>
struct Smem
{
    static constexpr int kABytes = (ROWS + 2) * AX * KC * 2;
    static constexpr int kBBytes = 9 * KC * BN * 2;
    static constexpr int kStage = ((kABytes + kBBytes + 1023) / 1024) * 1024;
};

__device__ __forceinline__ float act(float v, float slope) { return v > 0.0f ? v : v * slope; }

__device__ __forceinline__ uint4 pack8(const float* v)
{
    __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]);
    __nv_bfloat162 b = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 c = __floats2bfloat162_rn(v[4], v[5]);
    __nv_bfloat162 d = __floats2bfloat162_rn(v[6], v[7]);
    uint4 u;
    u.x = *reinterpret_cast<uint32_t*>(&a);
    u.y = *reinterpret_cast<uint32_t*>(&b);
    u.z = *reinterpret_cast<uint32_t*>(&c);
    u.w = *reinterpret_cast<uint32_t*>(&d);
    return u;
}
__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// Address of pixel (n, block b, y, x) of a blocked tensor with C channels.
__device__ __forceinline__ uint4* blk(__nv_bfloat16* base, int C, int H, int W, int n, int b, int y, int x)
{
    return reinterpret_cast<uint4*>(base + ((((size_t)n * (C >> 3) + b) * H + y) * W + x) * 8);
}

__device__ __forceinline__ void unpack8(uint4 u, float* v)
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
// 16 channels (two blocks starting at block b) of pixel (n, y, x).
__device__ __forceinline__ void load16(const __nv_bfloat16* base, int C, int H, int W, int n, int b, int y, int x,
                                       float* v)
{
    unpack8(__ldg(reinterpret_cast<const uint4*>(base + ((((size_t)n * (C >> 3) + b) * H + y) * W + x) * 8)), v);
    unpack8(__ldg(reinterpret_cast<const uint4*>(base + ((((size_t)n * (C >> 3) + b + 1) * H + y) * W + x) * 8)),
            v + 8);
}
__device__ __forceinline__ float dact(float y, float slope) { return y > 0.0f ? 1.0f : slope; }

// Input-gradient epilogues (see ConvEpilogue).  v[r][j]: gradient of conv
// input channel cg+j at (y0+r, x) of this (backward) convolution.
__device__ __forceinline__ void bwd_epilogue(const ConvArgs& a, float (&v)[kRows][16], int n, int y0, int x, int cg,
                                             int b0)
{
    const bool xin = x < a.W;
    const int rb = (a.ref_coff + cg) >> 3;
    if (a.epilogue == kEpiBwdMask || a.epilogue == kEpiBwdStore)
    {
#pragma unroll
        for (int r = 0; r < kRows; ++r)
        {
            const int y = y0 + r;
            if (!xin || y >= a.H) continue;
            float o[16];
            if (a.epilogue == kEpiBwdMask)
            {
                float ref[16];
                load16(a.ref, a.ref_C, a.H, a.W, n, rb, y, x, ref);
#pragma unroll
                for (int j = 0; j < 16; ++j) o[j] = v[r][j] * dact(ref[j], a.slope);
            }
            else
            {
#pragma unroll
                for (int j = 0; j < 16; ++j) o[j] = v[r][j];
            }
            *blk(a.out, a.out_C, a.H, a.W, n, b0, y, x) = pack8(o);
            *blk(a.out, a.out_C, a.H, a.W, n, b0 + 1, y, x) = pack8(o + 8);
        }
    }
    else if (a.epilogue == kEpiBwdSumPool)
    {
        // Gradient of a nearest 2x upsample: sum of the 2x2 children.
        float s[16];
#pragma unroll
        for (int j = 0; j < 16; ++j)
        {
            const float t = v[0][j] + v[1][j];
            s[j] = t + __shfl_xor_sync(0xffffffffu, t, 1);
        }
        const int H2 = a.H >> 1, W2 = a.W >> 1;
        if (((x & 1) == 0) && (x >> 1) < W2 && (y0 >> 1) < H2)
        {
            // act' of the upsampled tensor is read at the even child (ref is 2x too).
            float ref[16];
            load16(a.ref, a.ref_C, a.H, a.W, n, rb, y0, x, ref);
#pragma unroll
            for (int j = 0; j < 16; ++j) s[j] *= dact(ref[j], a.slope);
            *blk(a.out, a.out_C, H2, W2, n, b0, y0 >> 1, x >> 1) = pack8(s);
            *blk(a.out, a.out_C, H2, W2, n, b0 + 1, y0 >> 1, x >> 1) = pack8(s + 8);
        }
    }
    else  // kEpiBwdUnpool: this conv ran at the pooled resolution; ref/skip/out are 2H x 2W
    {
        const int H2 = a.H * 2, W2 = a.W * 2;
        const int sb = (a.skip_coff + cg) >> 3;
#pragma unroll 1
        for (int r = 0; r < kRows; ++r)
        {
            const int y = y0 + r;
            if (!xin || y >= a.H) continue;
            float win[4][16];
#pragma unroll
            for (int q = 0; q < 4; ++q) load16(a.ref, a.ref_C, H2, W2, n, rb, 2 * y + (q >> 1), 2 * x + (q & 1), win[q]);
            // First maximum in raster order wins, as max_pool2d's backward routes it.
            int arg[16];
#pragma unroll
            for (int j = 0; j < 16; ++j)
            {
                int best = 0;
                float bv = win[0][j];
#pragma unroll
                for (int q = 1; q < 4; ++q)
                    if (win[q][j] > bv) { bv = win[q][j]; best = q; }
                arg[j] = best;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
            {
                const int yy = 2 * y + (q >> 1), xx = 2 * x + (q & 1);
                float g[16];
                load16(a.skip, a.skip_C, H2, W2, n, sb, yy, xx, g);
#pragma unroll
                for (int j = 0; j < 16; ++j)
                {
                    const float t = g[j] + (arg[j] == q ? v[r][j] : 0.0f);
                    g[j] = t * dact(win[q][j], a.slope);
                }
                *blk(a.out, a.out_C, H2, W2, n, b0, yy, xx) = pack8(g);
                *blk(a.out, a.out_C, H2, W2, n, b0 + 1, yy, xx) = pack8(g + 8);
            }
        }
    }
}

// The epilogue's per-layer constants, staged once per CTA in shared memory so
// the epilogue reads them as 16-byte vectors instead of one global load per
// value: bias (Cout <= 256) and the UNet tail's 3 x 32 weights and 3 biases.
struct __align__(16) EpiConsts
{
    float bias[256];
    float tw[96];
    float tb[4];
};
__device__ __forceinline__ void stage_epi_consts(const ConvArgs& a, EpiConsts& ec, int tid, int nthreads)
{
    if (a.bias && a.epilogue <= kEpiTail)
        for (int i = tid; i < a.Cout; i += nthreads) ec.bias[i] = a.bias[i];
    if (a.epilogue == kEpiTail)
    {
        for (int i = tid; i < 96; i += nthreads) ec.tw[i] = a.tail_w[i];
        if (tid < 3) ec.tb[tid] = a.tail_b[tid];
    }
}
__device__ __forceinline__ void ld16(const float* p, float (&v)[16])  // p 16-byte aligned (shared memory)
{
    const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        const float4 t = q[i];
        v[4 * i] = t.x;
        v[4 * i + 1] = t.y;
        v[4 * i + 2] = t.z;
        v[4 * i + 3] = t.w;
    }
}

// Epilogue of one output tile (2 rows x 128 pixels x BN channels of output
// block ct): the accumulator at TMEM column `tmem` holds row r at columns
// r*BN..r*BN+BN-1; lane p = pixel x0 + p.  The calling warp reads its quarter
// of the lanes: `warp` (0..3) selects lanes 32*warp..32*warp+31 and
// tid = 32*warp + lane is the pixel offset.  With nparts > 1 several warps
// share a quarter: part `part` takes every nparts-th 16-channel chunk, or
// for the tail (which needs a pixel's 32 channels together) every
// nparts-th row.
template <int BN>
__device__ __forceinline__ void tile_epilogue(const ConvArgs& a, const EpiConsts& ec, uint32_t tmem, int warp, int tid,
                                              int n, int ct, int x0, int y0, int part = 0, int nparts = 1)
{
    const uint32_t lanebase = tmem + ((uint32_t)(warp * 32) << 16);
    const int x = x0 + tid;
    const bool xin = x < a.W;
    if (a.epilogue == kEpiTail)
    {
        // BN == Cout == 32: whole pixel in this thread.
        float o[kRows][3];
        float res[kRows][3];  // the residual input, loaded before the accumulator so the two latencies overlap
#pragma unroll
        for (int r = 0; r < kRows; ++r)
        {
            const int y = y0 + r;
#pragma unroll
            for (int k = 0; k < 3; ++k)
                res[r][k] = (r % nparts == part && xin && y < a.H)
                                ? a.resid[(((size_t)n * a.resid_C + k) * a.H + y) * a.W + x]
                                : 0.0f;
        }
#pragma unroll
        for (int r = 0; r < kRows; ++r)
        {
            if (r % nparts != part) continue;
            float v[32];
            uint32_t q0[16], q1[16];
            tc::tmem_ld16_issue(lanebase + (uint32_t)(r * BN), q0);
            tc::tmem_ld16_issue(lanebase + (uint32_t)(r * BN + 16), q1);
            tc::tmem_wait_ld();
            tc::tmem_ld16_take(q0, v);
            tc::tmem_ld16_take(q1, v + 16);
#pragma unroll
            for (int c0 = 0; c0 < 32; c0 += 16)
            {
                float bb[16];
                ld16(ec.bias + c0, bb);
#pragma unroll
                for (int j = 0; j < 16; ++j) v[c0 + j] = bf16r(act(v[c0 + j] + bb[j], a.slope));
            }
            const int y = y0 + r;
            if (a.out && xin && y < a.H)
            {
#pragma unroll
                for (int b = 0; b < 4; ++b)
                    *blk(a.out, a.out_C, a.H, a.W, n, (a.out_coff >> 3) + b, y, x) = pack8(v + 8 * b);
            }
#pragma unroll
            for (int k = 0; k < 3; ++k)
            {
                float acc = ec.tb[k];
#pragma unroll
                for (int c0 = 0; c0 < 32; c0 += 16)
                {
                    float ww[16];
                    ld16(ec.tw + k * 32 + c0, ww);
#pragma unroll
                    for (int j = 0; j < 16; ++j) acc = fmaf(ww[j], v[c0 + j], acc);
                }
                o[r][k] = acc;
            }
        }
#pragma unroll
        for (int r = 0; r < kRows; ++r)
        {
            const int y = y0 + r;
            if (r % nparts != part || !xin || y >= a.H) continue;
#pragma unroll
            for (int k = 0; k < 3; ++k)
            {
                const size_t po = (((size_t)n * 3 + k) * a.H + y) * a.W + x;
                if (a.log_hdr) a.final_out[po] = expm1f(fmaxf(log1pf(res[r][k]) + o[r][k], 0.0f));
                else a.final_out[po] = fminf(fmaxf(res[r][k] + o[r][k], 0.0f), 1.0f);
            }
        }
    }
    else
    {
#pragma unroll 1
        for (int c0 = 16 * part; c0 < BN; c0 += 16 * nparts)
        {
            float v[kRows][16];
            {
                uint32_t q[kRows][16];
#pragma unroll
                for (int r = 0; r < kRows; ++r) tc::tmem_ld16_issue(lanebase + (uint32_t)(r * BN + c0), q[r]);
                tc::tmem_wait_ld();
#pragma unroll
                for (int r = 0; r < kRows; ++r) tc::tmem_ld16_take(q[r], v[r]);
            }
            const int cg = ct * BN + c0;  // layer channel of v[.][0]
            if (a.epilogue <= kEpiUpsample)
            {
                // stored through pack8, which rounds to BF16 once; the 2x2 max of the pooled output commutes
                // with that (monotonic) rounding, so no separate rounding step is needed here
                float bb[16];
                ld16(ec.bias + cg, bb);
#pragma unroll
                for (int r = 0; r < kRows; ++r)
#pragma unroll
                    for (int j = 0; j < 16; ++j) v[r][j] = act(v[r][j] + bb[j], a.slope);
            }
            const int b0 = (a.out_coff + cg) >> 3;
            if (a.epilogue >= kEpiBwdMask)
            {
                bwd_epilogue(a, v, n, y0, x, cg, b0);
            }
            else if (a.epilogue == kEpiStore)
            {
#pragma unroll
                for (int r = 0; r < kRows; ++r)
                {
                    const int y = y0 + r;
                    if (xin && y < a.H)
                    {
                        *blk(a.out, a.out_C, a.H, a.W, n, b0, y, x) = pack8(v[r]);
                        *blk(a.out, a.out_C, a.H, a.W, n, b0 + 1, y, x) = pack8(v[r] + 8);
                    }
                }
                if (a.out2)
                {
                    float m[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                    {
                        float t = fmaxf(v[0][j], v[1][j]);
                        m[j] = fmaxf(t, __shfl_xor_sync(0xffffffffu, t, 1));
                    }
                    const int H2 = a.H >> 1, W2 = a.W >> 1;
                    if (((x & 1) == 0) && (x >> 1) < W2 && (y0 >> 1) < H2)
                    {
                        const int pb = (a.out2_coff + cg) >> 3;
                        *blk(a.out2, a.out2_C, H2, W2, n, pb, y0 >> 1, x >> 1) = pack8(m);
                        *blk(a.out2, a.out2_C, H2, W2, n, pb + 1, y0 >> 1, x >> 1) = pack8(m + 8);
                    }
                }
            }
            else  // kEpiUpsample: nearest 2x into a 2H x 2W buffer (H x 2W with up_x_only)
            {
                const int ry = a.up_x_only ? 1 : 2;
                const int H2 = a.H * ry, W2 = a.W * 2;
#pragma unroll
                for (int r = 0; r < kRows; ++r)
                {
                    const int y = y0 + r;
                    if (!xin || y >= a.H) continue;
                    const uint4 lo = pack8(v[r]), hi = pack8(v[r] + 8);
                    // pixels 2x and 2x+1 are 32 contiguous bytes of a channel plane: one store each
                    for (int i = 0; i < ry; ++i)
                    {
                        tc::st_global_v8(blk(a.out, a.out_C, H2, W2, n, b0, ry * y + i, 2 * x), lo, lo);
                        tc::st_global_v8(blk(a.out, a.out_C, H2, W2, n, b0 + 1, ry * y + i, 2 * x), hi, hi);
                    }
                }
            }
        }
    }
}

template <int BN, int KC, int STAGES>
__global__ void __launch_bounds__(kThreads, 1) conv3x3_tc_kernel(const __grid_constant__ CUtensorMap tmap, ConvArgs a)
{
    using S = Smem<BN, KC>;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * S::kStage);
    uint64_t* empty = full + STAGES;
    uint64_t* done = empty + STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    __shared__ int s_fail;
    __shared__ EpiConsts ec;

    const int tid = threadIdx.x, warp = tid >> 5;
    stage_epi_consts(a, ec, tid, kThreads);  // visible after the __syncthreads below
    const int n_cot = a.Cout / BN;
    const int x0 = blockIdx.x * kTileX;
    const int y0 = blockIdx.y * kRows;
    const int n = blockIdx.z / n_cot;
    const int ct = blockIdx.z % n_cot;
    const int KB = a.Cin / KC;
    constexpr uint32_t kCols = 2 * BN;  // two accumulators of BN FP32 columns
    constexpr uint32_t kIdesc = tc::idesc_bf16_f32(128, BN);
    constexpr uint32_t kLboA = kHaloY * kHaloX * 16;
    constexpr uint32_t kLboB = BN * 16;

    if (warp == 0)
    {
        tc::tmem_alloc(tmem_slot, kCols);
        tc::tmem_relinquish();
    }
    if (tid == 0)
    {
        s_fail = 0;
        for (int s = 0; s < STAGES; ++s)
        {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        tc::mbar_init(done, 1);
        tc::fence_mbar_init();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (tid == 0)
    {
        const __nv_bfloat16* wsrc = a.wpack + (size_t)ct * KB * (9 * KC * BN);
        auto issue_load = [&](int s, int kb) {
            uint8_t* A = smem + s * S::kStage;
            uint8_t* B = A + S::kABytes;
            tc::mbar_expect_tx(&full[s], (uint32_t)(S::kABytes + S::kBBytes));
            tc::tma_load_5d(A, &tmap, &full[s], 0, x0 - 1, y0 - 1, kb * (KC / 8), n);
            tc::bulk_load(B, wsrc + (size_t)kb * (9 * KC * BN), (uint32_t)S::kBBytes, &full[s]);
        };
        const int pre = KB < STAGES ? KB : STAGES;
        for (int s = 0; s < pre; ++s) issue_load(s, s);
        bool ok = true;
        for (int kb = 0; kb < KB && ok; ++kb)
        {
            const int s = kb % STAGES;
            if (!tc::mbar_wait(&full[s], (uint32_t)((kb / STAGES) & 1))) { ok = false; break; }
            tc::tc_fence_after();
            const uint32_t abase = tc::smem_u32(smem + s * S::kStage);
            const uint32_t bbase = abase + S::kABytes;
#pragma unroll 1
            for (int tap = 0; tap < 9; ++tap)
            {
                const int dy = tap / 3, dx = tap % 3;
#pragma unroll
                for (int ks = 0; ks < KC / 16; ++ks)
                {
                    const uint64_t bd = tc::smem_desc(bbase + (uint32_t)((tap * (KC / 8) + 2 * ks) * BN * 16), kLboB, 128);
#pragma unroll
                    for (int r = 0; r < kRows; ++r)
                    {
                        const uint32_t aoff = (uint32_t)(2 * ks) * kLboA + (uint32_t)(((r + dy) * kHaloX + dx) * 16);
                        const uint64_t ad = tc::smem_desc(abase + aoff, kLboA, 128);
                        tc::mma_bf16(tmem + (uint32_t)(r * BN), ad, bd, kIdesc, (kb | tap | ks) != 0 ? 1u : 0u);
                    }
                }
            }
            tc::mma_commit(&empty[s]);
            // Refill the stage used one K-block ago (its MMAs are queued ahead of this one's).
            if (kb >= 1)
            {
                const int ps = (kb - 1) % STAGES;
                const int nk = kb - 1 + STAGES;
                if (nk < KB)
                {
                    if (!tc::mbar_wait(&empty[ps], (uint32_t)(((kb - 1) / STAGES) & 1))) { ok = false; break; }
                    issue_load(ps, nk);
                }
            }
        }
        if (!ok)
        {
            s_fail = 1;
            if (a.err) atomicExch(a.err, 1);
        }
        tc::mma_commit(done);  // completes when every MMA issued above has finished
    }
    __syncwarp();
    // Epilogue: every thread owns TMEM lane = pixel x0 + tid.
    const bool got = tc::mbar_wait(done, 0);
    if (!got && a.err) atomicExch(a.err, 2);
    tc::tc_fence_after();
    if (got && !s_fail) tile_epilogue<BN>(a, ec, tmem, warp, tid, n, ct, x0, y0);

    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0)
    {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, kCols);
    }
}


// Persistent, warp-specialised form of conv3x3_tc_kernel: one CTA per SM
// walks the output tiles in a grid-stride loop.
//   warp 0 (one lane)  TMA loads of input halos and weight blocks into a
//                      STAGES-deep ring (full/empty mbarriers);
//   warp 1 (one lane)  tcgen05.mma into one of two TMEM accumulators (each two
//                      rows x BN columns), committing the ring stage when its
//                      MMAs retire and the accumulator when the tile is done;
//   warps 2..9         the epilogue of tile i (tile_epilogue: two warps per
//                      TMEM lane quarter, splitting the channel chunks, or the
//                      rows of the tail) while tile i+1's loads and MMAs run;
//                      eight warps hide the epilogue's load and store latency
//                      behind one another.
// Loads run ahead across tile boundaries; TMEM is allocated once per CTA.
// The same packed weights, the same MMAs in the same order: results are
// identical to conv3x3_tc_kernel's.
// RESW (layers with one output block, Cout == BN): every K-block's weights
// are copied into shared memory once per CTA, so a ring stage holds only the
// input halo, and more stages fit; the weights are the same for every tile.
// ROWS (2, 4 or 8, persistent kernel only): output rows per tile; a 4-row
// tile reads a 6-row halo for four rows of MMAs (each weight block feeds four
// M tiles) and hands the epilogue two 2-row sub-tiles.
// DYP (row taps packed into N): with BN = 32 or 64 a 128 x BN x 16 MMA is
// bound by the tensor core reading its 4 KB A tile from shared memory, not by
// its math.  So the weights of one column tap dx are packed with the three
// row taps side by side along N, in the order dy = 2, 1, 0, and one MMA per
// (halo row h, dx, K step) multiplies halo row h by all three: its N columns
// land on the accumulators of output rows h-2, h-1, h, which lie next to
// each other in TMEM (row r at column r * BN).  Rows outside the tile are
// left out by narrowing N at the first and last halo rows.  Each output row
// then receives the same products in the same order as with one MMA per tap
// (dy outer, dx, K step inner), so results are bit-identical, from
// ROWS + 2 MMAs per (dx, K step) instead of 3 * ROWS.  The first MMA that
// reaches an output row (dx = 0, first K step of the first K-block) is
// issued alone for that row so that it can overwrite instead of add.
constexpr int kEpiWarps = 8;
constexpr int kPThreads = 64 + 32 * kEpiWarps;
template <int BN, int KC, bool RESW, int ROWS = kRows, int AX = kHaloX>
struct PSmem
{
    using S = Smem<BN, KC, ROWS, AX>;
    static constexpr int kStage = RESW ? ((S::kABytes + 1023) / 1024) * 1024 : S::kStage;
    static constexpr int kBarBytes = 1024;  // mbarriers and the TMEM slot, after the ring
    // dynamic shared memory of a launch with KB K-blocks (1024 B for aligning the base)
    static constexpr int bytes(int stages, int KB)
    {
        return stages * kStage + kBarBytes + (RESW ? KB * S::kBBytes : 0) + 1024;
    }
};
// Folded upsampling (VUP): the first up_C input channels are the nearest 2x
// upsampling of a low-resolution tensor, read as up_h (upsampled along x
// only, H/2 rows).  Output row y reads upsampled rows y-1, y, y+1, which are
// low-resolution rows (y-1)/2, y/2, (y+1)/2: two distinct rows, so the row
// taps fold per parity (even y = 2r: ky0 on row r-1, ky1+ky2 on row r; odd
// y = 2r+1: ky0+ky1 on row r, ky2 on row r+1).  Low-resolution row h then
// reaches the four consecutive output rows 2h-1 .. 2h+2 with weights ky2,
// ky1+ky2, ky0+ky1, ky0: one MMA with N = 4*BN per (row, column tap, K
// step), over ROWS/2 + 2 low-resolution rows instead of ROWS + 2 upsampled
// ones (two thirds of the MMA work, half the rows loaded).  The skip
// channels' K-blocks run first, as in the DYP kernel, so every output row
// is initialised before the folded ones accumulate.
template <int BN, int KC, int STAGES, bool RESW, int ROWS = kRows, bool DYP = false, bool VUP = false>
__global__ void __launch_bounds__(kPThreads, 1) conv3x3_tc_persistent(const __grid_constant__ CUtensorMap tmap,
                                                                      const __grid_constant__ CUtensorMap tmap2,
                                                                      ConvArgs a)
{
    static_assert(ROWS == 2 || ROWS == 4 || ROWS == 8, "2-, 4- or 8-row tiles");
    static_assert(!DYP || 3 * BN <= 256, "row taps packed into N need 3 * BN <= 256");
    static_assert(!VUP || (DYP && !RESW && ROWS >= 4 && 4 * BN <= 256), "folded upsampling: streamed DYP, 4*BN <= 256");
    // DYP kernels load their A tiles through the chunked view (make_map_chunked)
    constexpr int AX = DYP ? kChunkX : kHaloX;  // pixels per halo row in shared memory
    constexpr int AX0 = DYP ? 7 : 0;            // position of pixel x0 - 1 in a halo row
    using S = Smem<BN, KC, ROWS, AX>;
    using P = PSmem<BN, KC, RESW, ROWS, AX>;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * P::kStage);
    uint64_t* empty = full + STAGES;
    uint64_t* acc_full = empty + STAGES;  // [2]
    uint64_t* acc_empty = acc_full + 2;   // [2]
    uint64_t* done = acc_empty + 2;
    uint64_t* wfull = done + 1;  // RESW: the resident weights have landed
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(wfull + 1);
    uint8_t* wres = smem + STAGES * P::kStage + P::kBarBytes;  // RESW: KB x 9 x KC x BN weights
    __shared__ volatile int s_fail;
    __shared__ EpiConsts ec;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    stage_epi_consts(a, ec, tid, kPThreads);  // visible after the __syncthreads below
    const int n_cot = a.Cout / BN;
    const int tiles_x = (a.W + kTileX - 1) / kTileX, tiles_y = (a.H + ROWS - 1) / ROWS;
    const int n_tiles = tiles_x * tiles_y * a.N * n_cot;
    const int KB = a.Cin / KC;
    const int KBS = VUP ? (a.Cin - a.up_C) / KC : KB;  // K-blocks of `in` (the skip channels, with VUP)
    constexpr int kRowsU = ROWS / 2 + 2;                 // VUP: low-resolution rows of a tile
    constexpr uint32_t kAUBytes = (uint32_t)(kRowsU * AX * KC * 2), kBUBytes = (uint32_t)(12 * KC * BN * 2);
    static_assert(!VUP || kAUBytes + kBUBytes <= (uint32_t)P::kStage, "a folded K-block must fit a stage");
    constexpr uint32_t kLboAU = kRowsU * AX * 16, kLboBU = 4 * BN * 16;
    constexpr uint32_t kIdesc4 = tc::idesc_bf16_f32(128, VUP ? 4 * BN : BN);
    constexpr uint32_t kAccCols = ROWS * BN;   // one accumulator: ROWS rows x BN FP32 columns
    constexpr uint32_t kCols = 2 * kAccCols;  // two of them (a power of two >= 32 for BN >= 16)
    static_assert(kCols <= 512, "two accumulators must fit in TMEM");
    constexpr uint32_t kIdesc = tc::idesc_bf16_f32(128, BN);
    constexpr uint32_t kLboA = (ROWS + 2) * AX * 16;
    constexpr uint32_t kLboB = (DYP ? 3 : 1) * BN * 16;
    constexpr uint32_t kIdesc2 = tc::idesc_bf16_f32(128, DYP ? 2 * BN : BN);
    constexpr uint32_t kIdesc3 = tc::idesc_bf16_f32(128, DYP ? 3 * BN : BN);
    // tile t -> (n, ct, y0, x0); output blocks innermost so concurrent tiles share input rows
    auto coords = [&](int t, int& n, int& ct, int& x0, int& y0) {
        ct = t % n_cot;
        t /= n_cot;
        x0 = (t % tiles_x) * kTileX;
        t /= tiles_x;
        y0 = (t % tiles_y) * ROWS;
        n = t / tiles_y;
    };
    auto fail = [&](int code) {
        s_fail = 1;
        if (a.err) atomicExch(a.err, code);
    };

    if (warp == 1)
    {
        tc::tmem_alloc(tmem_slot, kCols);
        tc::tmem_relinquish();
    }
    if (tid == 0)
    {
        s_fail = 0;
        for (int s = 0; s < STAGES; ++s)
        {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b)
        {
            tc::mbar_init(&acc_full[b], 1);
            tc::mbar_init(&acc_empty[b], kEpiWarps);  // one arrival per epilogue warp
        }
        tc::mbar_init(done, 1);
        tc::mbar_init(wfull, 1);
        tc::fence_mbar_init();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0)
    {
        if (lane == 0)
        {
            if (RESW)
            {
                // all K-blocks of the single output block, one bulk copy each
                tc::mbar_expect_tx(wfull, (uint32_t)(KB * S::kBBytes));
                for (int kb = 0; kb < KB; ++kb)
                    tc::bulk_load(wres + kb * S::kBBytes, a.wpack + (size_t)kb * (9 * KC * BN), (uint32_t)S::kBBytes,
                                  wfull);
            }
            int it = 0;
            for (int t = blockIdx.x; t < n_tiles && !s_fail; t += gridDim.x)
            {
                int n, ct, x0, y0;
                coords(t, n, ct, x0, y0);
                const __nv_bfloat16* wsrc =
                    a.wpack + (size_t)ct * (KBS * (9 * KC * BN) + (KB - KBS) * (12 * KC * BN));
                for (int kb = 0; kb < KB; ++kb, ++it)
                {
                    const int s = it % STAGES, u = it / STAGES;
                    if (u > 0 && !tc::mbar_wait(&empty[s], (uint32_t)((u - 1) & 1)))
                    {
                        fail(3);
                        break;
                    }
                    uint8_t* A = smem + s * P::kStage;
                    // x coordinate: pixel x0 - 1; for the 144-pixel rows of the DYP
                    // kernels pixel x0 - 8, or the 8-pixel run that starts there
                    const int ax = DYP ? (a.a_chunked ? x0 / 8 - 1 : x0 - 8) : x0 - 1;
                    if (VUP && kb >= KBS)
                    {
                        // low-resolution rows y0/2 - 1 .. y0/2 + ROWS/2 of up_h, then the K-block's folded weights
                        uint8_t* B = A + kAUBytes;
                        tc::mbar_expect_tx(&full[s], kAUBytes + kBUBytes);
                        tc::tma_load_5d(A, &tmap2, &full[s], 0, ax, y0 / 2 - 1, (kb - KBS) * (KC / 8), n);
                        tc::bulk_load(B, wsrc + (size_t)KBS * (9 * KC * BN) + (size_t)(kb - KBS) * (12 * KC * BN),
                                      kBUBytes, &full[s]);
                    }
                    else if (RESW)
                    {
                        tc::mbar_expect_tx(&full[s], (uint32_t)S::kABytes);
                        tc::tma_load_5d(A, &tmap, &full[s], 0, ax, y0 - 1, kb * (KC / 8), n);
                    }
                    else
                    {
                        uint8_t* B = A + S::kABytes;
                        tc::mbar_expect_tx(&full[s], (uint32_t)(S::kABytes + S::kBBytes));
                        tc::tma_load_5d(A, &tmap, &full[s], 0, ax, y0 - 1, (VUP ? a.up_C / 8 : 0) + kb * (KC / 8), n);
                        tc::bulk_load(B, wsrc + (size_t)kb * (9 * KC * BN), (uint32_t)S::kBBytes, &full[s]);
                    }
                }
            }
        }
    }
    else if (warp == 1)
    {
        if (lane == 0)
        {
            int it = 0, j = 0;
            if (RESW && !tc::mbar_wait(wfull, 0)) fail(5);
            for (int t = blockIdx.x; t < n_tiles && !s_fail; t += gridDim.x, ++j)
            {
                const int b = j & 1, v = j >> 1;
                if (v > 0 && !tc::mbar_wait(&acc_empty[b], (uint32_t)((v - 1) & 1)))
                {
                    fail(4);
                    break;
                }
                tc::tc_fence_after();
                const uint32_t acc = tmem + (uint32_t)b * kAccCols;
                bool ok = true;
                for (int kb = 0; kb < KB; ++kb, ++it)
                {
                    const int s = it % STAGES;
                    if (!tc::mbar_wait(&full[s], (uint32_t)((it / STAGES) & 1)))
                    {
                        ok = false;
                        break;
                    }
                    tc::tc_fence_after();
                    const uint32_t abase = tc::smem_u32(smem + s * P::kStage);
                    const uint32_t bbase =
                        RESW ? tc::smem_u32(wres) + (uint32_t)(kb * S::kBBytes) : abase + (uint32_t)S::kABytes;
                    if (VUP && kb >= KBS)
                    {
                        // folded K-block: weights [dx][KC/8][ky2 | ky1+ky2 | ky0+ky1 | ky0][BN][8]; low-resolution
                        // row h of the tile reaches output rows 2h-3+s (slot s) of those inside the tile
                        const uint32_t ubase = abase + kAUBytes;
#pragma unroll 1
                        for (int h = 0; h < kRowsU; ++h)
                        {
                            const int smin = h == 0 ? 3 : (h == 1 ? 1 : 0);
                            const int smax = ROWS + 2 - 2 * h < 3 ? ROWS + 2 - 2 * h : 3;
                            const int nb = smax - smin + 1;
                            const uint32_t id = nb == 4 ? kIdesc4 : nb == 3 ? kIdesc3 : (nb == 2 ? kIdesc2 : kIdesc);
                            const uint32_t dcol = acc + (uint32_t)((2 * h - 3 + smin) * BN);
#pragma unroll
                            for (int dx = 0; dx < 3; ++dx)
#pragma unroll
                                for (int ks = 0; ks < KC / 16; ++ks)
                                {
                                    const uint32_t aoff =
                                        (uint32_t)(2 * ks) * kLboAU + (uint32_t)((h * AX + AX0 + dx) * 16);
                                    const uint64_t ad = tc::smem_desc(abase + aoff, kLboAU, 128);
                                    const uint32_t plane = ubase + (uint32_t)((dx * (KC / 8) + 2 * ks) * kLboBU);
                                    const uint64_t bd =
                                        tc::smem_desc(plane + (uint32_t)(smin * BN * 16), kLboBU, 128);
                                    tc::mma_bf16(dcol, ad, bd, id, 1u);
                                }
                        }
                    }
                    else if (DYP)
                    {
                        // weights of K-block kb: [dx][KC/8][dy = 2, 1, 0][BN][8]
#pragma unroll 1
                        for (int h = 0; h < ROWS + 2; ++h)
                        {
                            const int dmax = h < 2 ? h : 2;                        // the row taps whose output
                            const int dmin = h - ROWS + 1 > 0 ? h - ROWS + 1 : 0;  // row h - dy is in the tile
                            const int nb = dmax - dmin + 1;
                            const uint32_t id = nb == 3 ? kIdesc3 : (nb == 2 ? kIdesc2 : kIdesc);
                            const uint32_t dcol = acc + (uint32_t)((h - dmax) * BN);
                            const bool first = kb == 0 && dmin == 0;  // output row h starts here
#pragma unroll
                            for (int dx = 0; dx < 3; ++dx)
#pragma unroll
                                for (int ks = 0; ks < KC / 16; ++ks)
                                {
                                    const uint32_t aoff =
                                        (uint32_t)(2 * ks) * kLboA + (uint32_t)((h * AX + AX0 + dx) * 16);
                                    const uint64_t ad = tc::smem_desc(abase + aoff, kLboA, 128);
                                    const uint32_t plane = bbase + (uint32_t)((dx * (KC / 8) + 2 * ks) * kLboB);
                                    const uint64_t bd =
                                        tc::smem_desc(plane + (uint32_t)((2 - dmax) * BN * 16), kLboB, 128);
                                    if (first && dx == 0 && ks == 0)
                                    {
                                        tc::mma_bf16(acc + (uint32_t)(h * BN), ad,
                                                     tc::smem_desc(plane + 2 * BN * 16, kLboB, 128), kIdesc, 0u);
                                        if (dmax > 0) tc::mma_bf16(dcol, ad, bd, dmax == 2 ? kIdesc2 : kIdesc, 1u);
                                    }
                                    else
                                        tc::mma_bf16(dcol, ad, bd, id, 1u);
                                }
                        }
                    }
                    else
                    {
#pragma unroll 1
                        for (int tap = 0; tap < 9; ++tap)
                        {
                            const int dy = tap / 3, dx = tap % 3;
#pragma unroll
                            for (int ks = 0; ks < KC / 16; ++ks)
                            {
                                const uint64_t bd = tc::smem_desc(
                                    bbase + (uint32_t)((tap * (KC / 8) + 2 * ks) * BN * 16), kLboB, 128);
#pragma unroll
                                for (int r = 0; r < ROWS; ++r)
                                {
                                    const uint32_t aoff =
                                        (uint32_t)(2 * ks) * kLboA + (uint32_t)(((r + dy) * AX + dx) * 16);
                                    const uint64_t ad = tc::smem_desc(abase + aoff, kLboA, 128);
                                    tc::mma_bf16(acc + (uint32_t)(r * BN), ad, bd, kIdesc,
                                                 (kb | tap | ks) != 0 ? 1u : 0u);
                                }
                            }
                        }
                    }
                    tc::mma_commit(&empty[s]);  // frees the stage when these MMAs retire
                }
                if (!ok)
                {
                    fail(1);
                    break;
                }
                tc::mma_commit(&acc_full[b]);
            }
            tc::mma_commit(done);  // completes when every MMA issued above has finished
        }
    }
    else
    {
        const int q = warp & 3;                // the TMEM lane quarter this warp may read
        const int part = (warp - 2) >> 2;      // which of the quarter's warps this is
        constexpr int kParts = kEpiWarps / 4;
        int j = 0;
        for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++j)
        {
            const int b = j & 1, v = j >> 1;
            if (!tc::mbar_wait(&acc_full[b], (uint32_t)(v & 1)))
            {
                fail(2);
                break;
            }
            tc::tc_fence_after();
            int n, ct, x0, y0;
            coords(t, n, ct, x0, y0);
#pragma unroll 1
            for (int sub = 0; sub < ROWS / 2; ++sub)  // 2-row sub-tiles
                tile_epilogue<BN>(a, ec, tmem + (uint32_t)b * kAccCols + (uint32_t)(sub * 2 * BN), q, q * 32 + lane,
                                  n, ct, x0, y0 + 2 * sub, part, kParts);
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&acc_empty[b]);
        }
    }
    __syncthreads();
    if (warp == 1)
    {
        bool drained = true;
        if (lane == 0) drained = tc::mbar_wait(done, 0);
        drained = __shfl_sync(0xffffffffu, drained ? 1 : 0, 0) != 0;
        if (!drained && lane == 0 && a.err) atomicExch(a.err, 2);
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, kCols);
    }
}

// ---- host side ----
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    });
    return fn;
}

// 5-D map over a blocked BF16 tensor: (8 channels, W, H, C/8, N), box
// (8, 130, 4, KC/8, 1).
cudaError_t make_map(CUtensorMap* m, const __nv_bfloat16* base, int N, int C, int H, int W, int KC,
                     int halo_y = kHaloY, int box_x = kHaloX)
{
    EncodeTiledFn enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    cuuint64_t dims[5] = {8, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)(C / 8), (cuuint64_t)N};
    cuuint64_t strides[4] = {16, (cuuint64_t)W * 16, (cuuint64_t)H * W * 16, (cuuint64_t)(C / 8) * H * W * 16};
    cuuint32_t box[5] = {8, (cuuint32_t)box_x, (cuuint32_t)halo_y, (cuuint32_t)(KC / 8), 1};
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, (void*)base, dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// Chunked view of the same tensor: (64 = 8 pixels x 8 channels, W/8, H, C/8,
// N), box (64, 18, halo_y, KC/8, 1).  Each box row is 128 contiguous bytes;
// with one pixel per box row (make_map) every 16-byte row costs the TMA unit
// a request and a 32-byte sector.  The box lands in shared memory with the
// same pixel-major layout, 144 pixels per row from pixel x0 - 8 on.  Needs
// W % 8 == 0 (the runs must not cross into the next row); other widths load
// the same 144 pixels one by one (make_map with box_x = 144).
cudaError_t make_map_chunked(CUtensorMap* m, const __nv_bfloat16* base, int N, int C, int H, int W, int KC, int halo_y)
{
    EncodeTiledFn enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    if (W % 8) return cudaErrorInvalidValue;
    cuuint64_t dims[5] = {64, (cuuint64_t)(W / 8), (cuuint64_t)H, (cuuint64_t)(C / 8), (cuuint64_t)N};
    cuuint64_t strides[4] = {128, (cuuint64_t)W * 16, (cuuint64_t)H * W * 16, (cuuint64_t)(C / 8) * H * W * 16};
    cuuint32_t box[5] = {64, (cuuint32_t)(kChunkX / 8), (cuuint32_t)halo_y, (cuuint32_t)(KC / 8), 1};
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, (void*)base, dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// Dynamic shared memory a CTA may use on sm_100: 227 KB less 2 KB of headroom
// for the kernel's static shared memory (the epilogue constants, 1.4 KB).
constexpr int kMaxSmem = 225 * 1024;

template <int BN, int KC, int STAGES, bool RESW = false, int ROWS = kRows, bool DYP = false, bool VUP = false>
cudaError_t launch_persistent(const __nv_bfloat16* in, const ConvArgs& a, cudaStream_t stream)
{
    const int KB = a.Cin / KC;
    if (RESW && a.Cout != BN) return cudaErrorInvalidValue;  // one output block only
    if (VUP != (a.up_C > 0)) return cudaErrorInvalidValue;
    // folded upsampling: both parts whole K-blocks, at least one skip K-block first, even rows
    if (VUP && (!a.up_h || a.up_C % KC || a.Cin - a.up_C < KC || (a.H & 1))) return cudaErrorInvalidValue;
    const int smem = PSmem<BN, KC, RESW, ROWS, DYP ? kChunkX : kHaloX>::bytes(STAGES, KB);
    if (smem > kMaxSmem) return cudaErrorInvalidValue;
    CUtensorMap m, m2;
    ConvArgs b = a;
    b.a_chunked = DYP && a.W % 8 == 0;
    cudaError_t e = !DYP ? make_map(&m, in, a.N, a.Cin, a.H, a.W, KC, ROWS + 2)
                    : b.a_chunked ? make_map_chunked(&m, in, a.N, a.Cin, a.H, a.W, KC, ROWS + 2)
                                  : make_map(&m, in, a.N, a.Cin, a.H, a.W, KC, ROWS + 2, kChunkX);
    if (e != cudaSuccess) return e;
    m2 = m;
    if (VUP)
    {
        e = b.a_chunked ? make_map_chunked(&m2, a.up_h, a.N, a.up_C, a.H / 2, a.W, KC, ROWS / 2 + 2)
                        : make_map(&m2, a.up_h, a.N, a.up_C, a.H / 2, a.W, KC, ROWS / 2 + 2, kChunkX);
        if (e != cudaSuccess) return e;
    }
    auto fn = conv3x3_tc_persistent<BN, KC, STAGES, RESW, ROWS, DYP, VUP>;
    // The resident-weights form's smem depends on KB: size the attribute for
    // the largest launch it may see and query occupancy per launch size.
    static bool attr_done = false;
    static int sm_count = 0;
    if (!attr_done)
    {
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
        if (e != cudaSuccess) return e;
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev);
        attr_done = true;
    }
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kPThreads, smem);
    if (e != cudaSuccess) return e;
    // TMEM: each CTA holds 2*ROWS*BN of the SM's 512 columns for its lifetime
    const int tmem_fit = 512 / (2 * ROWS * BN);
    if (per_sm > tmem_fit) per_sm = tmem_fit;
    if (per_sm < 1) per_sm = 1;
    const long long tiles = (long long)((a.W + kTileX - 1) / kTileX) * ((a.H + ROWS - 1) / ROWS) * a.N * (a.Cout / BN);
    const long long grid = std::min<long long>(tiles, (long long)per_sm * sm_count);
    fn<<<(unsigned)grid, kPThreads, smem, stream>>>(m, m2, b);
    return cudaGetLastError();
}

template <int BN, int KC, int STAGES>
cudaError_t launch(const __nv_bfloat16* in, const ConvArgs& a, cudaStream_t stream)
{
    CUtensorMap m;
    cudaError_t e = make_map(&m, in, a.N, a.Cin, a.H, a.W, KC);
    if (e != cudaSuccess) return e;
    const int smem = STAGES * Smem<BN, KC>::kStage + 1024 + 256;
    static bool attr_done = false;
    if (!attr_done)
    {
        e = cudaFuncSetAttribute(conv3x3_tc_kernel<BN, KC, STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        attr_done = true;
    }
    dim3 grid((a.W + kTileX - 1) / kTileX, (a.H + kRows - 1) / kRows, a.N * (a.Cout / BN));
    conv3x3_tc_kernel<BN, KC, STAGES><<<grid, kThreads, smem, stream>>>(m, a);
    return cudaGetLastError();
}

// Position i of a packed weight array -> (ct, kb, tap, kc8, j, e): output
// block, K-block, tap (dy * 3 + dx), 8-channel plane, output channel in the
// block, channel in the plane.  Plain layout: (ct, kb, tap, kc8, j, e),
// innermost last.  Row taps packed into N (DYP kernels): (ct, kb, dx, kc8,
// 2 - dy, j, e).
__device__ __forceinline__ void packed_index(size_t r, int BN, int KC, int KB, bool dyp, int& ct, int& kb, int& tap,
                                             int& kc8, int& j, int& e)
{
    e = (int)(r % 8); r /= 8;
    j = (int)(r % BN); r /= BN;
    if (dyp)
    {
        const int dyr = (int)(r % 3); r /= 3;
        kc8 = (int)(r % (KC / 8)); r /= (KC / 8);
        const int dx = (int)(r % 3); r /= 3;
        tap = (2 - dyr) * 3 + dx;
    }
    else
    {
        kc8 = (int)(r % (KC / 8)); r /= (KC / 8);
        tap = (int)(r % 9); r /= 9;
    }
    kb = (int)(r % KB); r /= KB;
    ct = (int)r;
}

// Packed forward weight at position i (packed_index layout).
__device__ __forceinline__ float pack_value(const float* __restrict__ w, size_t i, int Cin_real, int Cin, int BN,
                                            int KC, bool dyp)
{
    const int KB = Cin / KC;
    int ct, kb, tap, kc8, j, e;
    packed_index(i, BN, KC, KB, dyp, ct, kb, tap, kc8, j, e);
    const int co = ct * BN + j;
    const int ci = kb * KC + kc8 * 8 + e;
    return ci < Cin_real ? w[(((size_t)co * Cin_real + ci) * 3 + tap / 3) * 3 + tap % 3] : 0.0f;
}

// Input-gradient weight at position i: output (ct, kb, tap, kc8, j, e) of a conv with Cin' = Cout (forward)
// and Cout' = ci_cnt reads w[co = ci'][ci_lo + co'][2-ky][2-kx].
__device__ __forceinline__ float pack_dgrad_value(const float* __restrict__ w, size_t i, int Cout, int Cin_real,
                                                  int ci_lo, int ci_cnt, int BN, int KC, bool dyp)
{
    const int KB = Cout / KC;
    int ct, kb, tap, kc8, j, e;
    packed_index(i, BN, KC, KB, dyp, ct, kb, tap, kc8, j, e);
    const int cop = ct * BN + j;            // output channel of the backward conv
    const int cip = kb * KC + kc8 * 8 + e;  // its input channel = forward output channel
    const int ky = 2 - tap / 3, kx = 2 - tap % 3;
    const int ci = ci_lo + cop;
    return (cop < ci_cnt && ci < Cin_real) ? w[(((size_t)cip * Cin_real + ci) * 3 + ky) * 3 + kx] : 0.0f;
}

__global__ void pack_kernel(const float* __restrict__ w, int Cout, int Cin_real, int Cin, int BN, int KC, int dyp,
                            __nv_bfloat16* __restrict__ out, size_t total)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    out[i] = __float2bfloat16_rn(pack_value(w, i, Cin_real, Cin, BN, KC, dyp != 0));
}

// Every layer of a ConvPackJob list in one launch: thread i packs position i - begin of the job whose
// [begin, begin + elems) range holds i, with the single-layer kernels' arithmetic (identical bits).
struct PackTable
{
    ConvPackJob job[kMaxPackJobs];
    size_t begin[kMaxPackJobs + 1];
    int n;
};
__global__ void pack_many_kernel(const __grid_constant__ PackTable t)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.begin[t.n]) return;
    int k = 0;
    while (i >= t.begin[k + 1]) ++k;
    const ConvPackJob& j = t.job[k];
    const size_t r = i - t.begin[k];
    const float v = j.dgrad ? pack_dgrad_value(j.w, r, j.Cout, j.Cin_real, j.ci_lo, j.ci_cnt, j.bn, j.kc, j.dyp != 0)
                            : pack_value(j.w, r, j.Cin_real, j.Cin, j.bn, j.kc, j.dyp != 0);
    j.out[r] = __float2bfloat16_rn(v);
}

// Folded-upsampling weights (conv_pack_weights_folded): per output block,
// the skip channels up_C..Cin-1 in the DYP layout, then the upsampled
// channels 0..up_C-1 as (kb, dx, kc8, slot, j, e) with the four folded row
// taps of output rows 2h-1 .. 2h+2: ky2, ky1 + ky2, ky0 + ky1, ky0 (summed in
// FP32, rounded once).
__global__ void pack_folded_kernel(const float* __restrict__ w, int Cout, int Cin, int up_C, int BN, int KC,
                                   __nv_bfloat16* __restrict__ out, size_t total)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int KBS = (Cin - up_C) / KC;
    const size_t skip_elems = (size_t)KBS * 9 * KC * BN;
    const size_t per_ct = skip_elems + (size_t)(up_C / KC) * 12 * KC * BN;
    const int ct = (int)(i / per_ct);
    size_t r = i % per_ct;
    float v;
    if (r < skip_elems)
    {
        int ct0, kb, tap, kc8, j, e;
        packed_index(r, BN, KC, KBS, true, ct0, kb, tap, kc8, j, e);
        const int co = ct * BN + j, ci = up_C + kb * KC + kc8 * 8 + e;
        v = w[(((size_t)co * Cin + ci) * 3 + tap / 3) * 3 + tap % 3];
    }
    else
    {
        r -= skip_elems;
        const int e = (int)(r % 8); r /= 8;
        const int j = (int)(r % BN); r /= BN;
        const int slot = (int)(r % 4); r /= 4;
        const int kc8 = (int)(r % (KC / 8)); r /= (KC / 8);
        const int dx = (int)(r % 3); r /= 3;
        const int kb = (int)r;
        const int co = ct * BN + j, ci = kb * KC + kc8 * 8 + e;
        const float* wk = w + ((size_t)co * Cin + ci) * 9 + dx;  // wk[3 * ky]
        v = slot == 0 ? wk[6] : slot == 1 ? wk[3] + wk[6] : slot == 2 ? wk[0] + wk[3] : wk[0];
    }
    out[i] = __float2bfloat16_rn(v);
}

// Input-gradient weights: output (ct, kb, tap, kc8, j, e) of a conv with
// Cin' = Cout (forward) and Cout' = ci_cnt reads w[co = ci'][ci_lo + co'][2-ky][2-kx].

// One thread per (image, 8-channel block, pixel) of the first nb blocks:
// reads the block's channels from their NCHW planes (consecutive threads,
// consecutive pixels of a plane) and writes the pixel's 16 bytes.
__global__ void to_blocked_kernel(const float* __restrict__ x, int N, int C, int H, int W,
                                  __nv_bfloat16* __restrict__ out, int Cpad, int nb, int log1p_in)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // over N * nb * H * W
    const size_t HW = (size_t)H * W;
    if (i >= (size_t)N * nb * HW) return;
    const size_t p = i % HW;
    const int b = (int)((i / HW) % nb);
    const int n = (int)(i / (HW * nb));
    float v[8];
#pragma unroll
    for (int e = 0; e < 8; ++e)
    {
        const int c = b * 8 + e;
        float t = c < C ? x[((size_t)n * C + c) * HW + p] : 0.0f;
        if (log1p_in) t = log1pf(t);
        v[e] = t;
    }
    reinterpret_cast<uint4*>(out)[((size_t)n * (Cpad / 8) + b) * HW + p] = pack8(v);
}

__global__ void from_blocked_kernel(const __nv_bfloat16* __restrict__ in, int N, int C, int H, int W,
                                    float* __restrict__ out)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // over N*C*H*W (NCHW)
    const size_t total = (size_t)N * C * H * W;
    if (i >= total) return;
    size_t r = i;
    const int xx = (int)(r % W); r /= W;
    const int y = (int)(r % H); r /= H;
    const int c = (int)(r % C); r /= C;
    const int n = (int)r;
    out[i] = __bfloat162float(in[((((size_t)n * (C / 8) + c / 8) * H + y) * W + xx) * 8 + c % 8]);
}
}  // namespace

size_t conv_packed_elems(int Cin, int Cout) { return (size_t)9 * Cin * Cout; }

ConvTile conv_default_tile(int Cin, int Cout) { return pick_cfg(Cin, Cout); }

// The shapes conv3x3_forward is compiled for.
constexpr ConvTile kCompiledTiles[] = {{32, 16, 4, 0},  {32, 32, 2, 0},  {32, 32, 4, 0},  {64, 16, 4, 0},
                                       {64, 32, 2, 0},  {64, 32, 3, 0},  {128, 16, 3, 0}, {128, 32, 2, 0},
                                       {32, 16, 4, 1},  {32, 32, 2, 1},  {32, 32, 4, 1},  {64, 16, 4, 1},
                                       {64, 32, 2, 1},  {64, 32, 3, 1},  {128, 16, 3, 1}, {128, 32, 2, 1},
                                       {32, 16, 10, 2}, {32, 32, 2, 2},  {32, 32, 5, 2},  {32, 32, 6, 2},
                                       {64, 32, 3, 2},  {64, 32, 4, 2},  {32, 16, 8, 3},  {32, 32, 3, 3},
                                       {32, 32, 4, 3},  {64, 32, 3, 3},  {32, 16, 7, 4},  {32, 32, 3, 4},
                                       {64, 32, 2, 4},  {64, 32, 3, 4},  {32, 16, 4, 5},  {32, 32, 2, 5},
                                       {64, 32, 2, 6},  {32, 32, 3, 6},  {32, 32, 2, 7}};

// Kernel choices (ConvTile::persist): 0 one tile per CTA; 1 persistent; 2 resident weights; 3 resident weights,
// 4-row tiles; 4 as 3 with the row taps packed into N (and A tiles through the chunked view); 5 the same on
// 8-row tiles; 6 and 7: row taps packed into N with streamed weights, 4- and 8-row tiles.
static bool tile_resident(int p) { return p >= 2 && p <= 5; }
static int tile_rows(int p) { return (p == 5 || p == 7) ? 8 : (p == 3 || p == 4 || p == 6) ? 4 : 2; }
static bool tile_dyp(int p) { return p >= 4; }

// Shared memory of a tile shape's launch for a layer with Cin input channels.
int tile_smem(const ConvTile& t, int Cin)
{
    const int KB = Cin / t.kc;
    const int a = (tile_rows(t.persist) + 2) * (tile_dyp(t.persist) ? kChunkX : kHaloX) * t.kc * 2,
              b = 9 * t.kc * t.bn * 2;
    if (tile_resident(t.persist)) return t.stages * (((a + 1023) / 1024) * 1024) + 1024 + KB * b + 1024;
    return t.stages * (((a + b + 1023) / 1024) * 1024) + 1024 + 1024;
}

int conv_tile_candidates(int Cin, int Cout, ConvTile* out, int max)
{
    int k = 0;
    for (const ConvTile& t : kCompiledTiles)
        if (k < max && t.bn <= Cout && Cout % t.bn == 0 && Cin % t.kc == 0 &&
            (t.persist < 2 || ((t.bn == Cout || !tile_resident(t.persist)) && tile_smem(t, Cin) <= kMaxSmem)))
            out[k++] = t;
    return k;
}

static ConvTile resolve(ConvTile t, int Cin, int Cout) { return t.bn ? t : pick_cfg(Cin, Cout); }

cudaError_t conv_pack_weights(const float* d_w, int Cout, int Cin_real, int Cin, __nv_bfloat16* d_packed,
                              cudaStream_t stream, ConvTile tile)
{
    const TileCfg c = resolve(tile, Cin, Cout);
    const size_t total = conv_packed_elems(Cin, Cout);
    pack_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(d_w, Cout, Cin_real, Cin, c.bn, c.kc,
                                                                     tile_dyp(c.persist) ? 1 : 0, d_packed, total);
    return cudaGetLastError();
}

size_t conv_packed_elems_folded(int Cin, int Cout, int up_C)
{
    return (size_t)9 * (Cin - up_C) * Cout + (size_t)12 * up_C * Cout;
}

bool conv_tile_folds(ConvTile tile, int Cin, int Cout, int up_C)
{
    const TileCfg c = resolve(tile, Cin, Cout);
    const int key = c.bn * 1000 + c.kc * 10 + c.stages;
    const bool compiled = (c.persist == 7 && key == 32322) || (c.persist == 6 && (key == 64322 || key == 32323));
    return compiled && up_C > 0 && up_C % c.kc == 0 && Cin - up_C >= c.kc && (Cin - up_C) % c.kc == 0 &&
           Cout % c.bn == 0;
}

cudaError_t conv_pack_weights_folded(const float* d_w, int Cout, int Cin, int up_C, __nv_bfloat16* d_packed,
                                     cudaStream_t stream, ConvTile tile)
{
    if (!conv_tile_folds(tile, Cin, Cout, up_C)) return cudaErrorInvalidValue;
    const TileCfg c = resolve(tile, Cin, Cout);
    const size_t total = conv_packed_elems_folded(Cin, Cout, up_C);
    pack_folded_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(d_w, Cout, Cin, up_C, c.bn, c.kc,
                                                                            d_packed, total);
    return cudaGetLastError();
}

ConvPackJob conv_pack_job(const float* d_w, int Cout, int Cin_real, int Cin, __nv_bfloat16* d_packed, ConvTile tile)
{
    const TileCfg c = resolve(tile, Cin, Cout);
    ConvPackJob j{};
    j.w = d_w;
    j.out = d_packed;
    j.elems = conv_packed_elems(Cin, Cout);
    j.Cout = Cout;
    j.Cin_real = Cin_real;
    j.Cin = Cin;
    j.bn = c.bn;
    j.kc = c.kc;
    j.dyp = tile_dyp(c.persist) ? 1 : 0;
    return j;
}

ConvPackJob conv_pack_job_dgrad(const float* d_w, int Cout, int Cin_real, int ci_lo, int ci_cnt,
                                __nv_bfloat16* d_packed, ConvTile tile)
{
    const TileCfg c = resolve(tile, Cout, ci_cnt);
    ConvPackJob j{};
    j.w = d_w;
    j.out = d_packed;
    j.elems = conv_packed_elems(Cout, ci_cnt);
    j.Cout = Cout;
    j.Cin_real = Cin_real;
    j.bn = c.bn;
    j.kc = c.kc;
    j.dyp = tile_dyp(c.persist) ? 1 : 0;
    j.dgrad = 1;
    j.ci_lo = ci_lo;
    j.ci_cnt = ci_cnt;
    return j;
}

cudaError_t conv_pack_many(const ConvPackJob* jobs, int n, cudaStream_t stream)
{
    if (n < 0 || n > kMaxPackJobs) return cudaErrorInvalidValue;
    if (n == 0) return cudaSuccess;
    PackTable t{};
    t.n = n;
    t.begin[0] = 0;
    for (int k = 0; k < n; ++k)
    {
        t.job[k] = jobs[k];
        t.begin[k + 1] = t.begin[k] + jobs[k].elems;
    }
    const size_t total = t.begin[n];
    pack_many_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(t);
    return cudaGetLastError();
}


cudaError_t conv3x3_forward(const __nv_bfloat16* in, const ConvArgs& a, cudaStream_t stream)
{
    if (a.Cin % 16 != 0 || (a.Cout != 32 && a.Cout != 64 && a.Cout != 128 && a.Cout != 256)) return cudaErrorInvalidValue;
    if (a.epilogue == kEpiTail && a.Cout != 32) return cudaErrorInvalidValue;
    if (a.epilogue == kEpiStore && a.out2 && ((a.H & 1) || (a.W & 1))) return cudaErrorInvalidValue;
    if (a.epilogue == kEpiBwdSumPool && ((a.H & 1) || (a.W & 1))) return cudaErrorInvalidValue;
    if ((a.epilogue == kEpiBwdMask || a.epilogue == kEpiBwdSumPool || a.epilogue == kEpiBwdUnpool) && !a.ref)
        return cudaErrorInvalidValue;
    if (a.epilogue == kEpiBwdUnpool && !a.skip) return cudaErrorInvalidValue;
    const TileCfg c = resolve(a.tile, a.Cin, a.Cout);
    if (a.Cout % c.bn || a.Cin % c.kc) return cudaErrorInvalidValue;
    const int key = c.bn * 1000 + c.kc * 10 + c.stages;
    if (a.up_C > 0)
    {
        if (!conv_tile_folds(c, a.Cin, a.Cout, a.up_C)) return cudaErrorInvalidValue;
        if (c.persist == 7) return launch_persistent<32, 32, 2, false, 8, true, true>(in, a, stream);
        if (key == 64322) return launch_persistent<64, 32, 2, false, 4, true, true>(in, a, stream);
        return launch_persistent<32, 32, 3, false, 4, true, true>(in, a, stream);
    }
    if (c.persist == 7)
        switch (key)
        {
        case 32322: return launch_persistent<32, 32, 2, false, 8, true>(in, a, stream);
        default: return cudaErrorInvalidValue;
        }
    if (c.persist == 6)
        switch (key)
        {
        case 64322: return launch_persistent<64, 32, 2, false, 4, true>(in, a, stream);
        case 32323: return launch_persistent<32, 32, 3, false, 4, true>(in, a, stream);
        default: return cudaErrorInvalidValue;
        }
    if (c.persist == 5)
        switch (key)
        {
        case 32164: return launch_persistent<32, 16, 4, true, 8, true>(in, a, stream);
        case 32322: return launch_persistent<32, 32, 2, true, 8, true>(in, a, stream);
        default: return cudaErrorInvalidValue;
        }
    if (c.persist == 4)
        switch (key)
        {
        case 32167: return launch_persistent<32, 16, 7, true, 4, true>(in, a, stream);
        case 32323: return launch_persistent<32, 32, 3, true, 4, true>(in, a, stream);
        case 64322: return launch_persistent<64, 32, 2, true, 4, true>(in, a, stream);
        case 64323: return launch_persistent<64, 32, 3, true, 4, true>(in, a, stream);
        default: return cudaErrorInvalidValue;
        }
    if (c.persist == 3)
        switch (key)
        {
        case 32168: return launch_persistent<32, 16, 8, true, 4>(in, a, stream);
        case 32323: return launch_persistent<32, 32, 3, true, 4>(in, a, stream);
        case 32324: return launch_persistent<32, 32, 4, true, 4>(in, a, stream);
        case 64323: return launch_persistent<64, 32, 3, true, 4>(in, a, stream);
        default: return cudaErrorInvalidValue;
        }
    if (c.persist == 2)
        switch (key)
        {
        case 32170: return launch_persistent<32, 16, 10, true>(in, a, stream);
        case 32322: return launch_persistent<32, 32, 2, true>(in, a, stream);
        case 32325: return launch_persistent<32, 32, 5, true>(in, a, stream);
        case 32326: return launch_persistent<32, 32, 6, true>(in, a, stream);
        case 64323: return launch_persistent<64, 32, 3, true>(in, a, stream);
        case 64324: return launch_persistent<64, 32, 4, true>(in, a, stream);
        default: return cudaErrorInvalidValue;
        }
    if (c.persist)
        switch (key)
        {
        case 32164: return launch_persistent<32, 16, 4>(in, a, stream);
        case 32322: return launch_persistent<32, 32, 2>(in, a, stream);
        case 32324: return launch_persistent<32, 32, 4>(in, a, stream);
        case 64164: return launch_persistent<64, 16, 4>(in, a, stream);
        case 64322: return launch_persistent<64, 32, 2>(in, a, stream);
        case 64323: return launch_persistent<64, 32, 3>(in, a, stream);
        case 128163: return launch_persistent<128, 16, 3>(in, a, stream);
        case 128322: return launch_persistent<128, 32, 2>(in, a, stream);
        default: return cudaErrorInvalidValue;
        }
    switch (key)
    {
    case 32164: return launch<32, 16, 4>(in, a, stream);
    case 32322: return launch<32, 32, 2>(in, a, stream);
    case 32324: return launch<32, 32, 4>(in, a, stream);
    case 64164: return launch<64, 16, 4>(in, a, stream);
    case 64322: return launch<64, 32, 2>(in, a, stream);
    case 64323: return launch<64, 32, 3>(in, a, stream);
    case 128163: return launch<128, 16, 3>(in, a, stream);
    case 128322: return launch<128, 32, 2>(in, a, stream);
    }
    return cudaErrorInvalidValue;
}

cudaError_t to_blocked_bf16(const float* x, int N, int C, int H, int W, __nv_bfloat16* out, int Cpad,
                            cudaStream_t stream, bool log1p_in, bool skip_zero_blocks)
{
    const int nb = skip_zero_blocks ? (C + 7) / 8 : Cpad / 8;
    const size_t total = (size_t)N * nb * H * W;
    to_blocked_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(x, N, C, H, W, out, Cpad, nb,
                                                                         log1p_in ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t from_blocked_bf16(const __nv_bfloat16* in, int N, int C, int H, int W, float* out, cudaStream_t stream)
{
    const size_t total = (size_t)N * C * H * W;
    from_blocked_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(in, N, C, H, W, out);
    return cudaGetLastError();
}
namespace
{
__global__ void wait_probe_kernel(int* err, unsigned long long limit_ns)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0)
    {
        tc::mbar_init(&bar, 1);
        tc::fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && !tc::mbar_wait(&bar, 0, limit_ns)) atomicExch(err, 3);
}
}  // namespace

cudaError_t launch_wait_probe(int* err, unsigned long long limit_ns, cudaStream_t stream)
{
    wait_probe_kernel<<<1, 32, 0, stream>>>(err, limit_ns);
    return cudaGetLastError();
}
}  // namespace lg
