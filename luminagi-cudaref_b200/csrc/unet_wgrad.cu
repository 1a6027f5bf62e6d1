// unet_wgrad.cu -- weight gradient of a 3x3 convolution on tcgen05.
//
//   dW[co][ci][ky][kx] += sum over (n, y, x) of dZ[n][co][y][x] * X[n][ci][y+ky-1][x+kx-1]
//
// A GEMM with M = output channels (128 per CTA), N = input channels (BNW per
// CTA), K = pixels.  Both operands come straight from the channel-blocked
// BF16 activations: a TMA box of 8 channels x 128 pixels per channel block
// is, in shared memory, a stack of 8-pixel x 8-channel core matrices -- the
// MMA's MN-major no-swizzle layout with K = pixels.  One CTA owns one kernel
// row ky and all three kx taps: the X box is 130 pixels wide and tap kx reads
// it 16*kx bytes further on, accumulating into three TMEM tiles.  Each CTA
// sums a chunk of image rows and stores its partial dW in a scratch slice of
// its own; a second pass adds the chunks' partials to dW in a fixed order, so
// gradients (and training) are bit-reproducible.
// A K-step is 128 pixels: one 128-pixel row segment for layers wider than 64
// pixels; for narrower ones (the deep levels of training crops) R rows of Wp
// pixels (Wp = W rounded up to 16, R * Wp <= 128) with one MMA per 16 pixels
// of a row, so the step is not mostly zero padding.
// Layers with 32 output channels (KYP) fill M with the three kernel rows
// instead of zeros: the A tile stacks dZ rows y+1, y, y-1 (ky = 0, 1, 2) of
// channels 0..31 against X row y, so one CTA and one B tile serve all three
// kernel rows; TMEM lane 32 * ky + co holds dW[co][.][ky][.].
#include <algorithm>
#include <cstdint>
#include <mutex>

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.h"
#include "tc_ptx.cuh"
#include "unet_wgrad.cuh"

namespace lg
{
namespace
{
constexpr int kPix = 128;         // pixels per K-step
constexpr int kThreads = 128;
constexpr int kStages = 3;
constexpr int kMaxRowPix = 144;   // the largest R * (Wp + 2) of a step (R = 8, Wp = 16)

// Rows and pixels per row of a K-step for width W.
__host__ __device__ inline void step_shape(int W, int& R, int& Wp)
{
    if (W > 64)
    {
        R = 1;
        Wp = kPix;
        return;
    }
    Wp = (W + 15) / 16 * 16;
    R = kPix / Wp;
}

template <int BNW>
struct WSmem
{
    static constexpr int kABytes = 16 * kPix * 16;  // 16 channel blocks (M = 128) x 128 px
    static constexpr int kMaxStage = ((kABytes + (BNW / 8) * kMaxRowPix * 16 + 1023) / 1024) * 1024;
    // B: BNW/8 channel blocks x R rows x (Wp + 2) pixels
    __host__ __device__ static int stage(int R, int Wp)
    {
        return ((kABytes + (BNW / 8) * R * (Wp + 2) * 16 + 1023) / 1024) * 1024;
    }
};

template <int BNW, bool KYP>
__global__ void __launch_bounds__(kThreads, 1)
    wgrad_kernel(const __grid_constant__ CUtensorMap map_dz, const __grid_constant__ CUtensorMap map_x, WgradArgs a)
{
    using S = WSmem<BNW>;
    int R, Wp;
    step_shape(a.W, R, Wp);
    const int kStage = S::stage(R, Wp);
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStage);
    uint64_t* empty = full + kStages;
    uint64_t* done = empty + kStages;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    __shared__ int s_fail;

    const int tid = threadIdx.x, warp = tid >> 5;
    const int n_cit = a.Cin / BNW;
    const int ky = KYP ? 0 : blockIdx.y / n_cit;  // KYP: all three
    const int ci0 = (blockIdx.y % n_cit) * BNW;
    const int co0 = blockIdx.z * 128;
    const int gpi = (a.H + R - 1) / R;  // row groups per image
    const int groups = a.N * gpi;
    const int g0 = blockIdx.x * a.rows_per_cta;  // this CTA's row groups
    const int g1 = min(groups, g0 + a.rows_per_cta);
    const int xsegs = (a.W + Wp - 1) / Wp;
    const int steps = (g1 - g0) * xsegs;
    const int co_blocks = min(16, (a.Cout - co0) / 8);  // channel blocks loaded; the rest stay zero
    constexpr uint32_t kCols = (3 * BNW <= 32) ? 32 : (3 * BNW <= 64) ? 64 : (3 * BNW <= 128) ? 128 : (3 * BNW <= 256) ? 256 : 512;
    // M = 128, N = BNW, both operands MN-major.
    constexpr uint32_t kIdesc = tc::idesc_bf16_f32(128, BNW) | (1u << 15) | (1u << 16);
    const uint32_t a_bytes = (uint32_t)((KYP ? 12 : co_blocks) * R * Wp * 16);
    const uint32_t b_bytes = (uint32_t)((BNW / 8) * R * (Wp + 2) * 16);
    const uint32_t a_sbo = (uint32_t)(R * Wp * 16), b_sbo = (uint32_t)(R * (Wp + 2) * 16);  // channel-block strides

    // Zero the A buffers once: channel blocks beyond Cout are never written by TMA.
    for (int i = tid; i < kStages * kStage / 16; i += kThreads)
        reinterpret_cast<uint4*>(smem)[i] = make_uint4(0, 0, 0, 0);
    tc::fence_proxy_async();
    if (warp == 0)
    {
        tc::tmem_alloc(tmem_slot, kCols);
        tc::tmem_relinquish();
    }
    if (tid == 0)
    {
        s_fail = 0;
        for (int s = 0; s < kStages; ++s)
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

    if (tid == 0 && steps > 0)
    {
        auto issue = [&](int s, int step) {
            const int g = g0 + step / xsegs;
            const int x0 = (step % xsegs) * Wp;
            const int n = g / gpi, y = (g % gpi) * R;
            uint8_t* A = smem + s * kStage;
            uint8_t* B = A + S::kABytes;
            tc::mbar_expect_tx(&full[s], a_bytes + b_bytes);
            if (KYP)
            {
                // M blocks 4 * k .. 4 * k + 3: dZ rows y + 1 - k against X rows y (kernel row k)
                for (int k = 0; k < 3; ++k)
                    tc::tma_load_5d(A + k * 4 * R * Wp * 16, &map_dz, &full[s], 0, x0, y + 1 - k, 0, n);
                tc::tma_load_5d(B, &map_x, &full[s], 0, x0 - 1, y, ci0 / 8, n);
            }
            else
            {
                tc::tma_load_5d(A, &map_dz, &full[s], 0, x0, y, co0 / 8, n);
                tc::tma_load_5d(B, &map_x, &full[s], 0, x0 - 1, y + ky - 1, ci0 / 8, n);
            }
        };
        const int pre = steps < kStages ? steps : kStages;
        for (int s = 0; s < pre; ++s) issue(s, s);
        bool ok = true;
        for (int step = 0; step < steps; ++step)
        {
            const int s = step % kStages;
            if (!tc::mbar_wait(&full[s], (uint32_t)((step / kStages) & 1))) { ok = false; break; }
            tc::tc_fence_after();
            const uint32_t abase = tc::smem_u32(smem + s * kStage);
            const uint32_t bbase = abase + S::kABytes;
#pragma unroll 1
            for (int dx = 0; dx < 3; ++dx)
#pragma unroll 1
                for (int r = 0; r < R; ++r)
                    for (int ks = 0; ks < Wp / 16; ++ks)
                    {
                        const uint64_t ad = tc::smem_desc(abase + (uint32_t)((r * Wp + ks * 16) * 16), 128, a_sbo);
                        const uint64_t bd =
                            tc::smem_desc(bbase + (uint32_t)((r * (Wp + 2) + ks * 16 + dx) * 16), 128, b_sbo);
                        tc::mma_bf16(tmem + (uint32_t)(dx * BNW), ad, bd, kIdesc, (step | r | ks) != 0 ? 1u : 0u);
                    }
            tc::mma_commit(&empty[s]);
            if (step >= 1)
            {
                const int ps = (step - 1) % kStages;
                const int nk = step - 1 + kStages;
                if (nk < steps)
                {
                    if (!tc::mbar_wait(&empty[ps], (uint32_t)(((step - 1) / kStages) & 1))) { ok = false; break; }
                    issue(ps, nk);
                }
            }
        }
        if (!ok)
        {
            s_fail = 1;
            if (a.err) atomicExch(a.err, 3);
        }
        tc::mma_commit(done);
    }
    __syncwarp();
    // This CTA's slice of the scratch: chunk blockIdx.x of [chunk][ky][kx][Cin_real][Cout], output channels
    // innermost so that a warp's 32 lanes (32 output channels) store 128 contiguous bytes.
    float* part = a.partial + (size_t)blockIdx.x * a.Cout * a.Cin_real * 9;
    // TMEM lane = output channel; with KYP, lane 32 * k + co is kernel row k
    const int co = KYP ? (tid & 31) : co0 + tid;
    const int kyo = KYP ? (tid >> 5) : ky;
    bool have = false;
    if (steps > 0)
    {
        const bool got = tc::mbar_wait(done, 0);
        if (!got && a.err) atomicExch(a.err, 4);
        tc::tc_fence_after();
        have = got && !s_fail;
    }
    const uint32_t lanebase = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int dx = 0; dx < 3; ++dx)
#pragma unroll 1
        for (int c0 = 0; c0 < BNW; c0 += 16)
        {
            float v[16];
            if (have) tc::tmem_ld16(lanebase + (uint32_t)(dx * BNW + c0), v);
            else
            {
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = 0.0f;  // an empty chunk (or a failed one) adds zeros
            }
            if (co < a.Cout && kyo < 3)
            {
#pragma unroll
                for (int j = 0; j < 16; ++j)
                {
                    const int ci = ci0 + c0 + j;
                    if (ci < a.Cin_real) part[((size_t)(kyo * 3 + dx) * a.Cin_real + ci) * a.Cout + co] = v[j];
                }
            }
        }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0)
    {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, kCols);
    }
}

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

cudaError_t make_map(CUtensorMap* m, const __nv_bfloat16* base, int N, int C, int H, int W, int box_x, int box_y,
                     int box_cb)
{
    EncodeTiledFn enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    cuuint64_t dims[5] = {8, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)(C / 8), (cuuint64_t)N};
    cuuint64_t strides[4] = {16, (cuuint64_t)W * 16, (cuuint64_t)H * W * 16, (cuuint64_t)(C / 8) * H * W * 16};
    cuuint32_t box[5] = {8, (cuuint32_t)box_x, (cuuint32_t)box_y, (cuuint32_t)box_cb, 1};
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, (void*)base, dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// dw[co][ci][ky][kx] += the chunks' partials of that weight, in a fixed
// order: a block takes 32 consecutive partial entries ([ky][kx][ci][co]
// order, so reads are coalesced) and splits the chunks into 8 consecutive
// slices, one warp each; the slice sums are then added in slice order.
__global__ void __launch_bounds__(256) wgrad_reduce_kernel(const float* __restrict__ partial, int chunks, int Cout,
                                                           int Cin_real, float* __restrict__ dw)
{
    __shared__ float t[8][32];
    const size_t n = (size_t)Cout * Cin_real * 9;
    const int lane = threadIdx.x & 31, slice = threadIdx.x >> 5;
    const size_t e = (size_t)blockIdx.x * 32 + lane;
    const int per = (chunks + 7) / 8;
    const int c0 = slice * per, c1 = min(chunks, c0 + per);
    float s = 0.0f;
    if (e < n)
        for (int c = c0; c < c1; ++c) s += partial[(size_t)c * n + e];
    t[slice][lane] = s;
    __syncthreads();
    if (slice == 0 && e < n)
    {
        float tot = t[0][lane];
#pragma unroll
        for (int k = 1; k < 8; ++k) tot += t[k][lane];
        const int co = (int)(e % Cout);
        const size_t r = e / Cout;
        const int ci = (int)(r % Cin_real), tap = (int)(r / Cin_real);  // tap = ky * 3 + kx
        dw[((size_t)co * Cin_real + ci) * 9 + tap] += tot;
    }
}

// Chunks of a launch: about two CTAs per SM over the (ky, input block,
// output block) grid, at most one per row group (R rows of the K-step shape
// for width W; W = 0 counts single rows, an upper bound for sizing scratch).
int wgrad_chunks(int N, int H, int W, int Cout, int Cin, int bnw, int sm_count, int* rows_per_cta)
{
    const int cot = (Cout + 127) / 128, cit = Cin / bnw;
    const int kys = Cout == 32 ? 1 : 3;  // CTAs per (input block, output block): one with the kernel rows in M
    int R = 1, Wp = kPix;
    if (W > 0) step_shape(W, R, Wp);
    const int rows = N * ((H + R - 1) / R);
    int chunks = (2 * sm_count) / (kys * cit * cot);
    if (chunks < 1) chunks = 1;
    if (chunks > rows) chunks = rows;
    const int rpc = (rows + chunks - 1) / chunks;
    if (rows_per_cta) *rows_per_cta = rpc;
    return (rows + rpc - 1) / rpc;
}

int wgrad_bnw(int Cin) { return Cin % 128 == 0 ? 128 : Cin % 64 == 0 ? 64 : Cin % 32 == 0 ? 32 : 16; }

template <int BNW, bool KYP>
cudaError_t launch_w(const __nv_bfloat16* dz, const __nv_bfloat16* x, const WgradArgs& a, int sm_count,
                     cudaStream_t stream)
{
    int R, Wp;
    step_shape(a.W, R, Wp);
    CUtensorMap mdz, mx;
    cudaError_t e = make_map(&mdz, dz, a.N, a.Cout, a.H, a.W, Wp, R, a.Cout / 8 < 16 ? a.Cout / 8 : 16);
    if (e != cudaSuccess) return e;
    e = make_map(&mx, x, a.N, a.Cin, a.H, a.W, Wp + 2, R, BNW / 8);
    if (e != cudaSuccess) return e;
    const int smem_max = kStages * WSmem<BNW>::kMaxStage + 1024 + 256;
    const int smem = kStages * WSmem<BNW>::stage(R, Wp) + 1024 + 256;
    static bool attr = false;
    if (!attr)
    {
        e = cudaFuncSetAttribute(wgrad_kernel<BNW, KYP>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    WgradArgs b = a;
    const int cot = (a.Cout + 127) / 128, cit = a.Cin / BNW;
    const int chunks = wgrad_chunks(a.N, a.H, a.W, a.Cout, a.Cin, BNW, sm_count, &b.rows_per_cta);
    dim3 grid(chunks, (KYP ? 1 : 3) * cit, cot);
    wgrad_kernel<BNW, KYP><<<grid, kThreads, smem, stream>>>(mdz, mx, b);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const size_t n = (size_t)a.Cout * a.Cin_real * 9;
    wgrad_reduce_kernel<<<(unsigned)((n + 31) / 32), 256, 0, stream>>>(b.partial, chunks, a.Cout, a.Cin_real, a.dw);
    return cudaGetLastError();
}

constexpr int kBiasBlocks = 64;  // blocks per 8-channel group; each writes its own partial
// Block `chunk` of 8-channel group cb of dz (N x C x HW, blocked BF16): the sum of its pixels p = chunk*256 + t,
// stepping by kBiasBlocks*256, per thread, then over the warps in order, into out[0..7].
__device__ __forceinline__ void bias_block_sum(const __nv_bfloat16* __restrict__ dz, int N, int C, int HW, int cb,
                                               int chunk, float* __restrict__ out)
{
    __shared__ float warp_sum[8][8];
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const size_t pixels = (size_t)N * HW;
    for (size_t p = (size_t)chunk * blockDim.x + threadIdx.x; p < pixels; p += (size_t)kBiasBlocks * blockDim.x)
    {
        const size_t n = p / HW, q = p % HW;
        const uint4 u = __ldg(reinterpret_cast<const uint4*>(dz + ((n * (C / 8) + cb) * HW + q) * 8));
        const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
            const float2 f = __bfloat1622float2(h[i]);
            acc[2 * i] += f.x;
            acc[2 * i + 1] += f.y;
        }
    }
    const int warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < 8; ++i)
    {
        float v = acc[i];
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) warp_sum[warp][i] = v;
    }
    __syncthreads();
    if (threadIdx.x < 8)
    {
        float s = 0.0f;
        for (int w = 0; w < 8; ++w) s += warp_sum[w][threadIdx.x];  // warps in order
        out[threadIdx.x] = s;
    }
}

// Several layers' bias gradients: blockIdx.y runs over every layer's 8-channel groups (group g of the whole
// list belongs to the job k with gbegin[k] <= g < gbegin[k+1]); block (chunk, g) writes the 8 partials
// partial[(g * kBiasBlocks + chunk) * 8 ..].
struct BiasTable
{
    BiasGradJob job[kMaxBiasJobs];
    int gbegin[kMaxBiasJobs + 1];  // 8-channel groups before job k
    int n;
};
__global__ void bias_grad_many_kernel(const __grid_constant__ BiasTable t, float* __restrict__ partial)
{
    const int g = blockIdx.y;
    int k = 0;
    while (g >= t.gbegin[k + 1]) ++k;
    const BiasGradJob& j = t.job[k];
    bias_block_sum(j.dz, j.N, j.C, j.HW, g - t.gbegin[k], blockIdx.x,
                   partial + ((size_t)g * kBiasBlocks + blockIdx.x) * 8);
}
// db[c] += the kBiasBlocks partials of channel c, in block order, for every job's channels.
__global__ void bias_reduce_many_kernel(const __grid_constant__ BiasTable t, const float* __restrict__ partial)
{
    const int gc = blockIdx.x * blockDim.x + threadIdx.x;  // channel in the whole list
    if (gc >= 8 * t.gbegin[t.n]) return;
    int k = 0;
    while (gc >= 8 * t.gbegin[k + 1]) ++k;
    const int g = gc >> 3, i = gc & 7;
    float s = 0.0f;
    for (int b = 0; b < kBiasBlocks; ++b) s += partial[((size_t)g * kBiasBlocks + b) * 8 + i];
    t.job[k].db[gc - 8 * t.gbegin[k]] += s;
}

}  // namespace

size_t conv3x3_wgrad_partial_floats(int N, int H, int Cout, int Cin, int Cin_real, int sm_count)
{
    const int chunks = wgrad_chunks(N, H, 0, Cout, Cin, wgrad_bnw(Cin), sm_count, nullptr);
    return (size_t)chunks * Cout * Cin_real * 9;
}

cudaError_t conv3x3_wgrad(const __nv_bfloat16* dz, const __nv_bfloat16* x, const WgradArgs& a, int sm_count,
                          cudaStream_t stream)
{
    if (a.Cout % 32 || a.Cin % 16 || !a.partial) return cudaErrorInvalidValue;
    const int bnw = wgrad_bnw(a.Cin);
    if (a.Cout == 32)  // the three kernel rows share M
        switch (bnw)
        {
        case 128: return launch_w<128, true>(dz, x, a, sm_count, stream);
        case 64: return launch_w<64, true>(dz, x, a, sm_count, stream);
        case 32: return launch_w<32, true>(dz, x, a, sm_count, stream);
        default: return launch_w<16, true>(dz, x, a, sm_count, stream);
        }
    switch (bnw)
    {
    case 128: return launch_w<128, false>(dz, x, a, sm_count, stream);
    case 64: return launch_w<64, false>(dz, x, a, sm_count, stream);
    case 32: return launch_w<32, false>(dz, x, a, sm_count, stream);
    default: return launch_w<16, false>(dz, x, a, sm_count, stream);
    }
}

size_t conv_bias_grad_partial_floats(int C) { return (size_t)(C / 8) * kBiasBlocks * 8; }

cudaError_t conv_bias_grad_many(const BiasGradJob* jobs, int n, float* partial, cudaStream_t stream)
{
    if (n < 0 || n > kMaxBiasJobs || !partial) return cudaErrorInvalidValue;
    if (n == 0) return cudaSuccess;
    BiasTable t{};
    t.n = n;
    for (int k = 0; k < n; ++k)
    {
        if (jobs[k].C % 8) return cudaErrorInvalidValue;
        t.job[k] = jobs[k];
        t.gbegin[k + 1] = t.gbegin[k] + jobs[k].C / 8;
    }
    bias_grad_many_kernel<<<dim3(kBiasBlocks, t.gbegin[n]), 256, 0, stream>>>(t, partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    bias_reduce_many_kernel<<<(8 * t.gbegin[n] + 255) / 256, 256, 0, stream>>>(t, partial);
    return cudaGetLastError();
}

}  // namespace lg
