// radix_sort.cu -- see radix_sort.cuh.
#include "radix_sort.cuh"

namespace lg
{
namespace
{
constexpr int kThreads = 256;
constexpr int kItems = 16;  // keys per thread per tile
constexpr int kTile = kThreads * kItems;
constexpr int kWarps = kThreads / 32;

size_t tiles_for(size_t n) { return (n + kTile - 1) / kTile; }
size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

__global__ void __launch_bounds__(kThreads) hist_kernel(const uint32_t* __restrict__ keys, size_t n, int shift,
                                                        int bits, uint32_t* __restrict__ counts, int tiles)
{
    __shared__ uint32_t h[256];
    for (int i = threadIdx.x; i < 256; i += kThreads) h[i] = 0;
    __syncthreads();
    const size_t base = (size_t)blockIdx.x * kTile;
    const uint32_t mask = (1u << bits) - 1u;
#pragma unroll
    for (int k = 0; k < kItems; ++k)
    {
        size_t i = base + (size_t)k * kThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & mask], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += kThreads) counts[(size_t)d * tiles + blockIdx.x] = h[d];
}

// Exclusive scan of each digit's row of the [digit][tile] count table, one
// block per digit (tiles is n / 4096, so a row is short), and the digit's
// total.  The digits' own offsets (an exclusive scan of the 256 totals) are
// added by every scatter block, so no single-block pass over the whole table
// is needed.
constexpr int kScanThreads = 256;
__global__ void __launch_bounds__(kScanThreads) digit_scan_kernel(uint32_t* __restrict__ counts, int tiles,
                                                                  uint32_t* __restrict__ digit_total)
{
    __shared__ uint32_t warp_sums[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t* row = counts + (size_t)blockIdx.x * tiles;
    const int per = (tiles + kScanThreads - 1) / kScanThreads;  // consecutive entries per thread
    const int first = threadIdx.x * per;
    uint32_t sum = 0;
    for (int k = 0; k < per; ++k)
        if (first + k < tiles) sum += row[first + k];
    uint32_t x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    uint32_t before = 0;
    for (int w = 0; w < warp; ++w) before += warp_sums[w];
    uint32_t run = before + x - sum;
    for (int k = 0; k < per; ++k)
        if (first + k < tiles)
        {
            const uint32_t v = row[first + k];
            row[first + k] = run;
            run += v;
        }
    if (threadIdx.x == kScanThreads - 1) digit_total[blockIdx.x] = run;
}

__global__ void __launch_bounds__(kThreads) scatter_kernel(const uint32_t* __restrict__ keys_in,
                                                           const uint32_t* __restrict__ vals_in,
                                                           uint32_t* __restrict__ keys_out,
                                                           uint32_t* __restrict__ vals_out, size_t n, int shift,
                                                           int bits, const uint32_t* __restrict__ offsets, int tiles,
                                                           const uint32_t* __restrict__ digit_total)
{
    __shared__ uint32_t digit_base[256];         // running position inside this tile
    __shared__ uint32_t global_base[256];
    __shared__ uint32_t warp_cnt[kWarps][256];   // per-round counts, then exclusive prefix across warps
    __shared__ uint32_t round_total[256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t mask = (1u << bits) - 1u;
    // Digit offsets: exclusive scan of the 256 digit totals (one per thread).
    static_assert(kThreads == 256, "one digit per thread");
    {
        const uint32_t t = digit_total[threadIdx.x];
        uint32_t x = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) round_total[warp] = x;
        __syncthreads();
        uint32_t before = 0;
        for (int w = 0; w < warp; ++w) before += round_total[w];
        digit_base[threadIdx.x] = 0;
        global_base[threadIdx.x] = before + x - t + offsets[(size_t)threadIdx.x * tiles + blockIdx.x];
        __syncthreads();
    }
    const size_t base = (size_t)blockIdx.x * kTile;
    const uint32_t lt_mask = (1u << lane) - 1u;
    for (int k = 0; k < kItems; ++k)
    {
        for (int d = threadIdx.x; d < 256 * kWarps; d += kThreads) (&warp_cnt[0][0])[d] = 0;
        __syncthreads();
        const size_t i = base + (size_t)k * kThreads + threadIdx.x;
        const bool valid = i < n;
        uint32_t key = valid ? keys_in[i] : 0u;
        uint32_t val = valid ? vals_in[i] : 0u;
        // Invalid lanes get digit 256 so they never match a real digit.
        uint32_t digit = valid ? ((key >> shift) & mask) : 256u;
        uint32_t peers = __match_any_sync(0xffffffffu, digit);
        uint32_t rank_in_warp = __popc(peers & lt_mask);
        if (valid && rank_in_warp == 0) warp_cnt[warp][digit] = __popc(peers);
        __syncthreads();
        // Exclusive prefix across warps, one digit per thread.
        for (int d = threadIdx.x; d < 256; d += kThreads)
        {
            uint32_t run = 0;
#pragma unroll
            for (int w = 0; w < kWarps; ++w)
            {
                uint32_t c = warp_cnt[w][d];
                warp_cnt[w][d] = run;
                run += c;
            }
            round_total[d] = run;
        }
        __syncthreads();
        if (valid)
        {
            uint32_t pos = global_base[digit] + digit_base[digit] + warp_cnt[warp][digit] + rank_in_warp;
            keys_out[pos] = key;
            vals_out[pos] = val;
        }
        __syncthreads();
        for (int d = threadIdx.x; d < 256; d += kThreads) digit_base[d] += round_total[d];
        __syncthreads();
    }
}
}  // namespace

size_t radix_sort_scratch_bytes(size_t n)
{
    size_t t = tiles_for(n ? n : 1);
    return align256(n * 4) * 2 + align256(256 * t * 4) + 256 * 4 + 256;
}

RadixSortScratch radix_sort_bind(void* base, size_t n)
{
    char* p = (char*)(((uintptr_t)base + 255) & ~(uintptr_t)255);
    RadixSortScratch s;
    s.keys_alt = (uint32_t*)p;
    p += align256(n * 4);
    s.vals_alt = (uint32_t*)p;
    p += align256(n * 4);
    s.counts = (uint32_t*)p;
    p += align256(256 * tiles_for(n ? n : 1) * 4);
    s.digit_total = (uint32_t*)p;
    s.capacity = n;
    return s;
}

cudaError_t radix_sort_pairs(uint32_t* keys, uint32_t* vals, size_t n, int begin_bit, int end_bit,
                             const RadixSortScratch& s, cudaStream_t stream)
{
    if (n <= 1 || end_bit <= begin_bit) return cudaSuccess;
    const int tiles = (int)tiles_for(n);
    uint32_t *ki = keys, *vi = vals, *ko = s.keys_alt, *vo = s.vals_alt;
    for (int shift = begin_bit; shift < end_bit; shift += 8)
    {
        const int bits = (end_bit - shift) < 8 ? (end_bit - shift) : 8;
        hist_kernel<<<tiles, kThreads, 0, stream>>>(ki, n, shift, bits, s.counts, tiles);
        digit_scan_kernel<<<256, kScanThreads, 0, stream>>>(s.counts, tiles, s.digit_total);
        scatter_kernel<<<tiles, kThreads, 0, stream>>>(ki, vi, ko, vo, n, shift, bits, s.counts, tiles,
                                                       s.digit_total);
        uint32_t* t = ki; ki = ko; ko = t;
        t = vi; vi = vo; vo = t;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (ki != keys)
    {
        e = cudaMemcpyAsync(keys, ki, n * 4, cudaMemcpyDeviceToDevice, stream);
        if (e != cudaSuccess) return e;
        e = cudaMemcpyAsync(vals, vi, n * 4, cudaMemcpyDeviceToDevice, stream);
    }
    return e;
}
}  // namespace lg
