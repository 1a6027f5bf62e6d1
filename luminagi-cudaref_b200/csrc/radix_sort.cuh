// radix_sort.cuh -- stable LSD radix sort of (u32 key, u32 value) pairs.
//
// One pass per 8-bit digit, three launches per pass:
//   1. per-tile digit histogram (tile = 256 threads x kItems keys),
//   2. exclusive scan of each digit's row of the [digit][tile] count table
//      (one block per digit) and the digit totals,
//   3. stable scatter: each block scans the 256 digit totals for the digit
//      offsets; keys of a tile are ranked in input order (warp match_any
//      peers + per-warp digit counts), then written to digit offset +
//      row prefix[digit][tile] + rank.
// Stability makes the result a total order on (key, input position), which
// is what the BVH build relies on for a deterministic triangle order.
#pragma once
#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace lg
{
struct RadixSortScratch
{
    uint32_t* keys_alt = nullptr;
    uint32_t* vals_alt = nullptr;
    uint32_t* counts = nullptr;  // 256 * tiles
    uint32_t* digit_total = nullptr;  // 256
    size_t capacity = 0;         // elements
};

// Bytes of scratch needed for n elements.
size_t radix_sort_scratch_bytes(size_t n);
// Carves the scratch pointers out of `base` (aligned to 256 bytes).
RadixSortScratch radix_sort_bind(void* base, size_t n);

// Sorts keys/vals in place over bits [begin_bit, end_bit).  Returns a CUDA error.
cudaError_t radix_sort_pairs(uint32_t* keys, uint32_t* vals, size_t n, int begin_bit, int end_bit,
                             const RadixSortScratch& s, cudaStream_t stream);
}  // namespace lg
