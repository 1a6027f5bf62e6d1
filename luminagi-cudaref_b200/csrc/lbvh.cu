// lbvh.cu -- on-device LBVH build, node-for-node identical to the reference's
// CPU build (LuminaGI-CudaRef src/bvh.cpp:164-211).
//
// Why a radix tree reproduces the reference.  build_recursive (bvh.cpp:75-120)
// splits a range of Morton-sorted triangles at the highest bit in which the
// range's codes differ (find_split is a binary search for that bit), stops at
// <= 4 triangles or when all codes in the range are equal, and numbers the
// nodes breadth-first afterwards (relayout_bfs, bvh.cpp:122-162).  The binary
// radix tree over the sorted codes, with duplicate codes made distinct by
// their sorted position (Karras 2012), contains every one of those ranges as
// a node, split the same way.  The reference tree is that radix tree cut off
// below every node whose range has <= 4 triangles or one distinct code:
//   kept(node)      = node is the root, or its parent is not collapsed
//   collapsed(node) = size <= 4 or code[first] == code[last]
// Breadth-first order with left before right is the order of (depth, first
// triangle), so the BFS index is the rank of that key.  Bounding boxes are
// refitted bottom-up; a leaf box scans its triangles in order and a parent
// box starts from the left child and widens by the right child, with the
// reference's strict < / > updates, so the float bits (signed zeros
// included) are the reference's.
//
// Kernels: scene bounds (order-aware min/max), Morton codes (IEEE-exact
// ops), radix sort, Karras hierarchy, keep/depth keys, BFS sort, node write +
// refit, triangle gather.
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "common.h"
#include "lbvh.cuh"
#include "radix_sort.cuh"

namespace lg
{
namespace
{
constexpr int kTB = 256;

constexpr int kFirstBits = 26;    // up to 2^26 triangles

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
inline int blocks_for(size_t n, int tb = kTB) { return (int)((n + tb - 1) / tb); }

// Total order key for "first occurrence of the minimum": value (with -0 and
// +0 equal, NaN excluded) in the high word, position in the low word.
__device__ __forceinline__ uint64_t min_key(float f, uint32_t pos)
{
    if (f != f) return ~0ull;  // NaN never wins
    uint32_t u = __float_as_uint(f == 0.0f ? 0.0f : f);
    u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return ((uint64_t)u << 32) | pos;
}
// For the maximum, larger value wins and, among equal values, the smaller position.
__device__ __forceinline__ uint64_t max_key(float f, uint32_t pos)
{
    if (f != f) return 0ull;
    uint32_t u = __float_as_uint(f == 0.0f ? 0.0f : f);
    u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return ((uint64_t)u << 32) | (0xFFFFFFFFu - pos);
}

__device__ __forceinline__ uint64_t warp_min_u64(uint64_t v)
{
    for (int o = 16; o; o >>= 1)
    {
        uint64_t w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}
__device__ __forceinline__ uint64_t warp_max_u64(uint64_t v)
{
    for (int o = 16; o; o >>= 1)
    {
        uint64_t w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// bvh.cpp:170-173 -- scene box over every vertex in input order.
// out[0..2] = min keys (init ~0), out[3..5] = max keys (init 0).
__global__ void __launch_bounds__(kTB) bounds_kernel(const lg_triangle* __restrict__ tris, int n,
                                                     unsigned long long* out)
{
    uint64_t mn[3] = {~0ull, ~0ull, ~0ull}, mx[3] = {0, 0, 0};
    for (int t = blockIdx.x * kTB + threadIdx.x; t < n; t += gridDim.x * kTB)
    {
        const lg_triangle& tr = tris[t];
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            const uint32_t pos = (uint32_t)t * 3u + (uint32_t)k;
#pragma unroll
            for (int a = 0; a < 3; ++a)
            {
                const float f = tr.v[k][a];
                uint64_t a0 = min_key(f, pos), a1 = max_key(f, pos);
                mn[a] = a0 < mn[a] ? a0 : mn[a];
                mx[a] = a1 > mx[a] ? a1 : mx[a];
            }
        }
    }
    __shared__ uint64_t s[6][kTB / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        uint64_t x = warp_min_u64(mn[a]);
        uint64_t y = warp_max_u64(mx[a]);
        if (lane == 0) { s[a][warp] = x; s[3 + a][warp] = y; }
    }
    __syncthreads();
    if (threadIdx.x < 6)
    {
        const int a = threadIdx.x;
        uint64_t v = s[a][0];
        for (int w = 1; w < kTB / 32; ++w) v = a < 3 ? (s[a][w] < v ? s[a][w] : v) : (s[a][w] > v ? s[a][w] : v);
        if (a < 3) atomicMin(&out[a], (unsigned long long)v);
        else atomicMax(&out[a], (unsigned long long)v);
    }
}

// Turns the winning keys back into the vertex values and the normalisation
// extent (bvh.cpp:176-178: ext <= 0 -> 1).  box[0..2] = min, box[3..5] = ext.
__global__ void bounds_finish_kernel(const lg_triangle* __restrict__ tris, const unsigned long long* keys,
                                     float* box)
{
    if (threadIdx.x != 0) return;
    float mn[3], mx[3];
    for (int a = 0; a < 3; ++a)
    {
        uint64_t k = keys[a];
        if (k == ~0ull) mn[a] = __int_as_float(0x7f800000);
        else
        {
            uint32_t pos = (uint32_t)(k & 0xFFFFFFFFu);
            mn[a] = tris[pos / 3].v[pos % 3][a];
        }
        uint64_t m = keys[3 + a];
        if (m == 0ull) mx[a] = __int_as_float(0xff800000);
        else
        {
            uint32_t pos = 0xFFFFFFFFu - (uint32_t)(m & 0xFFFFFFFFu);
            mx[a] = tris[pos / 3].v[pos % 3][a];
        }
    }
    for (int a = 0; a < 3; ++a)
    {
        float e = __fsub_rn(mx[a], mn[a]);
        if (e <= 0.0f) e = 1.0f;
        box[a] = mn[a];
        box[3 + a] = e;
    }
}

__device__ __forceinline__ uint32_t spread3(uint32_t v)
{
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
// bvh.cpp:23-32 quantiser: clamp(f * 1024, 0, 1023) then truncate.
__device__ __forceinline__ uint32_t quant10(float f)
{
    f = __fmul_rn(f, 1024.0f);
    if (f < 0.0f) f = 0.0f;
    if (f > 1023.0f) f = 1023.0f;
    return __float2uint_rz(f);
}

// bvh.cpp:185-191 with every operation rounded individually (no FMA).
__global__ void __launch_bounds__(kTB) morton_kernel(const lg_triangle* __restrict__ tris, int n,
                                                     const float* __restrict__ box, uint32_t* __restrict__ codes,
                                                     uint32_t* __restrict__ idx)
{
    const int t = blockIdx.x * kTB + threadIdx.x;
    if (t >= n) return;
    const lg_triangle& tr = tris[t];
    const float third = 1.0f / 3.0f;
    uint32_t q[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        float c = __fmul_rn(__fadd_rn(__fadd_rn(tr.v[0][a], tr.v[1][a]), tr.v[2][a]), third);
        q[a] = quant10(__fdiv_rn(__fsub_rn(c, box[a]), box[3 + a]));
    }
    codes[t] = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
    idx[t] = (uint32_t)t;
}

// Common-prefix length of sorted keys i and j, duplicates separated by index.
__device__ __forceinline__ int delta(const uint32_t* __restrict__ codes, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    uint32_t a = codes[i], b = codes[j];
    if (a == b) return 32 + __clz((uint32_t)(i ^ j));
    return __clz(a ^ b);
}

// Karras 2012, Algorithm 2.  Node ids: internal 0..n-2, leaf k -> n-1+k.
__global__ void __launch_bounds__(kTB) karras_kernel(const uint32_t* __restrict__ codes, int n,
                                                     int* __restrict__ first, int* __restrict__ last,
                                                     int* __restrict__ childL, int* __restrict__ childR,
                                                     int* __restrict__ parent)
{
    const int i = blockIdx.x * kTB + threadIdx.x;
    if (i >= n - 1) return;
    const int d = (delta(codes, n, i, i + 1) - delta(codes, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = delta(codes, n, i, i - d);
    int lmax = 2;
    while (delta(codes, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(codes, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = delta(codes, n, i, j);
    int s = 0;
    int t = l;
    do
    {
        t = (t + 1) >> 1;
        if (delta(codes, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int gamma = i + s * d + (d < 0 ? -1 : 0);
    const int lo = i < j ? i : j, hi = i < j ? j : i;
    const int left = (lo == gamma) ? (n - 1 + gamma) : gamma;
    const int right = (hi == gamma + 1) ? (n - 1 + gamma + 1) : gamma + 1;
    first[i] = lo;
    last[i] = hi;
    childL[i] = left;
    childR[i] = right;
    parent[left] = i;
    parent[right] = i;
    if (i == 0) parent[0] = -1;
}

__device__ __forceinline__ bool collapsed(const uint32_t* __restrict__ codes, const int* __restrict__ first,
                                          const int* __restrict__ last, int n, int u)
{
    if (u >= n - 1) return true;  // single-triangle radix leaf
    const int f = first[u], l = last[u];
    return (l - f + 1) <= 4 || codes[f] == codes[l];
}

// Key = (depth << 26) | first for kept nodes, 0xFFFFFFFF for the rest.
__global__ void __launch_bounds__(kTB) keep_kernel(const uint32_t* __restrict__ codes, int n,
                                                   const int* __restrict__ first, const int* __restrict__ last,
                                                   const int* __restrict__ parent, uint32_t* __restrict__ keys,
                                                   uint32_t* __restrict__ ids, int* __restrict__ kept_count)
{
    const int u = blockIdx.x * kTB + threadIdx.x;
    const int total = 2 * n - 1;
    if (u >= total) return;
    bool kept;
    int f;
    if (u == 0) { kept = true; f = 0; }
    else
    {
        const int p = parent[u];
        kept = !collapsed(codes, first, last, n, p);
        f = (u >= n - 1) ? (u - (n - 1)) : first[u];
    }
    uint32_t key = 0xFFFFFFFFu;
    if (kept)
    {
        int depth = 0;
        for (int a = u; a != 0; a = parent[a]) ++depth;
        key = ((uint32_t)depth << kFirstBits) | (uint32_t)f;
        atomicAdd(kept_count, 1);
    }
    keys[u] = key;
    ids[u] = (uint32_t)u;
}

__global__ void __launch_bounds__(kTB) bfs_index_kernel(const uint32_t* __restrict__ sorted_ids,
                                                        const int* __restrict__ kept_count, int* __restrict__ bfs_of)
{
    const int p = blockIdx.x * kTB + threadIdx.x;
    if (p >= *kept_count) return;
    bfs_of[sorted_ids[p]] = p;
}

__device__ __forceinline__ void fit_vertex(float mn[3], float mx[3], const float* v)
{
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        if (v[a] < mn[a]) mn[a] = v[a];
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        if (v[a] > mx[a]) mx[a] = v[a];
    }
}

// Writes every kept node's topology, then refits boxes bottom-up from the
// leaves: the second child to arrive at a parent computes its box.
__global__ void __launch_bounds__(kTB) nodes_kernel(const uint32_t* __restrict__ codes, int n,
                                                    const int* __restrict__ first, const int* __restrict__ last,
                                                    const int* __restrict__ childL, const int* __restrict__ childR,
                                                    const int* __restrict__ parent, const int* __restrict__ bfs_of,
                                                    const uint32_t* __restrict__ sorted_ids,
                                                    const int* __restrict__ kept_count,
                                                    const lg_triangle* __restrict__ tris_sorted,
                                                    lg_bvh_node* nodes, int* arrivals)
{
    const int p = blockIdx.x * kTB + threadIdx.x;
    if (p >= *kept_count) return;
    const int u = (int)sorted_ids[p];
    const bool leaf = collapsed(codes, first, last, n, u);
    lg_bvh_node* out = &nodes[p];
    if (!leaf)
    {
        out->left = bfs_of[childL[u]];
        out->right = bfs_of[childR[u]];
        out->firstTri = -1;
        out->triCount = 0;
        return;
    }
    const int f = (u >= n - 1) ? (u - (n - 1)) : first[u];
    const int l = (u >= n - 1) ? f : last[u];
    float mn[3] = {__int_as_float(0x7f800000), __int_as_float(0x7f800000), __int_as_float(0x7f800000)};
    float mx[3] = {__int_as_float(0xff800000), __int_as_float(0xff800000), __int_as_float(0xff800000)};
    for (int t = f; t <= l; ++t)
        for (int k = 0; k < 3; ++k) fit_vertex(mn, mx, tris_sorted[t].v[k]);
    out->left = -1;
    out->right = -1;
    out->firstTri = f;
    out->triCount = l - f + 1;
    for (int a = 0; a < 3; ++a) { out->bbMin[a] = mn[a]; out->bbMax[a] = mx[a]; }
    // Walk up; the second arrival at each parent refits it.
    int v = u;
    while (v != 0)
    {
        __threadfence();
        const int par = parent[v];
        if (atomicAdd(&arrivals[par], 1) == 0) return;
        __threadfence();
        const volatile lg_bvh_node* L = &nodes[bfs_of[childL[par]]];
        const volatile lg_bvh_node* R = &nodes[bfs_of[childR[par]]];
        float bmn[3], bmx[3];
        for (int a = 0; a < 3; ++a) { bmn[a] = L->bbMin[a]; bmx[a] = L->bbMax[a]; }
        for (int a = 0; a < 3; ++a)
            if (R->bbMin[a] < bmn[a]) bmn[a] = R->bbMin[a];
        for (int a = 0; a < 3; ++a)
            if (R->bbMax[a] > bmx[a]) bmx[a] = R->bbMax[a];
        volatile lg_bvh_node* P = &nodes[bfs_of[par]];
        for (int a = 0; a < 3; ++a) { P->bbMin[a] = bmn[a]; P->bbMax[a] = bmx[a]; }
        v = par;
    }
}

__global__ void __launch_bounds__(kTB) gather_kernel(const lg_triangle* __restrict__ in,
                                                     const uint32_t* __restrict__ perm, int n,
                                                     lg_triangle* __restrict__ out, int32_t* __restrict__ perm_out)
{
    // One warp copies one 100-byte triangle as 25 words.
    const int gw = (blockIdx.x * kTB + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= n) return;
    const uint32_t src = perm[gw];
    const uint32_t* s = reinterpret_cast<const uint32_t*>(in + src);
    uint32_t* d = reinterpret_cast<uint32_t*>(out + gw);
    if (lane < 25) d[lane] = s[lane];
    if (lane == 0 && perm_out) perm_out[gw] = (int32_t)src;
}

// Single-triangle scene: one leaf (bvh.cpp:92-104 with count 1).
__global__ void single_leaf_kernel(const lg_triangle* __restrict__ tris, lg_bvh_node* nodes)
{
    float mn[3] = {__int_as_float(0x7f800000), __int_as_float(0x7f800000), __int_as_float(0x7f800000)};
    float mx[3] = {__int_as_float(0xff800000), __int_as_float(0xff800000), __int_as_float(0xff800000)};
    for (int k = 0; k < 3; ++k) fit_vertex(mn, mx, tris[0].v[k]);
    for (int a = 0; a < 3; ++a) { nodes[0].bbMin[a] = mn[a]; nodes[0].bbMax[a] = mx[a]; }
    nodes[0].left = -1;
    nodes[0].right = -1;
    nodes[0].firstTri = 0;
    nodes[0].triCount = 1;
}

struct Layout
{
    size_t bytes = 0;
    size_t off_bounds, off_box, off_codes, off_idx, off_sort1, off_first, off_last, off_cl, off_cr, off_parent,
        off_keys, off_ids, off_sort2, off_bfs, off_arr, off_count, off_tmp_tris;
};

Layout layout_for(size_t n, bool need_tmp_tris)
{
    Layout L;
    size_t at = 0;
    auto take = [&](size_t b) { size_t o = at; at += align256(b); return o; };
    const size_t total = 2 * n - 1;
    L.off_bounds = take(6 * sizeof(unsigned long long));
    L.off_box = take(6 * sizeof(float));
    L.off_codes = take(n * 4);
    L.off_idx = take(n * 4);
    L.off_sort1 = take(radix_sort_scratch_bytes(n));
    L.off_first = take(n * 4);
    L.off_last = take(n * 4);
    L.off_cl = take(n * 4);
    L.off_cr = take(n * 4);
    L.off_parent = take(total * 4);
    L.off_keys = take(total * 4);
    L.off_ids = take(total * 4);
    L.off_sort2 = take(radix_sort_scratch_bytes(total));
    L.off_bfs = take(total * 4);
    L.off_arr = take(n * 4);
    L.off_count = take(4);
    L.off_tmp_tris = need_tmp_tris ? take(n * sizeof(lg_triangle)) : 0;
    L.bytes = at + 256;
    return L;
}
}  // namespace

size_t lbvh_scratch_bytes(int n_tris, bool tris_in_scratch)
{
    if (n_tris <= 1) return 256;
    return layout_for((size_t)n_tris, tris_in_scratch).bytes;
}

int lbvh_build(const lg_triangle* d_tris, int n, lg_bvh_node* d_nodes, int* n_nodes_host, int32_t* d_perm_out,
               lg_triangle* d_tris_out, void* scratch, size_t scratch_bytes, cudaStream_t stream)
{
    if (n < 0) return set_error(LG_ERR_INVALID, "BuildBVH: negative triangle count");
    if (n > (1 << kFirstBits)) return set_error(LG_ERR_INVALID, "BuildBVH: %d triangles exceeds 2^26", n);
    if (n == 0) { *n_nodes_host = 0; return LG_OK; }
    if (n == 1)
    {
        single_leaf_kernel<<<1, 1, 0, stream>>>(d_tris, d_nodes);
        if (d_tris_out && d_tris_out != d_tris)
            LG_TRY_CUDA(cudaMemcpyAsync(d_tris_out, d_tris, sizeof(lg_triangle), cudaMemcpyDeviceToDevice, stream));
        if (d_perm_out) LG_TRY_CUDA(cudaMemsetAsync(d_perm_out, 0, sizeof(int32_t), stream));
        LG_TRY_CUDA(cudaGetLastError());
        LG_TRY_CUDA(cudaStreamSynchronize(stream));
        *n_nodes_host = 1;
        return LG_OK;
    }
    // The leaf boxes read the triangles in sorted order; they are gathered into
    // scratch when the caller wants them in place or not at all.
    const bool need_tmp = d_tris_out == nullptr || d_tris_out == d_tris;
    const Layout L = layout_for((size_t)n, need_tmp);
    if (scratch_bytes < L.bytes) return set_error(LG_ERR_CAPACITY, "BuildBVH: scratch too small");
    char* base = (char*)(((uintptr_t)scratch + 255) & ~(uintptr_t)255);
    auto at = [&](size_t off) { return (void*)(base + off); };
    unsigned long long* bounds = (unsigned long long*)at(L.off_bounds);
    float* box = (float*)at(L.off_box);
    uint32_t* codes = (uint32_t*)at(L.off_codes);
    uint32_t* idx = (uint32_t*)at(L.off_idx);
    int* first = (int*)at(L.off_first);
    int* last = (int*)at(L.off_last);
    int* cl = (int*)at(L.off_cl);
    int* cr = (int*)at(L.off_cr);
    int* parent = (int*)at(L.off_parent);
    uint32_t* keys = (uint32_t*)at(L.off_keys);
    uint32_t* ids = (uint32_t*)at(L.off_ids);
    int* bfs_of = (int*)at(L.off_bfs);
    int* arrivals = (int*)at(L.off_arr);
    int* kept = (int*)at(L.off_count);
    const int total = 2 * n - 1;

    // 1. scene bounds
    unsigned long long init[6] = {~0ull, ~0ull, ~0ull, 0ull, 0ull, 0ull};
    LG_TRY_CUDA(cudaMemcpyAsync(bounds, init, sizeof init, cudaMemcpyHostToDevice, stream));
    int bgrid = blocks_for((size_t)n);
    if (bgrid > 148 * 8) bgrid = 148 * 8;
    bounds_kernel<<<bgrid, kTB, 0, stream>>>(d_tris, n, bounds);
    bounds_finish_kernel<<<1, 32, 0, stream>>>(d_tris, bounds, box);
    // 2. Morton codes + 3. sort (30-bit codes, stable: ties stay in input order)
    morton_kernel<<<blocks_for((size_t)n), kTB, 0, stream>>>(d_tris, n, box, codes, idx);
    LG_TRY_CUDA(radix_sort_pairs(codes, idx, (size_t)n, 0, 30, radix_sort_bind(at(L.off_sort1), (size_t)n), stream));
    // 4. radix tree
    karras_kernel<<<blocks_for((size_t)n - 1), kTB, 0, stream>>>(codes, n, first, last, cl, cr, parent);
    // 5. kept nodes keyed by (depth, first); 6. BFS order by sorting the keys
    LG_TRY_CUDA(cudaMemsetAsync(kept, 0, sizeof(int), stream));
    keep_kernel<<<blocks_for((size_t)total), kTB, 0, stream>>>(codes, n, first, last, parent, keys, ids, kept);
    LG_TRY_CUDA(radix_sort_pairs(keys, ids, (size_t)total, 0, 32, radix_sort_bind(at(L.off_sort2), (size_t)total),
                                 stream));
    bfs_index_kernel<<<blocks_for((size_t)total), kTB, 0, stream>>>(ids, kept, bfs_of);
    // 7. triangles in sorted order (needed by the leaf boxes)
    lg_triangle* tris_sorted = need_tmp ? (lg_triangle*)at(L.off_tmp_tris) : d_tris_out;
    gather_kernel<<<blocks_for((size_t)n * 32), kTB, 0, stream>>>(d_tris, idx, n, tris_sorted, d_perm_out);
    // 8. node records + bottom-up refit
    LG_TRY_CUDA(cudaMemsetAsync(arrivals, 0, (size_t)n * sizeof(int), stream));
    nodes_kernel<<<blocks_for((size_t)total), kTB, 0, stream>>>(codes, n, first, last, cl, cr, parent, bfs_of, ids,
                                                               kept, tris_sorted, d_nodes, arrivals);
    if (d_tris_out && need_tmp)
        LG_TRY_CUDA(cudaMemcpyAsync(d_tris_out, tris_sorted, (size_t)n * sizeof(lg_triangle),
                                    cudaMemcpyDeviceToDevice, stream));
    LG_TRY_CUDA(cudaGetLastError());
    int count = 0;
    LG_TRY_CUDA(cudaMemcpyAsync(&count, kept, sizeof(int), cudaMemcpyDeviceToHost, stream));
    LG_TRY_CUDA(cudaStreamSynchronize(stream));
    *n_nodes_host = count;
    return LG_OK;
}
}  // namespace lg
