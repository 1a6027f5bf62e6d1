// render_tree.cu -- the binary tree the traversal records are built from.
//
// BuildBVH's tree (bit-exact to the reference) is what lg_build_bvh returns
// and what the G-buffer box comes from.  Rays do not need that exact tree:
// any binary tree over the same leaves gives the same closest hits (up to
// exact ties in t).  Two render trees are built here, both in depth order
// (every depth a contiguous range, the root first), which the 4-wide
// collapse relies on:
//   * mode 0: the input tree itself, stably re-sorted by depth (a tree the
//     caller supplies need not be in breadth-first order);
//   * mode 1: the input tree's leaves, regrouped by PLOC -- "Parallel
//     Locally-Ordered Clustering for BVH Construction" (Meister and Bittner,
//     HPG 2018).  Clusters start as the leaves in Morton order (their first
//     triangles); each round, every cluster finds the neighbour within +-R
//     positions whose union box has the smallest surface area, mutual
//     nearest neighbours merge into a new node, and the survivors are
//     compacted in order.  The Morton tree splits at code bits; PLOC groups
//     by actual box sizes, so traversal opens fewer boxes.
//   * mode 2: PLOC over the triangles themselves (in their Morton order),
//     one triangle per leaf: 2T - 1 nodes.  Leaves index the same triangle
//     array, so nothing is reordered; any BVH over the triangles finds the
//     same closest hits (up to exact ties in t).
// Ties in the neighbour search go to the lower position and every numbering
// comes from prefix sums, so both trees are deterministic.
#include <algorithm>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "bvh.h"
#include "common.h"
#include "radix_sort.cuh"
#include "render_tree.cuh"

namespace lg
{
namespace
{
constexpr int kTB = 256;
constexpr int kRadius = 8;  // PLOC search radius (positions on either side); 8 measured 1% faster to trace than 16 or 32

size_t a256(size_t b) { return (b + 255) & ~(size_t)255; }

// ---- exclusive scan of int flags/counts (block sums + one-block scan + add) ----
__device__ __forceinline__ int block_excl_scan(int v, int* warp_sums, int& total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    int before = 0;
    total = 0;
    for (int w = 0; w < kTB / 32; ++w)
    {
        if (w < warp) before += warp_sums[w];
        total += warp_sums[w];
    }
    __syncthreads();
    return before + x - v;
}
__global__ void scan_local_kernel(const int* __restrict__ in, int n, int* __restrict__ out, int* __restrict__ sums)
{
    __shared__ int ws[kTB / 32];
    const int i = blockIdx.x * kTB + threadIdx.x;
    int total;
    const int e = block_excl_scan(i < n ? in[i] : 0, ws, total);
    if (i < n) out[i] = e;
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}
__global__ void scan_sums_kernel(int* __restrict__ sums, int nb, int* __restrict__ grand_total)
{
    __shared__ int ws[kTB / 32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b = 0; b < nb; b += kTB)
    {
        const int i = b + threadIdx.x;
        int total;
        const int e = block_excl_scan(i < nb ? sums[i] : 0, ws, total);
        if (i < nb) sums[i] = carry + e;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0 && grand_total) *grand_total = carry;
}
__global__ void scan_add_kernel(int* __restrict__ out, int n, const int* __restrict__ sums)
{
    const int i = blockIdx.x * kTB + threadIdx.x;
    if (i < n) out[i] += sums[blockIdx.x];
}
// out = exclusive scan of in (in == out allowed); *total (device) = sum.
cudaError_t excl_scan(const int* in, int n, int* out, int* sums, int* total, cudaStream_t st)
{
    const int nb = (n + kTB - 1) / kTB;
    if (n <= 0) return cudaMemsetAsync(total, 0, sizeof(int), st);
    scan_local_kernel<<<nb, kTB, 0, st>>>(in, n, out, sums);
    scan_sums_kernel<<<1, kTB, 0, st>>>(sums, nb, total);
    scan_add_kernel<<<nb, kTB, 0, st>>>(out, n, sums);
    return cudaGetLastError();
}
// ---- depth order ----
__global__ void parent_of_kernel(const lg_bvh_node* __restrict__ nodes, int n, int* __restrict__ parent)
{
    const int i = blockIdx.x * kTB + threadIdx.x;
    if (i >= n) return;
    const lg_bvh_node nd = nodes[i];
    if (nd.triCount == 0)
    {
        parent[nd.left] = i;
        parent[nd.right] = i;
    }
}
__global__ void depth_of_kernel(int n, int root, const int* __restrict__ parent, uint32_t* __restrict__ depth,
                                uint32_t* __restrict__ ids)
{
    const int i = blockIdx.x * kTB + threadIdx.x;
    if (i >= n) return;
    uint32_t d = 0;
    // nodes no link reaches (possible in a caller's array) stop at parent -1
    for (int a = i; a != root && a >= 0 && a < n && d < 255u; a = parent[a]) ++d;
    depth[i] = d;
    ids[i] = (uint32_t)i;
}
__global__ void rank_kernel(const uint32_t* __restrict__ order, int n, int* __restrict__ newpos)
{
    const int r = blockIdx.x * kTB + threadIdx.x;
    if (r < n) newpos[order[r]] = r;
}
__global__ void emit_kernel(const lg_bvh_node* __restrict__ in, const uint32_t* __restrict__ order,
                            const int* __restrict__ newpos, int n, lg_bvh_node* __restrict__ out)
{
    const int r = blockIdx.x * kTB + threadIdx.x;
    if (r >= n) return;
    lg_bvh_node nd = in[order[r]];
    if (nd.triCount == 0)
    {
        nd.left = newpos[nd.left];
        nd.right = newpos[nd.right];
    }
    out[r] = nd;
}

// ---- PLOC ----
struct Box
{
    float4 lo, hi;  // w unused
};
__device__ __forceinline__ float half_area(const Box& b)
{
    const float dx = b.hi.x - b.lo.x, dy = b.hi.y - b.lo.y, dz = b.hi.z - b.lo.z;
    return dx * dy + dy * dz + dz * dx;
}
__device__ __forceinline__ Box join(const Box& a, const Box& b)
{
    Box c;
    c.lo = make_float4(fminf(a.lo.x, b.lo.x), fminf(a.lo.y, b.lo.y), fminf(a.lo.z, b.lo.z), 0.0f);
    c.hi = make_float4(fmaxf(a.hi.x, b.hi.x), fmaxf(a.hi.y, b.hi.y), fmaxf(a.hi.z, b.hi.z), 0.0f);
    return c;
}

// Leaves by first triangle (= Morton order): leaf_at[t] = node whose range starts at t.
__global__ void leaf_at_kernel(const lg_bvh_node* __restrict__ nodes, int n, int* __restrict__ leaf_at,
                               int* __restrict__ flag)
{
    const int i = blockIdx.x * kTB + threadIdx.x;
    if (i >= n) return;
    const lg_bvh_node nd = nodes[i];
    if (nd.triCount > 0)
    {
        leaf_at[nd.firstTri] = i;
        flag[nd.firstTri] = 1;
    }
}
// Cluster k = leaf k in Morton order, node id k of the new tree.
__global__ void init_clusters_kernel(const lg_bvh_node* __restrict__ nodes, const int* __restrict__ leaf_at,
                                     const int* __restrict__ flag, const int* __restrict__ pos, int n_tris,
                                     lg_bvh_node* __restrict__ tn, int* __restrict__ cid, Box* __restrict__ cbox)
{
    const int t = blockIdx.x * kTB + threadIdx.x;
    if (t >= n_tris || !flag[t]) return;
    const int k = pos[t];
    const lg_bvh_node nd = nodes[leaf_at[t]];
    tn[k] = nd;
    cid[k] = k;
    Box b;
    b.lo = make_float4(nd.bbMin[0], nd.bbMin[1], nd.bbMin[2], 0.0f);
    b.hi = make_float4(nd.bbMax[0], nd.bbMax[1], nd.bbMax[2], 0.0f);
    cbox[k] = b;
}
// Cluster t = triangle t (one-triangle leaf, node id t of the new tree).
__global__ void init_tri_clusters_kernel(const lg_triangle* __restrict__ tris, int n_tris,
                                         lg_bvh_node* __restrict__ tn, int* __restrict__ cid, Box* __restrict__ cbox)
{
    const int t = blockIdx.x * kTB + threadIdx.x;
    if (t >= n_tris) return;
    const lg_triangle tr = tris[t];
    lg_bvh_node nd;
    for (int a = 0; a < 3; ++a)
    {
        nd.bbMin[a] = fminf(fminf(tr.v[0][a], tr.v[1][a]), tr.v[2][a]);
        nd.bbMax[a] = fmaxf(fmaxf(tr.v[0][a], tr.v[1][a]), tr.v[2][a]);
    }
    nd.left = -1;
    nd.right = -1;
    nd.firstTri = t;
    nd.triCount = 1;
    tn[t] = nd;
    cid[t] = t;
    Box b;
    b.lo = make_float4(nd.bbMin[0], nd.bbMin[1], nd.bbMin[2], 0.0f);
    b.hi = make_float4(nd.bbMax[0], nd.bbMax[1], nd.bbMax[2], 0.0f);
    cbox[t] = b;
}
// Nearest neighbour within +-kRadius positions by union surface area; ties -> lower position.
// The clustering round's kernels read the cluster count c from device memory
// (the round loop checks it on the host only every few rounds).
__global__ void __launch_bounds__(kTB) nn_kernel(const Box* __restrict__ cbox, const int* __restrict__ dc,
                                                 int* __restrict__ nn)
{
    __shared__ Box sb[kTB + 2 * kRadius];
    const int c = *dc;
    const int base = blockIdx.x * kTB - kRadius;
    for (int j = threadIdx.x; j < kTB + 2 * kRadius; j += kTB)
    {
        const int g = base + j;
        if (g >= 0 && g < c) sb[j] = cbox[g];
    }
    __syncthreads();
    const int i = blockIdx.x * kTB + threadIdx.x;
    if (i >= c) return;
    const Box bi = sb[threadIdx.x + kRadius];
    float best = __int_as_float(0x7f800000);
    int bj = -1;
    const int lo = max(0, i - kRadius), hi = min(c - 1, i + kRadius);
    for (int j = lo; j <= hi; ++j)
    {
        if (j == i) continue;
        const float a = half_area(join(bi, sb[j - base]));
        if (a < best)
        {
            best = a;
            bj = j;
        }
    }
    nn[i] = bj;
}
// A clustering round in four launches: nn_kernel, round_flags_kernel (merge
// and keep flags and their block-local exclusive scans), round_sums_kernel
// (one block: the block offsets, and the next round's state), and
// round_apply_kernel (merge and compact).  State {c, next node id, error}
// is double-buffered, cur -> nxt, so no launch reads a value its round
// changes.  The integer scans give the same positions as the three-kernel
// scans, so the tree does not change.
__global__ void round_flags_kernel(const int* __restrict__ nn, const int* __restrict__ cur, int* __restrict__ mflag,
                                   int* __restrict__ kflag, int* __restrict__ midx, int* __restrict__ kpos,
                                   int* __restrict__ msums, int* __restrict__ ksums)
{
    __shared__ int ws[kTB / 32];
    const int c = cur[0];
    const int i = blockIdx.x * kTB + threadIdx.x;
    int m = 0, k = 0;
    if (i < c)
    {
        const int j = nn[i];
        const bool mutual = j >= 0 && nn[j] == i;
        m = (mutual && i < j) ? 1 : 0;  // i owns the merged node
        k = (mutual && i > j) ? 0 : 1;  // j's partner disappears
        mflag[i] = m;
        kflag[i] = k;
    }
    int tm, tk;
    const int em = block_excl_scan(m, ws, tm);
    const int ek = block_excl_scan(k, ws, tk);
    if (i < c)
    {
        midx[i] = em;
        kpos[i] = ek;
    }
    if (threadIdx.x == 0)
    {
        msums[blockIdx.x] = tm;
        ksums[blockIdx.x] = tk;
    }
}
__global__ void round_sums_kernel(int* __restrict__ msums, int* __restrict__ ksums, int nb, const int* __restrict__ cur,
                                  int* __restrict__ nxt)
{
    __shared__ int ws[kTB / 32];
    __shared__ int carry[2];
    if (threadIdx.x < 2) carry[threadIdx.x] = 0;
    __syncthreads();
    for (int b = 0; b < nb; b += kTB)
    {
        const int i = b + threadIdx.x;
        int tm, tk;
        const int em = block_excl_scan(i < nb ? msums[i] : 0, ws, tm);
        const int ek = block_excl_scan(i < nb ? ksums[i] : 0, ws, tk);
        if (i < nb)
        {
            msums[i] = carry[0] + em;
            ksums[i] = carry[1] + ek;
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            carry[0] += tm;
            carry[1] += tk;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        const int merges = carry[0];
        nxt[2] = cur[2] | ((cur[0] > 1 && merges == 0) ? 1 : 0);
        nxt[1] = cur[1] + merges;
        nxt[0] = carry[1];
    }
}
__global__ void round_apply_kernel(const int* __restrict__ nn, const int* __restrict__ cur,
                                   const int* __restrict__ mflag, const int* __restrict__ kflag,
                                   const int* __restrict__ midx, const int* __restrict__ kpos,
                                   const int* __restrict__ msums, const int* __restrict__ ksums, int* __restrict__ cid,
                                   Box* __restrict__ cbox, lg_bvh_node* __restrict__ tn, int* __restrict__ cid2,
                                   Box* __restrict__ cbox2)
{
    const int c = cur[0], node_base = cur[1];
    const int i = blockIdx.x * kTB + threadIdx.x;
    if (i >= c) return;
    int id = cid[i];
    Box b = cbox[i];
    if (mflag[i])
    {
        // merge with the mutual nearest neighbour j > i (j keeps nothing and writes nothing this round)
        const int j = nn[i];
        id = node_base + msums[blockIdx.x] + midx[i];
        const Box bj = cbox[j];
        b = join(b, bj);
        lg_bvh_node nd;
        nd.bbMin[0] = b.lo.x; nd.bbMin[1] = b.lo.y; nd.bbMin[2] = b.lo.z;
        nd.bbMax[0] = b.hi.x; nd.bbMax[1] = b.hi.y; nd.bbMax[2] = b.hi.z;
        nd.left = cid[i];
        nd.right = cid[j];
        nd.firstTri = -1;
        nd.triCount = 0;
        tn[id] = nd;
    }
    if (kflag[i])
    {
        const int pos = ksums[blockIdx.x] + kpos[i];
        cid2[pos] = id;
        cbox2[pos] = b;
    }
}

struct Scratch
{
    char* p;
    char* end;
    template <class T>
    T* take(size_t count)
    {
        T* r = (T*)p;
        p += a256(count * sizeof(T));
        return p <= end ? r : nullptr;
    }
};
}  // namespace

int render_tree_nodes(int n_nodes, int n_tris, int mode)
{
    return mode == 2 && n_tris > 0 ? 2 * n_tris - 1 : n_nodes;
}

size_t render_tree_scratch_bytes(int n_nodes, int n_tris)
{
    const size_t t = (size_t)(n_tris > 0 ? n_tris : 1);
    // the larger of the modes: BuildBVH's n_nodes, or 2T - 1 one-triangle-leaf nodes
    const size_t n = std::max((size_t)(n_nodes > 0 ? n_nodes : 1), 2 * t);
    const size_t L = std::max((n + 1) / 2, t);
    size_t b = 0;
    b += a256(n * sizeof(lg_bvh_node));         // tn
    b += 4 * a256(n * 4);                       // parent, depth, ids, newpos
    b += a256(radix_sort_scratch_bytes(n));
    b += 3 * a256(t * 4);                       // leaf_at, flag, pos
    b += 2 * (a256(L * 4) + a256(L * sizeof(Box)));  // cluster arrays (double buffered)
    b += 5 * a256(L * 4);                       // nn, mflag, midx, kflag, kpos
    b += a256(2 * (L / kTB + 2) * 4) + 256;     // block sums (merge and keep flags), totals
    return b + 1024;
}

int build_render_tree(const lg_bvh_node* d_nodes, int n_nodes, const lg_triangle* d_tris, int n_tris, int mode,
                      lg_bvh_node* d_out, void* scratch, size_t scratch_bytes, cudaStream_t st)
{
    if (n_nodes <= 0) return LG_OK;
    const int in_nodes = n_nodes;
    n_nodes = render_tree_nodes(n_nodes, n_tris, mode);
    Scratch s{(char*)(((uintptr_t)scratch + 255) & ~(uintptr_t)255), (char*)scratch + scratch_bytes};
    lg_bvh_node* tn = s.take<lg_bvh_node>((size_t)n_nodes);
    int* parent = s.take<int>((size_t)n_nodes);
    uint32_t* depth = s.take<uint32_t>((size_t)n_nodes);
    uint32_t* ids = s.take<uint32_t>((size_t)n_nodes);
    int* newpos = s.take<int>((size_t)n_nodes);
    char* sort_mem = s.take<char>(radix_sort_scratch_bytes((size_t)n_nodes));
    if (!tn || !parent || !depth || !ids || !newpos || !sort_mem)
        return set_error(LG_ERR_CAPACITY, "render tree: scratch too small");
    const lg_bvh_node* src = d_nodes;
    int root = 0;
    const int g = (n_nodes + kTB - 1) / kTB;

    if ((mode == 1 || mode == 2) && n_nodes > 1)
    {
        const int t = n_tris;
        int* leaf_at = s.take<int>((size_t)t);
        int* flag = s.take<int>((size_t)t);
        int* pos = s.take<int>((size_t)t);
        const int L = (n_nodes + 1) / 2;
        int* cid = s.take<int>((size_t)L);
        Box* cbox = s.take<Box>((size_t)L);
        int* cid2 = s.take<int>((size_t)L);
        Box* cbox2 = s.take<Box>((size_t)L);
        int* nn = s.take<int>((size_t)L);
        int* mflag = s.take<int>((size_t)L);
        int* midx = s.take<int>((size_t)L);
        int* kflag = s.take<int>((size_t)L);
        int* kpos = s.take<int>((size_t)L);
        int* sums = s.take<int>(2 * ((size_t)t / kTB + 2));
        int* totals = s.take<int>(64);
        if (!sums || !totals) return set_error(LG_ERR_CAPACITY, "render tree: scratch too small");
        int c = 0;
        if (mode == 2)
        {
            init_tri_clusters_kernel<<<(t + kTB - 1) / kTB, kTB, 0, st>>>(d_tris, t, tn, cid, cbox);
            LG_TRY_CUDA(cudaGetLastError());
            c = t;
        }
        else
        {
            LG_TRY_CUDA(cudaMemsetAsync(flag, 0, sizeof(int) * (size_t)t, st));
            leaf_at_kernel<<<(in_nodes + kTB - 1) / kTB, kTB, 0, st>>>(d_nodes, in_nodes, leaf_at, flag);
            LG_TRY_CUDA(excl_scan(flag, t, pos, sums, totals, st));
            init_clusters_kernel<<<(t + kTB - 1) / kTB, kTB, 0, st>>>(d_nodes, leaf_at, flag, pos, t, tn, cid, cbox);
            LG_TRY_CUDA(cudaGetLastError());
            LG_TRY_CUDA(cudaMemcpyAsync(&c, totals, sizeof(int), cudaMemcpyDeviceToHost, st));
            LG_TRY_CUDA(cudaStreamSynchronize(st));
            if (c != L) return set_error(LG_ERR_INVALID, "render tree: %d leaves by range start, %d expected", c, L);
        }
        // Rounds run kRoundsPerCheck at a time on a device-held count, grids sized by the last count read back (an
        // upper bound: rounds only merge); the host reads the state between groups.
        constexpr int kRoundsPerCheck = 8;
        int* sbuf[2] = {totals + 8, totals + 16};  // double-buffered state {c, next node id, error}
        int* ksums = sums + ((size_t)t / kTB + 2);  // the keep flags' block sums beside the merge flags'
        int cur = 0;
        int hstate[3] = {c, L, 0};
        LG_TRY_CUDA(cudaMemcpyAsync(sbuf[0], hstate, sizeof(hstate), cudaMemcpyHostToDevice, st));
        while (hstate[0] > 1)
        {
            const int gc = (hstate[0] + kTB - 1) / kTB;
            for (int k = 0; k < kRoundsPerCheck; ++k)
            {
                const int* sc = sbuf[cur];
                int* sn = sbuf[cur ^ 1];
                nn_kernel<<<gc, kTB, 0, st>>>(cbox, sc, nn);
                round_flags_kernel<<<gc, kTB, 0, st>>>(nn, sc, mflag, kflag, midx, kpos, sums, ksums);
                round_sums_kernel<<<1, kTB, 0, st>>>(sums, ksums, gc, sc, sn);
                round_apply_kernel<<<gc, kTB, 0, st>>>(nn, sc, mflag, kflag, midx, kpos, sums, ksums, cid, cbox, tn,
                                                       cid2, cbox2);
                LG_TRY_CUDA(cudaGetLastError());
                int* ti = cid; cid = cid2; cid2 = ti;
                Box* tb = cbox; cbox = cbox2; cbox2 = tb;
                cur ^= 1;
            }
            LG_TRY_CUDA(cudaMemcpyAsync(hstate, sbuf[cur], sizeof(hstate), cudaMemcpyDeviceToHost, st));
            LG_TRY_CUDA(cudaStreamSynchronize(st));
            if (hstate[2]) return set_error(LG_ERR_DEVICE, "render tree: a clustering round merged nothing");
        }
        const int next_id = hstate[1];
        if (next_id != n_nodes) return set_error(LG_ERR_DEVICE, "render tree: %d nodes, %d expected", next_id, n_nodes);
        LG_TRY_CUDA(cudaMemcpyAsync(&root, cid, sizeof(int), cudaMemcpyDeviceToHost, st));
        LG_TRY_CUDA(cudaStreamSynchronize(st));
        src = tn;
    }
    // Depth order: a stable sort of node ids by depth (ids ascending within a depth).
    LG_TRY_CUDA(cudaMemsetAsync(parent, 0xff, sizeof(int) * (size_t)n_nodes, st));
    parent_of_kernel<<<g, kTB, 0, st>>>(src, n_nodes, parent);
    depth_of_kernel<<<g, kTB, 0, st>>>(n_nodes, root, parent, depth, ids);
    LG_TRY_CUDA(cudaGetLastError());
    LG_TRY_CUDA(radix_sort_pairs(depth, ids, (size_t)n_nodes, 0, 8, radix_sort_bind(sort_mem, (size_t)n_nodes), st));
    uint32_t max_depth = 0;
    LG_TRY_CUDA(cudaMemcpyAsync(&max_depth, depth + n_nodes - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    rank_kernel<<<g, kTB, 0, st>>>(ids, n_nodes, newpos);
    emit_kernel<<<g, kTB, 0, st>>>(src, ids, newpos, n_nodes, d_out);
    LG_TRY_CUDA(cudaGetLastError());
    LG_TRY_CUDA(cudaStreamSynchronize(st));
    if (max_depth >= 255u) return set_error(LG_ERR_CAPACITY, "render tree: depth over 254");
    return LG_OK;
}
}  // namespace lg
