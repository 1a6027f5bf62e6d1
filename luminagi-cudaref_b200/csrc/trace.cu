// trace.cu -- the path tracer: device scene conversion, trace kernel, tonemap.
//
// Follows the reference's device code (LuminaGI-CudaRef src/pathtracer.cu)
// path for path: same camera model (primary_ray, :284-293), xorshift32
// stream seeded per (pixel, chunk of 8 samples) (:193-204, :349), Moller-
// Trumbore with |det| < 1e-6 culling (:82-107), slab test (:61-80), Lambert +
// next-event estimation to the sun and point lights with a shadow ray even
// at zero sun intensity (:230-272), Russian roulette from bounce 1 and
// cosine-weighted bounces (:295-331).  Every FP32 expression of the camera,
// the triangle test and the shading keeps the reference's operand order, so
// the compiler sees the same expressions.
//
// What is different (none of it changes which triangle a ray hits, except for
// exact ties in t and rays within rounding distance of a box face):
//   * BVH records hold up to four children's boxes (Wide4Node, 64 bytes, the
//     planes quantized to 8 bits on a per-record grid, rounded outwards),
//     built from a render tree over the same triangles; traversal enters the
//     nearest hit child and stacks the others nearest-on-top; the reference
//     pops children in fixed order and tests each box after a separate
//     40-byte fetch.  The 4-wide box test picks each axis's near and far
//     planes by the sign of 1/d and evaluates them with fused multiply-adds
//     (box4).  The 2-wide records (WideNode) keep the reference's exact boxes
//     and slab arithmetic.
//   * Triangle records for intersection are v0, e1, e2 as float4s
//     (e1 = v1 - v0 is the same IEEE subtraction the reference does per test);
//     normals are read from the 100-byte record only at the closest hit.
//   * The path is a per-lane state machine around ONE traversal shared by
//     camera, bounce and shadow rays; persistent warps refill idle lanes with
//     (pixel, chunk of 8 samples) items from an atomic counter.  The warp
//     steps its lanes' traversals one record or leaf at a time, postpones
//     leaves until every lane holds one, and lets lanes whose rays finished
//     shade and start their next ray once enough of them have.  Chunk sums
//     are added to the FP32 accumulator atomically: the order of chunk
//     additions (not their values) can differ from the reference's
//     launch-per-chunk order.
#include <algorithm>
#include <cstdint>

#include <cuda_runtime.h>

#include "trace.cuh"

namespace lg
{
namespace
{
constexpr int kMaxLevels = 128;  // depth limit of the 4-wide collapse (the reference tree is at most ~31 deep)
constexpr int kTraceThreads = 256;
constexpr int kTraceMinBlocks = 4;

// ---------------------------------------------------------------------------
// Scene conversion
// ---------------------------------------------------------------------------
constexpr int kScanTB = 1024;

__global__ void flags_kernel(const lg_bvh_node* __restrict__ nodes, int n, int* __restrict__ is_internal)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) is_internal[i] = nodes[i].triCount == 0 ? 1 : 0;
}

// In-block exclusive scan of `v` (one value per thread); returns the block total in *total.
__device__ int block_exclusive_scan(int v, int* total)
{
    __shared__ int ws[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    if (warp == 0)
    {
        int w = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        ws[lane] = w;
    }
    __syncthreads();
    const int excl = (warp ? ws[warp - 1] : 0) + x - v;
    *total = ws[(blockDim.x >> 5) - 1];
    __syncthreads();
    return excl;
}

// Dense indices: internal nodes and leaves each numbered in BFS order.
// Pass 1: per-block internal counts.
__global__ void __launch_bounds__(kScanTB) count_kernel(const int* __restrict__ is_internal, int n,
                                                        int* __restrict__ block_sums)
{
    const int i = blockIdx.x * kScanTB + threadIdx.x;
    int v = i < n ? is_internal[i] : 0;
    int total;
    block_exclusive_scan(v, &total);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}
// Pass 2: scan of block sums (single block, loops).
__global__ void __launch_bounds__(kScanTB) scan_sums_kernel(int* __restrict__ block_sums, int nb)
{
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b = 0; b < nb; b += kScanTB)
    {
        const int i = b + threadIdx.x;
        int v = i < nb ? block_sums[i] : 0;
        int total;
        int e = block_exclusive_scan(v, &total);
        if (i < nb) block_sums[i] = carry + e;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
}
// Pass 3: dense index per node (internal rank or leaf rank).
__global__ void __launch_bounds__(kScanTB) dense_kernel(const int* __restrict__ is_internal, int n,
                                                        const int* __restrict__ block_sums, int* __restrict__ dense)
{
    const int i = blockIdx.x * kScanTB + threadIdx.x;
    int v = i < n ? is_internal[i] : 0;
    int total;
    int e = block_exclusive_scan(v, &total) + block_sums[blockIdx.x];
    if (i < n) dense[i] = v ? e : (i - e);  // leaves: i - (#internal before i)
}

__device__ __forceinline__ int child_link(const lg_bvh_node* nodes, const int* dense, int c)
{
    return nodes[c].triCount == 0 ? dense[c] : ~dense[c];
}

__global__ void wide_kernel(const lg_bvh_node* __restrict__ nodes, int n, const int* __restrict__ dense,
                            WideNode* __restrict__ wide, int2* __restrict__ leaves)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const lg_bvh_node nd = nodes[i];
    if (nd.triCount > 0)
    {
        leaves[dense[i]] = make_int2(nd.firstTri, nd.triCount);
        return;
    }
    const lg_bvh_node a = nodes[nd.left], b = nodes[nd.right];
    WideNode w;
    w.xy0 = make_float4(a.bbMin[0], a.bbMax[0], a.bbMin[1], a.bbMax[1]);
    w.xy1 = make_float4(b.bbMin[0], b.bbMax[0], b.bbMin[1], b.bbMax[1]);
    w.z01 = make_float4(a.bbMin[2], a.bbMax[2], b.bbMin[2], b.bbMax[2]);
    w.link = make_int4(child_link(nodes, dense, nd.left), child_link(nodes, dense, nd.right), 0, 0);
    wide[dense[i]] = w;
}

// ---- 4-wide collapse ----
__global__ void parent_kernel(const lg_bvh_node* __restrict__ nodes, int n, int* __restrict__ parent)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (i == 0) parent[0] = -1;
    const lg_bvh_node nd = nodes[i];
    if (nd.triCount == 0)
    {
        parent[nd.left] = i;
        parent[nd.right] = i;
    }
}
// Depth of every node (BFS order: depths are non-decreasing along the array).
__global__ void depth_kernel(int n, const int* __restrict__ parent, int* __restrict__ depth)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int d = 0;
    for (int a = i; a != 0; a = parent[a]) ++d;
    depth[i] = d;
}
__global__ void level_start_kernel(int n, const int* __restrict__ depth, int* __restrict__ level_start, int max_levels)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if ((i == 0 || depth[i] != depth[i - 1]) && depth[i] < max_levels) level_start[depth[i]] = i;
}
__device__ __forceinline__ float half_area(const lg_bvh_node& b)
{
    const float dx = b.bbMax[0] - b.bbMin[0], dy = b.bbMax[1] - b.bbMin[1], dz = b.bbMax[2] - b.bbMin[2];
    return dx * dy + dy * dz + dz * dx;
}
// Children of the 4-wide record rooted at internal node i (a record root,
// is4[i] = 1), processed one BVH depth at a time from the root: start from
// i's two children and, while fewer than four, replace the internal child of
// largest surface area by its two children.  The record's internal children
// become record roots themselves (they are deeper, so their level comes later).
// rb[i]: stack entries a ray may hold when it reaches record root i (set by
// the record above it; 0 at the root); *bound receives the largest value a
// visit can leave, rb[i] + (children of i) - 1.
__global__ void select4_kernel(const lg_bvh_node* __restrict__ nodes, int lo, int hi, int* __restrict__ is4,
                               int* __restrict__ sel, int* __restrict__ rb, int* __restrict__ bound)
{
    const int i = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= hi || !is4[i]) return;
    const lg_bvh_node nd = nodes[i];
    int c[4] = {nd.left, nd.right, -1, -1};
    int k = 2;
    while (k < 4)
    {
        int best = -1;
        float best_a = -1.0f;
        for (int j = 0; j < k; ++j)
        {
            const lg_bvh_node& cj = nodes[c[j]];
            if (cj.triCount > 0) continue;
            const float a = half_area(cj);
            if (a > best_a) { best_a = a; best = j; }
        }
        if (best < 0) break;
        const lg_bvh_node& cb = nodes[c[best]];
        c[best] = cb.left;
        c[k++] = cb.right;
    }
    const int here = rb[i] + k - 1;
    atomicMax(bound, here);
    for (int j = 0; j < 4; ++j)
    {
        sel[4 * i + j] = c[j];
        if (c[j] >= 0 && nodes[c[j]].triCount == 0)
        {
            is4[c[j]] = 1;
            rb[c[j]] = here;
        }
    }
}

// Per-block totals, scan and dense numbering are shared with build_wide_nodes
// (count_kernel / scan_sums_kernel / dense_kernel).
__device__ __forceinline__ void put_child(float (&lo)[3][4], float (&hi)[3][4], int (&ln)[4], int& k,
                                          const lg_bvh_node& c, int link)
{
    for (int a = 0; a < 3; ++a)
    {
        lo[a][k] = c.bbMin[a];
        hi[a][k] = c.bbMax[a];
    }
    ln[k] = link;
    ++k;
}
// Leaf links of the 4-wide records carry the leaf itself: ~(first << 4 |
// count) for 1..15 triangles, so the traversal needs no leaf-table load; a
// larger leaf (a run of equal Morton codes) is ~(leaf index << 4), count 0,
// and is read from the table.  Scenes of 2^27 triangles or more keep ~leaf
// index for every leaf (inline_ok = 0).
__device__ __forceinline__ int leaf_link4(const lg_bvh_node& c, int leaf_index, int inline_ok)
{
    if (!inline_ok) return ~leaf_index;
    return c.triCount < 16 ? ~((c.firstTri << 4) | c.triCount) : ~(leaf_index << 4);
}

// Grid of one axis of a quantized record over its nk children's planes:
// step 2^E with the record's extent within 252 steps and at least two ulps of
// its coordinates, origin one step below its min rounded down, planes one
// step outside each child's exact box (floor for min, ceil for max).
__device__ void quantize_axis(const float (&lo)[4], const float (&hi)[4], int nk, float& origin, float& step_out,
                              uint32_t& qlo, uint32_t& qhi)
{
    float pl = lo[0], ph = hi[0];
    for (int k = 1; k < nk; ++k) { pl = fminf(pl, lo[k]); ph = fmaxf(ph, hi[k]); }
    const double ext = (double)ph - (double)pl;
    const double m = fmax(fabs((double)pl), fabs((double)ph));
    int E = -126;
    if (ext > 0.0) E = max(E, (int)ceil(log2(ext / 252.0)));
    if (m > 0.0) E = max(E, ilogb(m) - 22);
    E = min(E, 127);
    const double step = ldexp(1.0, E);
    origin = __double2float_rd((double)pl - step);
    step_out = (float)step;  // a power of two in the normal range: exact
    qlo = 0xffffffffu;  // absent children: 255 / 0
    qhi = 0u;
    for (int k = 0; k < nk; ++k)
    {
        const int ql = min(255, max(0, (int)floor(((double)lo[k] - (double)origin) / step) - 1));
        const int qh = min(255, max(0, (int)ceil(((double)hi[k] - (double)origin) / step) + 1));
        qlo = (qlo & ~(0xffu << (8 * k))) | ((uint32_t)ql << (8 * k));
        qhi |= (uint32_t)qh << (8 * k);
    }
}

__global__ void wide4_kernel(const lg_bvh_node* __restrict__ nodes, int n, const int* __restrict__ is4,
                             const int* __restrict__ dense4, const int* __restrict__ dense2,
                             const int* __restrict__ sel, Wide4Node* __restrict__ out, int inline_ok, int null_link)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !is4[i]) return;
    float lo[3][4], hi[3][4];
    int ln[4];
    for (int a = 0; a < 3; ++a)
        for (int k = 0; k < 4; ++k) { lo[a][k] = 0.0f; hi[a][k] = 0.0f; }
    for (int k = 0; k < 4; ++k) ln[k] = null_link;
    int k = 0;
    for (int j = 0; j < 4; ++j)
    {
        const int ci = sel[4 * i + j];
        if (ci < 0) continue;
        const lg_bvh_node c = nodes[ci];
        put_child(lo, hi, ln, k, c, c.triCount > 0 ? leaf_link4(c, dense2[ci], inline_ok) : dense4[ci]);
    }
    Wide4Node w;
    for (int a = 0; a < 3; ++a) quantize_axis(lo[a], hi[a], k, w.o[a], w.step[a], w.qlo[a], w.qhi[a]);
    for (int j = 0; j < 4; ++j) w.link[j] = ln[j];
    out[dense4[i]] = w;
}

__global__ void tri_prep_kernel(const lg_triangle* __restrict__ tris, int n, float4* __restrict__ tv, int watertight)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const lg_triangle t = tris[i];
    tv[kTriVec * i + 0] = make_float4(t.v[0][0], t.v[0][1], t.v[0][2], __int_as_float(t.material));
    if (kTriVec > 3) tv[kTriVec * i + 3] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (watertight)
    {
        // the watertight test needs the shared vertices themselves, not edges
        tv[kTriVec * i + 1] = make_float4(t.v[1][0], t.v[1][1], t.v[1][2], 0.0f);
        tv[kTriVec * i + 2] = make_float4(t.v[2][0], t.v[2][1], t.v[2][2], 0.0f);
        return;
    }
    tv[kTriVec * i + 1] = make_float4(__fsub_rn(t.v[1][0], t.v[0][0]), __fsub_rn(t.v[1][1], t.v[0][1]),
                                __fsub_rn(t.v[1][2], t.v[0][2]), 0.0f);
    tv[kTriVec * i + 2] = make_float4(__fsub_rn(t.v[2][0], t.v[0][0]), __fsub_rn(t.v[2][1], t.v[0][1]),
                                __fsub_rn(t.v[2][2], t.v[0][2]), 0.0f);
}

#include "trace_dev.cuh"

// Per-lane path state of the chunk being traced (accumulate_kernel's sample
// loop, :352-358, and trace_path, :295-331, unrolled into a state machine).
// Each unoccluded light's throughput x contribution goes straight into the
// chunk sum, where the reference first sums the lights of a bounce, then the
// bounces of a sample, then the samples: the same terms added in another
// FP32 order (rounding-level differences), with two vec3s less live state
// across the traversal.
struct PathState
{
    Ray ray;
    float tmax;
    vec3 throughput, P, N, albedo, contrib, sum;
    double sum64x, sum64y, sum64z;  // judge images only: the same terms added in FP64
    uint32_t rng;
    int px, py, k, n_this, bounce, li;  // li: -1 camera/bounce ray in flight, >= 0 shadow ray of light li
    unsigned pixel;                     // index of the pixel's first accumulator value
    int job;                            // batched launches: the frame this item belongs to
};

// Frame of a global work item in a batched launch: the last job whose
// item_begin is <= item (jobs are in item order).
__device__ __forceinline__ int find_job(const BatchJob* __restrict__ jobs, int n_jobs, unsigned long long item)
{
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&jobs[mid].item_begin) <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void start_sample(PathState& st, const DevCam& cam)
{
    st.throughput = v3(1, 1, 1);
    st.bounce = 0;
    st.li = -1;
    st.tmax = 1e30f;
    float jx = randf(st.rng);
    float jy = randf(st.rng);
    st.ray = primary_ray(cam, st.px, st.py, jx, jy);
}

// Consumes the result of the ray in flight and sets up the next one.
// Returns false when the chunk's last sample has finished.  kAcc64: every
// radiance term is also multiplied and added in FP64.
template <bool kAcc64>
__device__ __forceinline__ bool advance(PathState& st, const DevScene& s, const DevCam& cam, int maxBounces, int tri,
                                        float hitT, float hitU, float hitV)
{
    bool path_done = false;
    if (st.li < 0)
    {
        if (tri < 0) path_done = true;  // miss: no environment light
        else
        {
            const lg_triangle& t = s.tris[tri];
            float w = 1.0f - hitU - hitV;
            vec3 N = normalize(v3(w * t.n[0][0] + hitU * t.n[1][0] + hitV * t.n[2][0],
                                  w * t.n[0][1] + hitU * t.n[1][1] + hitV * t.n[2][1],
                                  w * t.n[0][2] + hitU * t.n[1][2] + hitV * t.n[2][2]));
            if (dot(N, st.ray.d) > 0.0f) N = vmul(N, -1.0f);
            st.N = N;
            st.P = vadd(st.ray.o, vmul(st.ray.d, hitT));
            const int mat = __float_as_int(__ldg(&s.tv[kTriVec * tri].w));
            st.albedo = hit_albedo(s, t, mat, w, hitU, hitV);
        }
    }
    else if (tri < 0)
    {
        // light li unoccluded
        st.sum = vadd(st.sum, vhad(st.throughput, st.contrib));
        if (kAcc64)
        {
            st.sum64x += (double)st.throughput.x * (double)st.contrib.x;
            st.sum64y += (double)st.throughput.y * (double)st.contrib.y;
            st.sum64z += (double)st.throughput.z * (double)st.contrib.z;
        }
    }
    if (!path_done)
    {
        for (int next = st.li + 1; next <= s.n_points; ++next)
            if (light_query(s, next, st.P, st.N, st.albedo, st.ray, st.tmax, st.contrib))
            {
                st.li = next;
                return true;
            }
        if (st.bounce == maxBounces) path_done = true;
        else
        {
            if (st.bounce >= 1)
            {
                float q = fminf(0.95f, fmaxf(st.throughput.x, fmaxf(st.throughput.y, st.throughput.z)));
                if (randf(st.rng) > q) path_done = true;
                else st.throughput = vmul(st.throughput, 1.0f / q);
            }
            if (!path_done)
            {
                vec3 newDir = sample_cos_hemi(st.N, st.rng);
                st.ray = make_ray(vadd(st.P, vmul(st.N, 1e-3f)), newDir);
                st.throughput = vhad(st.throughput, st.albedo);
                st.tmax = 1e30f;
                st.li = -1;
                ++st.bounce;
                return true;
            }
        }
    }
    if (++st.k == st.n_this) return false;
    start_sample(st, cam);
    return true;
}

// Persistent warps.  A lane owns one (pixel, chunk of <= 8 samples) item at a
// time and takes the next item as soon as it finishes, so every iteration of
// the loop is one warp-wide traversal (camera, bounce or shadow ray per lane)
// followed by a short state update.  Items are numbered chunk-major, then by
// 8x4 pixel tile, so neighbouring lanes start on neighbouring pixels.
// kBatch: several frames per launch (job.jobs), each item mapped to its frame
// at refill; the frame's camera and bounce limit are read from the job table.
template <bool kCount, bool kAcc64, int kWidth, bool kWT, bool kBatch, bool kTop = false, bool kChecked = true>
__global__ void __launch_bounds__(kTraceThreads, kTraceMinBlocks) trace_kernel(DevScene s, DevCam cam, TraceJob job)
{
    // kTop: the top of the tree (the first top_n records in BFS order), copied
    // once per block into dynamic shared memory; every ray starts there.  The
    // other instantiations carry no trace of it (top_n is the constant 0).
    extern __shared__ __align__(32) float4 smem_top[];
    const Wide4Node* s_top = reinterpret_cast<const Wide4Node*>(smem_top);
    const int top_n = (kTop && kWidth == 4) ? min(job.top_records, s.n4) : 0;
    for (int i = threadIdx.x; i < top_n * 4; i += kTraceThreads)
        smem_top[i] = __ldg(reinterpret_cast<const float4*>(s.nodes4) + i);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const unsigned long long total =
        kBatch ? job.total_items : (unsigned long long)job.n_tiles * job.n_chunks * 32ull;
    Counters cnt{0, 0, 0, 0, 0, 0};
    PathState st;
    Trav q;
    int stack[kStack];
    const int root = kWidth == 4 ? s.root4 : s.root;
    const int thresh = job.refill_threshold < 1 ? 1 : (job.refill_threshold > 32 ? 32 : job.refill_threshold);
    const int quorum = job.leaf_quorum < 0 ? 0 : (job.leaf_quorum > 31 ? 31 : job.leaf_quorum);
    bool active = false, exhausted = false, tdone = false;
    for (;;)
    {
        // Refill idle lanes with one atomic per warp.
        const unsigned need = __ballot_sync(0xffffffffu, !active);
        if (need && !exhausted)
        {
            const int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(job.work64, (unsigned long long)__popc(need));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base + __popc(need) >= total) exhausted = true;
            if (!active)
            {
                unsigned long long item = base + __popc(need & lt_mask);
                if (item < total)
                {
                    int n_tiles = job.n_tiles, tiles_x = job.tiles_x, spp = job.spp, sbase = job.sample_base;
                    if (kBatch)
                    {
                        st.job = find_job(job.jobs, job.n_jobs, item);
                        const BatchJob& b = job.jobs[st.job];
                        item -= b.item_begin;  // item_begin is a multiple of 32
                        n_tiles = b.n_tiles;
                        tiles_x = b.tiles_x;
                        spp = b.spp;
                        sbase = b.sample_base;
                    }
                    const DevCam& c = kBatch ? job.jobs[st.job].cam : cam;
                    const unsigned j = (unsigned)(item & 31ull);
                    const unsigned long long tw = item >> 5;  // tile-wide item
                    const int chunk = (int)(tw / (unsigned long long)n_tiles);
                    const int tile = (int)(tw % (unsigned long long)n_tiles);
                    st.px = (tile % tiles_x) * 8 + (int)(j & 7);
                    st.py = (tile / tiles_x) * 4 + (int)(j >> 3);
                    if (st.px < c.width && st.py < c.height)
                    {
                        const int first = chunk * 8;
                        st.n_this = min(8, spp - first);
                        const int sampleBase = sbase + first;
                        st.rng = (uint32_t)(st.px * 1973 + st.py * 9277 + sampleBase * 26699) | 1u;
                        st.sum = v3(0, 0, 0);
                        st.sum64x = st.sum64y = st.sum64z = 0.0;
                        st.k = 0;
                        st.pixel = (unsigned)((st.py * c.width + st.px) * 3);
                        start_sample(st, c);
                        trav_begin<kCount>(q, root, st.tmax, st.li >= 0, cnt);
                        tdone = false;
                        active = true;
                    }
                }
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        // Lanes that stay idle for good (work exhausted) do not count towards
        // the threshold; idle lanes that can still be refilled do.
        const int idle_final = exhausted ? __popc(__ballot_sync(0xffffffffu, !active)) : 0;
        for (;;)
        {
            if (warp_step<kWidth, kCount, kWT, kChecked>(s, st.ray, st.li >= 0, active && !tdone, quorum, q, stack,
                                                         cnt, s_top, top_n))
                tdone = true;
            const unsigned busy = __ballot_sync(0xffffffffu, active && !tdone);
            if (busy == 0 || 32 - __popc(busy) - idle_final >= thresh) break;
        }
        if (active && tdone)
        {
            const DevCam& c = kBatch ? job.jobs[st.job].cam : cam;
            // batched: the frame's bounce limit is read from the job table (one register less than keeping it)
            const int max_b = kBatch ? job.jobs[st.job].max_bounces : job.max_bounces;
            if (advance<kAcc64>(st, s, c, max_b, q.tri, q.t, q.u, q.v))
            {
                trav_begin<kCount>(q, root, st.tmax, st.li >= 0, cnt);
                tdone = false;
            }
            else
            {
                active = false;
                const unsigned i = st.pixel;
                if (kBatch)
                {
                    float* acc = job.jobs[st.job].accum;
                    atomicAdd(&acc[i + 0], st.sum.x);
                    atomicAdd(&acc[i + 1], st.sum.y);
                    atomicAdd(&acc[i + 2], st.sum.z);
                }
                else if (job.n_chunks == 1)
                {
                    job.accum[i + 0] += st.sum.x;
                    job.accum[i + 1] += st.sum.y;
                    job.accum[i + 2] += st.sum.z;
                }
                else
                {
                    atomicAdd(&job.accum[i + 0], st.sum.x);
                    atomicAdd(&job.accum[i + 1], st.sum.y);
                    atomicAdd(&job.accum[i + 2], st.sum.z);
                }
                if (kAcc64)
                {
                    atomicAdd(&job.accum64[i + 0], st.sum64x);
                    atomicAdd(&job.accum64[i + 1], st.sum64y);
                    atomicAdd(&job.accum64[i + 2], st.sum64z);
                }
            }
        }
    }
    if (kCount)
    {
        for (int o = 16; o; o >>= 1)
        {
            cnt.closest += __shfl_xor_sync(0xffffffffu, cnt.closest, o);
            cnt.shadow += __shfl_xor_sync(0xffffffffu, cnt.shadow, o);
            cnt.overflow += __shfl_xor_sync(0xffffffffu, cnt.overflow, o);
            cnt.nodes += __shfl_xor_sync(0xffffffffu, cnt.nodes, o);
            cnt.tris += __shfl_xor_sync(0xffffffffu, cnt.tris, o);
            cnt.leaves += __shfl_xor_sync(0xffffffffu, cnt.leaves, o);
        }
        if (lane == 0 && job.counters)
        {
            atomicAdd(&job.counters->closest_rays, cnt.closest);
            atomicAdd(&job.counters->shadow_rays, cnt.shadow);
            atomicAdd(&job.counters->stack_overflows, cnt.overflow);
            atomicAdd(&job.counters->node_fetches, cnt.nodes);
            atomicAdd(&job.counters->tri_tests, cnt.tris);
            atomicAdd(&job.counters->leaf_fetches, cnt.leaves);
        }
    }
}

// gbuffer_kernel (:366-411): primary hit through the pixel centre; albedo,
// encoded normal and box-normalised world position as 8-bit RGB.
__device__ __forceinline__ uint8_t enc8(float v) { return (uint8_t)(fminf(1.0f, fmaxf(0.0f, v)) * 255.0f); }

template <int kWidth, bool kWT>
__global__ void gbuffer_kernel(DevScene s, DevCam cam, vec3 bbMin, vec3 bbInvExtent, uint8_t* __restrict__ albedo_out,
                               uint8_t* __restrict__ normal_out, uint8_t* __restrict__ worldpos_out)
{
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    const int py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= cam.width || py >= cam.height) return;
    Ray r = primary_ray(cam, px, py, 0.5f, 0.5f);
    float hitT, hitU, hitV;
    Counters cnt{0, 0, 0, 0, 0, 0};
    const int tri = traverse_ray<kWidth, false, kWT>(s, r, 1e30f, false, hitT, hitU, hitV, cnt);
    const size_t i = ((size_t)py * cam.width + px) * 3;
    if (tri < 0)
    {
        albedo_out[i + 0] = albedo_out[i + 1] = albedo_out[i + 2] = 0;
        normal_out[i + 0] = 128;
        normal_out[i + 1] = 128;
        normal_out[i + 2] = 255;
        worldpos_out[i + 0] = worldpos_out[i + 1] = worldpos_out[i + 2] = 0;
        return;
    }
    const lg_triangle& t = s.tris[tri];
    float w = 1.0f - hitU - hitV;
    vec3 N = normalize(v3(w * t.n[0][0] + hitU * t.n[1][0] + hitV * t.n[2][0],
                          w * t.n[0][1] + hitU * t.n[1][1] + hitV * t.n[2][1],
                          w * t.n[0][2] + hitU * t.n[1][2] + hitV * t.n[2][2]));
    if (dot(N, r.d) > 0.0f) N = vmul(N, -1.0f);
    const int mat = __float_as_int(__ldg(&s.tv[kTriVec * tri].w));
    const vec3 a = hit_albedo(s, t, mat, w, hitU, hitV);
    albedo_out[i + 0] = enc8(a.x);
    albedo_out[i + 1] = enc8(a.y);
    albedo_out[i + 2] = enc8(a.z);
    normal_out[i + 0] = enc8(N.x * 0.5f + 0.5f);
    normal_out[i + 1] = enc8(N.y * 0.5f + 0.5f);
    normal_out[i + 2] = enc8(N.z * 0.5f + 0.5f);
    vec3 P = vadd(r.o, vmul(r.d, hitT));
    vec3 Pn = vhad(vsub(P, bbMin), bbInvExtent);
    worldpos_out[i + 0] = enc8(Pn.x);
    worldpos_out[i + 1] = enc8(Pn.y);
    worldpos_out[i + 2] = enc8(Pn.z);
}

// tonemap_kernel (:413-429), one value per thread.
__global__ void tonemap_kernel(const float* __restrict__ accum, uint8_t* __restrict__ rgb, long long n, float invSpp)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float v = sqrtf(fmaxf(0.0f, fminf(accum[i] * invSpp, 1.0f)));
    rgb[i] = (uint8_t)(v * 255.0f);
}

__global__ void acc64_to_32_kernel(const double* __restrict__ a, float* __restrict__ b, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}
}  // namespace

DevCam make_dev_cam(const lg_camera& c)
{
    DevCam cam;
    const float* m = c.camera_to_world;
    cam.pos = v3(c.pos[0], c.pos[1], c.pos[2]);
    cam.fwd = v3(m[0], m[1], m[2]);
    cam.left = v3(m[4], m[5], m[6]);
    cam.up = v3(m[8], m[9], m[10]);
    cam.tanHalfFov = tanf(c.fov_y_deg * 0.5f * 3.14159265358979f / 180.0f);
    cam.aspect = c.aspect;
    cam.width = c.width;
    cam.height = c.height;
    return cam;
}

cudaError_t build_wide_nodes(const lg_bvh_node* d_nodes, int n_nodes, WideNode* d_wide, int2* d_leaves,
                             int* d_scratch, int* root_host, int* n_internal_host, int* n_leaves_host,
                             cudaStream_t stream)
{
    const int nb = (n_nodes + kScanTB - 1) / kScanTB;
    int* is_internal = d_scratch;
    int* dense = d_scratch + n_nodes;
    int* block_sums = d_scratch + 2 * (size_t)n_nodes;
    flags_kernel<<<nb, kScanTB, 0, stream>>>(d_nodes, n_nodes, is_internal);
    count_kernel<<<nb, kScanTB, 0, stream>>>(is_internal, n_nodes, block_sums);
    scan_sums_kernel<<<1, kScanTB, 0, stream>>>(block_sums, nb);
    dense_kernel<<<nb, kScanTB, 0, stream>>>(is_internal, n_nodes, block_sums, dense);
    wide_kernel<<<(n_nodes + 255) / 256, 256, 0, stream>>>(d_nodes, n_nodes, dense, d_wide, d_leaves);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    int root_internal = 0;
    e = cudaMemcpyAsync(&root_internal, is_internal, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return e;
    *root_host = root_internal ? 0 : ~0;
    // n_nodes = 2L - 1 for L leaves.
    *n_leaves_host = (n_nodes + 1) / 2;
    *n_internal_host = n_nodes - *n_leaves_host;
    return cudaSuccess;
}

cudaError_t build_wide4_nodes(const lg_bvh_node* d_nodes, int n_nodes, int n_tris, int null_leaf, Wide4Node* d_wide4,
                              int* d_scratch, int* root4_host, int* n4_host, int* leaf_inline_host,
                              int* stack4_host, int* stack2_host, cudaStream_t stream)
{
    // scratch: [is_internal | dense2 | block_sums] from build_wide_nodes, then
    // [parent | is4 | dense4 | sums4 | depth | sel (4 per node) | level_start]
    const int nb = (n_nodes + kScanTB - 1) / kScanTB;
    const int* dense2 = d_scratch + n_nodes;
    int* parent = d_scratch + 2 * (size_t)n_nodes + nb + 8;
    int* is4 = parent + n_nodes;
    int* dense4 = is4 + n_nodes;
    int* sums4 = dense4 + n_nodes;
    int* depth = sums4 + nb + 8;
    int* sel = depth + n_nodes;
    int* level_start = sel + 4 * (size_t)n_nodes;
    const int tb = 256, g = (n_nodes + tb - 1) / tb;
    parent_kernel<<<g, tb, 0, stream>>>(d_nodes, n_nodes, parent);
    depth_kernel<<<g, tb, 0, stream>>>(n_nodes, parent, depth);
    level_start_kernel<<<g, tb, 0, stream>>>(n_nodes, depth, level_start, kMaxLevels);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    lg_bvh_node root{};
    int levels = 0;
    int starts[kMaxLevels + 1];
    e = cudaMemcpyAsync(&root, d_nodes, sizeof(root), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&levels, depth + n_nodes - 1, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return e;
    levels += 1;  // the last node has the largest depth
    if (levels > kMaxLevels) return cudaErrorInvalidValue;
    e = cudaMemcpyAsync(starts, level_start, sizeof(int) * levels, cudaMemcpyDeviceToHost, stream);
    // the depth array is free from here on: it holds the records' stack counts
    // (rb, root 0); the bound goes after the level table
    int* rb = depth;
    int* bound = level_start + kMaxLevels + 1;
    if (e == cudaSuccess) e = cudaMemsetAsync(rb, 0, sizeof(int), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(bound, 0, sizeof(int), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(is4, 0, sizeof(int) * (size_t)n_nodes, stream);
    static const int kOne = 1;
    if (e == cudaSuccess && root.triCount == 0) e = cudaMemcpyAsync(is4, &kOne, sizeof(int), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return e;
    starts[levels] = n_nodes;
    // Record roots and their children, one depth at a time from the top.
    for (int d = 0; d + 1 < levels; ++d)
    {
        const int lo = starts[d], hi = starts[d + 1];
        if (hi > lo)
            select4_kernel<<<(hi - lo + tb - 1) / tb, tb, 0, stream>>>(d_nodes, lo, hi, is4, sel, rb, bound);
    }
    count_kernel<<<nb, kScanTB, 0, stream>>>(is4, n_nodes, sums4);
    scan_sums_kernel<<<1, kScanTB, 0, stream>>>(sums4, nb);
    dense_kernel<<<nb, kScanTB, 0, stream>>>(is4, n_nodes, sums4, dense4);
    const int inline_ok = n_tris < (1 << 27) ? 1 : 0;
    *leaf_inline_host = inline_ok;
    const int null_link = inline_ok ? ~(null_leaf << 4) : ~null_leaf;
    wide4_kernel<<<g, tb, 0, stream>>>(d_nodes, n_nodes, is4, dense4, dense2, sel, d_wide4, inline_ok, null_link);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    int last_d = 0, last_v = 0, stack4 = 0;
    e = cudaMemcpyAsync(&last_d, dense4 + n_nodes - 1, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&last_v, is4 + n_nodes - 1, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&stack4, bound, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return e;
    *root4_host = root.triCount == 0 ? 0 : ~0;
    // dense4 of the last node: its rank among record roots if it is one, else
    // its rank among the others (so the roots before it number n - 1 - rank)
    *n4_host = last_v ? last_d + 1 : (n_nodes - 1 - last_d);
    *stack4_host = stack4;
    *stack2_host = levels - 1;  // one entry per internal ancestor, plus the deepest internal node's own push
    return cudaSuccess;
}

cudaError_t prepare_triangles(const lg_triangle* d_tris, int n, float4* d_tv, bool watertight, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    tri_prep_kernel<<<(n + 255) / 256, 256, 0, stream>>>(d_tris, n, d_tv, watertight ? 1 : 0);
    return cudaGetLastError();
}

template <bool kCount, bool kAcc64, int W, bool kWT, bool kBatch = false, bool kTop = false, bool kChecked = true>
static cudaError_t launch_trace_t(const DevScene& s, const DevCam& cam, const TraceJob& job, int sm_count,
                                  cudaStream_t stream)
{
    const void* fn = (const void*)trace_kernel<kCount, kAcc64, W, kWT, kBatch, kTop, kChecked>;
    const int top_n = (kTop && W == 4) ? std::min(std::max(job.top_records, 0), s.n4) : 0;
    const size_t smem = (size_t)top_n * sizeof(Wide4Node);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kTraceThreads, smem);
    if (e != cudaSuccess) return e;
    if (job.blocks_per_sm > 0 && job.blocks_per_sm < per_sm) per_sm = job.blocks_per_sm;
    const long long lanes = kBatch ? (long long)job.total_items : (long long)job.n_tiles * job.n_chunks * 32;
    long long blocks = (long long)(per_sm < 1 ? 1 : per_sm) * sm_count;
    const long long useful = (lanes + kTraceThreads - 1) / kTraceThreads;
    if (blocks > useful) blocks = useful;
    if (blocks < 1) blocks = 1;
    e = cudaMemsetAsync(job.work64, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    trace_kernel<kCount, kAcc64, W, kWT, kBatch, kTop, kChecked><<<(int)blocks, kTraceThreads, smem, stream>>>(s, cam,
                                                                                                          job);
    return cudaGetLastError();
}

cudaError_t launch_trace_batch(const DevScene& s, const TraceJob& job, int sm_count, int width, bool watertight,
                               cudaStream_t stream)
{
    const DevCam none{};
    if (width == 4 && job.top_records > 0)
        return watertight ? launch_trace_t<false, false, 4, true, true, true>(s, none, job, sm_count, stream)
                          : launch_trace_t<false, false, 4, false, true, true>(s, none, job, sm_count, stream);
    if (job.stack_safe)
    {
        if (watertight)
            return width == 4 ? launch_trace_t<false, false, 4, true, true, false, false>(s, none, job, sm_count, stream)
                              : launch_trace_t<false, false, 2, true, true, false, false>(s, none, job, sm_count, stream);
        return width == 4 ? launch_trace_t<false, false, 4, false, true, false, false>(s, none, job, sm_count, stream)
                          : launch_trace_t<false, false, 2, false, true, false, false>(s, none, job, sm_count, stream);
    }
    if (watertight)
        return width == 4 ? launch_trace_t<false, false, 4, true, true>(s, none, job, sm_count, stream)
                          : launch_trace_t<false, false, 2, true, true>(s, none, job, sm_count, stream);
    return width == 4 ? launch_trace_t<false, false, 4, false, true>(s, none, job, sm_count, stream)
                      : launch_trace_t<false, false, 2, false, true>(s, none, job, sm_count, stream);
}

template <int W, bool kWT>
static cudaError_t launch_trace_w(const DevScene& s, const DevCam& cam, const TraceJob& job, bool count, int sm_count,
                                 cudaStream_t stream)
{
    // the shared-memory top records serve the plain 4-wide frames (they change no result, so
    // counting and FP64 frames run without them)
    if (W == 4 && job.top_records > 0 && !count && !job.accum64)
        return launch_trace_t<false, false, W, kWT, false, true>(s, cam, job, sm_count, stream);
    // trees whose stack bound fits: no push checks (counting runs keep them, and count overflows)
    if (job.stack_safe && !count)
        return job.accum64 ? launch_trace_t<false, true, W, kWT, false, false, false>(s, cam, job, sm_count, stream)
                           : launch_trace_t<false, false, W, kWT, false, false, false>(s, cam, job, sm_count, stream);
    if (count)
        return job.accum64 ? launch_trace_t<true, true, W, kWT>(s, cam, job, sm_count, stream)
                           : launch_trace_t<true, false, W, kWT>(s, cam, job, sm_count, stream);
    return job.accum64 ? launch_trace_t<false, true, W, kWT>(s, cam, job, sm_count, stream)
                       : launch_trace_t<false, false, W, kWT>(s, cam, job, sm_count, stream);
}

// Four 256-thread blocks per SM (64 registers) measured fastest on B200:
// 653 ms per 64-spp engine-scale frame (binary nodes) vs 745 ms at three
// and 1007 ms at two.
cudaError_t launch_trace(const DevScene& s, const DevCam& cam, const TraceJob& job, bool count, int sm_count,
                         int width, bool watertight, cudaStream_t stream)
{
    if (watertight)
        return width == 4 ? launch_trace_w<4, true>(s, cam, job, count, sm_count, stream)
                          : launch_trace_w<2, true>(s, cam, job, count, sm_count, stream);
    return width == 4 ? launch_trace_w<4, false>(s, cam, job, count, sm_count, stream)
                      : launch_trace_w<2, false>(s, cam, job, count, sm_count, stream);
}

cudaError_t launch_gbuffer(const DevScene& s, const DevCam& cam, vec3 bbMin, vec3 bbInvExtent, uint8_t* d_albedo,
                           uint8_t* d_normal, uint8_t* d_worldpos, int width, bool watertight, cudaStream_t stream)
{
    dim3 block(16, 16);
    dim3 grid((cam.width + 15) / 16, (cam.height + 15) / 16);
    auto k = width == 4 ? (watertight ? gbuffer_kernel<4, true> : gbuffer_kernel<4, false>)
                        : (watertight ? gbuffer_kernel<2, true> : gbuffer_kernel<2, false>);
    k<<<grid, block, 0, stream>>>(s, cam, bbMin, bbInvExtent, d_albedo, d_normal, d_worldpos);
    return cudaGetLastError();
}

cudaError_t launch_tonemap(const float* d_accum, uint8_t* d_rgb, long long n_values, float inv_spp,
                           cudaStream_t stream)
{
    if (n_values <= 0) return cudaSuccess;
    tonemap_kernel<<<(unsigned)((n_values + 255) / 256), 256, 0, stream>>>(d_accum, d_rgb, n_values, inv_spp);
    return cudaGetLastError();
}

cudaError_t launch_accum64_to_32(const double* d_acc64, float* d_acc32, long long n_values, cudaStream_t stream)
{
    if (n_values <= 0) return cudaSuccess;
    acc64_to_32_kernel<<<(unsigned)((n_values + 255) / 256), 256, 0, stream>>>(d_acc64, d_acc32, n_values);
    return cudaGetLastError();
}
}  // namespace lg
