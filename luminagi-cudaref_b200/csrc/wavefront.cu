// wavefront.cu -- the ray-sorted render: the reference's --sort path,
// RenderSceneCUDASorted (LuminaGI-CudaRef src/pathtracer.cu:431-547 for its
// kernels, :759-909 for the host loop), traced with this library's records.
//
// Per sample: a camera ray for every pixel, keyed by a 30-bit Morton code of
// its direction; the (key, slot) pairs sorted stably on the device; then one
// launch per bounce over the sorted slots.  A launch traces each live ray,
// adds throughput x direct light (sun, point lights, a shadow ray each) to
// its pixel, and writes the next ray (cosine-weighted, no Russian roulette)
// with its key; the next bounce's rays are sorted again.
//
// What decides the image, kept as the reference has it:
//   * seeding per (pixel, sample): (px*1973 + py*9277 + sample*26699) | 1
//     (:470); the two jitter draws come from the pixel's own stream, every
//     later draw from the stream stored at the ray's sorted SLOT (rng_state
//     is indexed by slot and not permuted with the rays, :513-515), so the
//     sort order is part of the estimator;
//   * the sort is stable (thrust's radix sort there, this library's LSD
//     radix sort here), dead rays (missed, or finished) key 0xFFFFFFFF and
//     sort last;
//   * each pixel receives at most one atomic add per launch, so the order of
//     its additions is the launch order: the accumulator is deterministic.
//
// What is this library's own: rays move through the sort as 4-byte slot
// indices (the 48-byte rays are gathered through the permutation instead of
// being moved by the sort), and traversal uses the 4-wide quantized records
// (or the 2-wide exact ones) built from the render tree, one whole ray per
// thread -- the sort is what makes neighbouring threads' rays alike.
#include <cstdint>

#include <cuda_runtime.h>

#include "radix_sort.cuh"
#include "trace.cuh"
#include "wavefront.cuh"

namespace lg
{
namespace
{
#include "trace_dev.cuh"

constexpr int kWfThreads = 256;
constexpr uint32_t kDeadKey = 0xffffffffu;

// 10 bits of v spread to every third bit of the result (bit i -> bit 3i).
__device__ __forceinline__ uint32_t spread10(uint32_t v)
{
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// Morton key of a unit direction (direction_morton, :456-463): each
// component mapped from [-1, 1] to 0..1023 by (c + 1) * 511.5, clamped and
// truncated, then interleaved x, y, z from the high bit down.
__device__ __forceinline__ uint32_t dir_key(vec3 d)
{
    const uint32_t x = (uint32_t)fmaxf(0.0f, fminf(1023.0f, (d.x + 1.0f) * 511.5f));
    const uint32_t y = (uint32_t)fmaxf(0.0f, fminf(1023.0f, (d.y + 1.0f) * 511.5f));
    const uint32_t z = (uint32_t)fmaxf(0.0f, fminf(1023.0f, (d.z + 1.0f) * 511.5f));
    return (spread10(x) << 2) | (spread10(y) << 1) | spread10(z);
}

__device__ __forceinline__ void store_ray(WfRay* __restrict__ out, int slot, vec3 o, vec3 d, vec3 thr,
                                          uint32_t pixel, uint32_t alive)
{
    out[slot].o = make_float4(o.x, o.y, o.z, __uint_as_float(pixel));
    out[slot].d = make_float4(d.x, d.y, d.z, __uint_as_float(alive));
    out[slot].thr = make_float4(thr.x, thr.y, thr.z, 0.0f);
}

// gen_primary_kernel (:466-487): pixel idx's camera ray for sample `sample`,
// its key, its slot (= idx before sorting) and its RNG state after the
// jitter draws.
__global__ void __launch_bounds__(kWfThreads) wf_primary_kernel(DevCam cam, int sample, WfRay* __restrict__ rays,
                                                               uint32_t* __restrict__ keys,
                                                               uint32_t* __restrict__ slots,
                                                               uint32_t* __restrict__ rng_state)
{
    const int n = cam.width * cam.height;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const int px = idx % cam.width, py = idx / cam.width;
    uint32_t rng = ((uint32_t)px * 1973u + (uint32_t)py * 9277u + (uint32_t)sample * 26699u) | 1u;
    const float jx = randf(rng);
    const float jy = randf(rng);
    const Ray r = primary_ray(cam, px, py, jx, jy);
    store_ray(rays, idx, r.o, r.d, v3(1.0f, 1.0f, 1.0f), (uint32_t)idx, 1u);
    keys[idx] = dir_key(r.d);
    slots[idx] = (uint32_t)idx;
    rng_state[idx] = rng;
}

// trace_and_bounce_kernel (:489-547) for sorted slot j, whose ray is
// rays_in[order[j]].  Writes slot j of the next bounce (ray, key, slot) unless
// `last`.
template <int kWidth, bool kWT, bool kCount>
__global__ void __launch_bounds__(kWfThreads) wf_bounce_kernel(DevScene s, int n, const WfRay* __restrict__ rays_in,
                                                              const uint32_t* __restrict__ order,
                                                              float* __restrict__ accum,
                                                              WfRay* __restrict__ rays_out,
                                                              uint32_t* __restrict__ keys_out,
                                                              uint32_t* __restrict__ slots_out,
                                                              uint32_t* __restrict__ rng_state, int last,
                                                              RenderCounters* __restrict__ counters)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    Counters cnt{0, 0, 0, 0, 0, 0};
    if (j < n)
    {
        const uint32_t src = __ldg(&order[j]);
        const float4 a = __ldg(&rays_in[src].o), b = __ldg(&rays_in[src].d), c = __ldg(&rays_in[src].thr);
        const uint32_t pixel = __float_as_uint(a.w);
        bool alive = __float_as_uint(b.w) != 0u;
        vec3 P, N, thr = v3(c.x, c.y, c.z), albedo;
        if (alive)
        {
            const Ray r = make_ray(v3(a.x, a.y, a.z), v3(b.x, b.y, b.z));
            float hitT, hitU, hitV;
            const int tri = traverse_ray<kWidth, kCount, kWT>(s, r, 1e30f, false, hitT, hitU, hitV, cnt);
            if (tri < 0) alive = false;
            else
            {
                const lg_triangle& t = s.tris[tri];
                const float w = 1.0f - hitU - hitV;
                N = normalize(v3(w * t.n[0][0] + hitU * t.n[1][0] + hitV * t.n[2][0],
                                 w * t.n[0][1] + hitU * t.n[1][1] + hitV * t.n[2][1],
                                 w * t.n[0][2] + hitU * t.n[1][2] + hitV * t.n[2][2]));
                if (dot(N, r.d) > 0.0f) N = vmul(N, -1.0f);
                P = vadd(r.o, vmul(r.d, hitT));
                const int mat = __float_as_int(__ldg(&s.tv[kTriVec * tri].w));
                albedo = hit_albedo(s, t, mat, w, hitU, hitV);
                // shade_direct (:230-272): the sun, then each point light
                vec3 color = v3(0, 0, 0);
                for (int li = 0; li <= s.n_points; ++li)
                {
                    Ray shadow;
                    float tmax;
                    vec3 contrib;
                    if (!light_query(s, li, P, N, albedo, shadow, tmax, contrib)) continue;
                    float st, su, sv;
                    if (traverse_ray<kWidth, kCount, kWT>(s, shadow, tmax, true, st, su, sv, cnt) < 0)
                        color = vadd(color, contrib);
                }
                const vec3 add = vhad(thr, color);
                const unsigned i = pixel * 3u;
                atomicAdd(&accum[i + 0], add.x);
                atomicAdd(&accum[i + 1], add.y);
                atomicAdd(&accum[i + 2], add.z);
            }
        }
        if (!last)
        {
            if (alive)
            {
                uint32_t rng = rng_state[j];
                const vec3 d = sample_cos_hemi(N, rng);
                rng_state[j] = rng;
                store_ray(rays_out, j, vadd(P, vmul(N, 1e-3f)), d, vhad(thr, albedo), pixel, 1u);
                keys_out[j] = dir_key(d);
            }
            else
            {
                store_ray(rays_out, j, v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0), pixel, 0u);
                keys_out[j] = kDeadKey;
            }
            slots_out[j] = (uint32_t)j;
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
        if ((threadIdx.x & 31) == 0 && counters)
        {
            atomicAdd(&counters->closest_rays, cnt.closest);
            atomicAdd(&counters->shadow_rays, cnt.shadow);
            atomicAdd(&counters->stack_overflows, cnt.overflow);
            atomicAdd(&counters->node_fetches, cnt.nodes);
            atomicAdd(&counters->tri_tests, cnt.tris);
            atomicAdd(&counters->leaf_fetches, cnt.leaves);
        }
    }
}

// ---- staged bounce: the same launch split at its traversals ----
// A bounce of the sorted path is four launches: closest hits of the sorted
// rays (wf_trace_list_kernel), shading and the shadow rays
// (wf_shade_kernel), their occlusion (wf_trace_list_kernel again, any-hit),
// and the pixel update with the next rays (wf_finish_kernel).  Each kernel
// computes what wf_bounce_kernel computes for the slot, with the same
// expressions in the same order, so the image does not change (up to rays
// whose two nearest triangles tie exactly); the traversals become
// persistent warps that step their lanes through traversals one record or
// leaf at a time (warp_step, leaves postponed) and take the next ray of
// the list as soon as enough lanes are free, with no shading in between.
constexpr int kWfListThreads = 256;
// The staged bounce keeps a shadow ray, a contribution and a flag per (light, ray): 52 bytes per light and pixel.
// Scenes with more lights than this trace their bounces one ray per thread instead.
constexpr int kWfStagedLights = 8;

// Ray i of a traversal list.  Closest hits (kAny false): the sorted ray
// rays_in[order[i]], its origin and direction through make_ray as
// wf_bounce_kernel takes them; shadow rays (kAny true): origin o = so[i].xyz,
// tmax = so[i].w, the already normalised direction sd[i].xyz (sd[i].w != 0
// if the light was not skipped) and 1/d as make_ray computes it.
template <bool kAny>
__device__ __forceinline__ bool list_ray(const WfRay* __restrict__ rays_in, const uint32_t* __restrict__ order,
                                         const float4* __restrict__ so, const float4* __restrict__ sd, int i, Ray& r,
                                         float& tmax)
{
    if (kAny)
    {
        const float4 d = __ldg(&sd[i]);
        if (__float_as_uint(d.w) == 0u) return false;
        const float4 o = __ldg(&so[i]);
        r.o = v3(o.x, o.y, o.z);
        r.d = v3(d.x, d.y, d.z);
        r.inv_d = v3(1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z);
        tmax = o.w;
        return true;
    }
    const uint32_t src = __ldg(&order[i]);
    const float4 b = __ldg(&rays_in[src].d);
    if (__float_as_uint(b.w) == 0u) return false;
    const float4 a = __ldg(&rays_in[src].o);
    r = make_ray(v3(a.x, a.y, a.z), v3(b.x, b.y, b.z));
    tmax = 1e30f;
    return true;
}

// Persistent traversal of n listed rays.  kAny false: hit[i] = (triangle or
// -1, t, u, v as bits); kAny true: occ[i] = 1 when an occluder was found.
// Idle lanes are refilled, one atomic per warp on *work, once `thresh` of
// them are idle (or the warp has nothing left in flight).
template <int kWidth, bool kWT, bool kAny, bool kChecked>
__global__ void __launch_bounds__(kWfListThreads, 4)
    wf_trace_list_kernel(DevScene s, const WfRay* __restrict__ rays_in, const uint32_t* __restrict__ order,
                         const float4* __restrict__ so, const float4* __restrict__ sd, int n,
                         unsigned long long* __restrict__ work, int quorum, int thresh, int4* __restrict__ hit,
                         int* __restrict__ occ)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int root = kWidth == 4 ? s.root4 : s.root;
    Counters cnt{0, 0, 0, 0, 0, 0};
    int stack[kStack];
    Trav q;
    Ray ray;
    float tmax = 0.0f;
    int idx = -1;
    bool active = false, exhausted = false;
    for (;;)
    {
        const unsigned need = __ballot_sync(0xffffffffu, !active);
        if (need && !exhausted && (__popc(need) >= thresh || need == 0xffffffffu))
        {
            const int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(work, (unsigned long long)__popc(need));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base + __popc(need) >= (unsigned long long)n) exhausted = true;
            if (!active)
            {
                const unsigned long long i = base + __popc(need & lt_mask);
                if (i < (unsigned long long)n)
                {
                    idx = (int)i;
                    if (list_ray<kAny>(rays_in, order, so, sd, idx, ray, tmax))
                    {
                        trav_begin<false>(q, root, tmax, kAny, cnt);
                        active = true;
                    }
                    else if (kAny) occ[idx] = 0;  // a skipped light: nothing traced
                    else hit[idx] = make_int4(-1, 0, 0, 0);
                }
            }
        }
        if (!__any_sync(0xffffffffu, active))
        {
            if (exhausted) break;
            continue;
        }
        if (warp_step<kWidth, false, kWT, kChecked>(s, ray, kAny, active, quorum, q, stack, cnt, nullptr, 0) &&
            active)
        {
            if (kAny) occ[idx] = q.tri >= 0 ? 1 : 0;
            else hit[idx] = make_int4(q.tri, __float_as_int(q.t), __float_as_int(q.u), __float_as_int(q.v));
            active = false;
        }
    }
}

// Shading of sorted slot j after its closest hit: surface point, normal and
// albedo (surf[3j .. 3j+2]), and for light li (0 the sun, then the point
// lights) the shadow ray and its contribution at index li * n + j, or a
// skipped light (sd.w = 0), as wf_bounce_kernel computes them.
__global__ void __launch_bounds__(kWfThreads) wf_shade_kernel(DevScene s, int n, const WfRay* __restrict__ rays_in,
                                                             const uint32_t* __restrict__ order,
                                                             const int4* __restrict__ hit, float4* __restrict__ surf,
                                                             float4* __restrict__ so, float4* __restrict__ sd,
                                                             float4* __restrict__ sc)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int4 h = hit[j];
    if (h.x < 0)
    {
        for (int li = 0; li <= s.n_points; ++li) sd[(size_t)li * n + j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    const uint32_t src = __ldg(&order[j]);
    const float4 a = __ldg(&rays_in[src].o), b = __ldg(&rays_in[src].d);
    const Ray r = make_ray(v3(a.x, a.y, a.z), v3(b.x, b.y, b.z));
    const int tri = h.x;
    const float hitT = __int_as_float(h.y), hitU = __int_as_float(h.z), hitV = __int_as_float(h.w);
    const lg_triangle& t = s.tris[tri];
    const float w = 1.0f - hitU - hitV;
    vec3 N = normalize(v3(w * t.n[0][0] + hitU * t.n[1][0] + hitV * t.n[2][0],
                          w * t.n[0][1] + hitU * t.n[1][1] + hitV * t.n[2][1],
                          w * t.n[0][2] + hitU * t.n[1][2] + hitV * t.n[2][2]));
    if (dot(N, r.d) > 0.0f) N = vmul(N, -1.0f);
    const vec3 P = vadd(r.o, vmul(r.d, hitT));
    const int mat = __float_as_int(__ldg(&s.tv[kTriVec * tri].w));
    const vec3 albedo = hit_albedo(s, t, mat, w, hitU, hitV);
    surf[3 * (size_t)j + 0] = make_float4(P.x, P.y, P.z, 0.0f);
    surf[3 * (size_t)j + 1] = make_float4(N.x, N.y, N.z, 0.0f);
    surf[3 * (size_t)j + 2] = make_float4(albedo.x, albedo.y, albedo.z, 0.0f);
    for (int li = 0; li <= s.n_points; ++li)
    {
        Ray shadow;
        float tmax;
        vec3 contrib;
        const size_t k = (size_t)li * n + j;
        if (!light_query(s, li, P, N, albedo, shadow, tmax, contrib))
        {
            sd[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            continue;
        }
        so[k] = make_float4(shadow.o.x, shadow.o.y, shadow.o.z, tmax);
        sd[k] = make_float4(shadow.d.x, shadow.d.y, shadow.d.z, __uint_as_float(1u));
        sc[k] = make_float4(contrib.x, contrib.y, contrib.z, 0.0f);
    }
}

// Slot j after its shadow rays: the unoccluded lights' contributions summed
// in light order, one add to the pixel, and the next ray with its key (as
// the tail of wf_bounce_kernel).
__global__ void __launch_bounds__(kWfThreads) wf_finish_kernel(const DevScene s, int n,
                                                              const WfRay* __restrict__ rays_in,
                                                              const uint32_t* __restrict__ order,
                                                              const int4* __restrict__ hit,
                                                              const float4* __restrict__ surf,
                                                              const float4* __restrict__ sd,
                                                              const float4* __restrict__ sc,
                                                              const int* __restrict__ occ, float* __restrict__ accum,
                                                              WfRay* __restrict__ rays_out,
                                                              uint32_t* __restrict__ keys_out,
                                                              uint32_t* __restrict__ slots_out,
                                                              uint32_t* __restrict__ rng_state, int last)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t src = __ldg(&order[j]);
    const float4 a = __ldg(&rays_in[src].o), c = __ldg(&rays_in[src].thr);
    const uint32_t pixel = __float_as_uint(a.w);
    const vec3 thr = v3(c.x, c.y, c.z);
    const bool alive = hit[j].x >= 0;
    vec3 P, N, albedo;
    if (alive)
    {
        const float4 p4 = surf[3 * (size_t)j + 0], n4 = surf[3 * (size_t)j + 1], a4 = surf[3 * (size_t)j + 2];
        P = v3(p4.x, p4.y, p4.z);
        N = v3(n4.x, n4.y, n4.z);
        albedo = v3(a4.x, a4.y, a4.z);
        vec3 color = v3(0, 0, 0);
        for (int li = 0; li <= s.n_points; ++li)
        {
            const size_t k = (size_t)li * n + j;
            if (__float_as_uint(sd[k].w) != 0u && occ[k] == 0)
            {
                const float4 q = sc[k];
                color = vadd(color, v3(q.x, q.y, q.z));
            }
        }
        const vec3 add = vhad(thr, color);
        const unsigned i = pixel * 3u;
        atomicAdd(&accum[i + 0], add.x);
        atomicAdd(&accum[i + 1], add.y);
        atomicAdd(&accum[i + 2], add.z);
    }
    if (last) return;
    if (alive)
    {
        uint32_t rng = rng_state[j];
        const vec3 d = sample_cos_hemi(N, rng);
        rng_state[j] = rng;
        store_ray(rays_out, j, vadd(P, vmul(N, 1e-3f)), d, vhad(thr, albedo), pixel, 1u);
        keys_out[j] = dir_key(d);
    }
    else
    {
        store_ray(rays_out, j, v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0), pixel, 0u);
        keys_out[j] = kDeadKey;
    }
    slots_out[j] = (uint32_t)j;
}

template <int W, bool kWT, bool kCount>
cudaError_t launch_bounce(const DevScene& s, int n, const WfRay* in, const uint32_t* order, float* accum,
                          WfRay* out, uint32_t* keys_out, uint32_t* slots_out, uint32_t* rng, bool last,
                          RenderCounters* counters, cudaStream_t st)
{
    const int blocks = (n + kWfThreads - 1) / kWfThreads;
    wf_bounce_kernel<W, kWT, kCount><<<blocks, kWfThreads, 0, st>>>(s, n, in, order, accum, out, keys_out, slots_out,
                                                                    rng, last ? 1 : 0, counters);
    return cudaGetLastError();
}

cudaError_t bounce(const DevScene& s, int width, bool wt, bool count, int n, const WfRay* in, const uint32_t* order,
                   float* accum, WfRay* out, uint32_t* keys_out, uint32_t* slots_out, uint32_t* rng, bool last,
                   RenderCounters* counters, cudaStream_t st)
{
#define LG_WF_BOUNCE(W, T, C) launch_bounce<W, T, C>(s, n, in, order, accum, out, keys_out, slots_out, rng, last, counters, st)
    if (count)
        return width == 4 ? (wt ? LG_WF_BOUNCE(4, true, true) : LG_WF_BOUNCE(4, false, true))
                          : (wt ? LG_WF_BOUNCE(2, true, true) : LG_WF_BOUNCE(2, false, true));
    return width == 4 ? (wt ? LG_WF_BOUNCE(4, true, false) : LG_WF_BOUNCE(4, false, false))
                      : (wt ? LG_WF_BOUNCE(2, true, false) : LG_WF_BOUNCE(2, false, false));
#undef LG_WF_BOUNCE
}
// Buffers of the staged bounce.
struct Staged
{
    int4* hit;
    float4 *surf, *so, *sd, *sc;
    int* occ;
    unsigned long long* work;  // [2]: the closest-hit and the shadow-ray list
};

template <int W, bool kWT, bool kAny, bool kChecked>
cudaError_t launch_list(const DevScene& s, const WavefrontJob& job, const WfRay* in, const uint32_t* order,
                        const Staged& b, int n, unsigned long long* work, cudaStream_t st)
{
    const void* fn = (const void*)wf_trace_list_kernel<W, kWT, kAny, kChecked>;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kWfListThreads, 0);
    if (e != cudaSuccess) return e;
    long long blocks = (long long)(per_sm < 1 ? 1 : per_sm) * (job.sm_count > 0 ? job.sm_count : 1);
    const long long useful = ((long long)n + kWfListThreads - 1) / kWfListThreads;
    if (blocks > useful) blocks = useful;
    if (blocks < 1) blocks = 1;
    e = cudaMemsetAsync(work, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    const int thresh = job.refill < 1 ? 1 : (job.refill > 32 ? 32 : job.refill);
    const int quorum = job.quorum < 0 ? 0 : (job.quorum > 31 ? 31 : job.quorum);
    wf_trace_list_kernel<W, kWT, kAny, kChecked><<<(int)blocks, kWfListThreads, 0, st>>>(
        s, in, order, b.so, b.sd, n, work, quorum, thresh, b.hit, b.occ);
    return cudaGetLastError();
}

template <int W, bool kWT, bool kChecked>
cudaError_t staged_bounce_t(const DevScene& s, const WavefrontJob& job, int n, const WfRay* in, const uint32_t* order,
                            WfRay* out, uint32_t* keys_out, uint32_t* slots_out, uint32_t* rng, bool last,
                            const Staged& b, cudaStream_t st)
{
    const int nl = s.n_points + 1;
    const int blocks = (n + kWfThreads - 1) / kWfThreads;
    cudaError_t e = launch_list<W, kWT, false, kChecked>(s, job, in, order, b, n, b.work, st);
    if (e != cudaSuccess) return e;
    wf_shade_kernel<<<blocks, kWfThreads, 0, st>>>(s, n, in, order, b.hit, b.surf, b.so, b.sd, b.sc);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    e = launch_list<W, kWT, true, kChecked>(s, job, nullptr, nullptr, b, nl * n, b.work + 1, st);
    if (e != cudaSuccess) return e;
    wf_finish_kernel<<<blocks, kWfThreads, 0, st>>>(s, n, in, order, b.hit, b.surf, b.sd, b.sc, b.occ, job.accum, out,
                                                   keys_out, slots_out, rng, last ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t staged_bounce(const DevScene& s, const WavefrontJob& job, int n, const WfRay* in, const uint32_t* order,
                          WfRay* out, uint32_t* keys_out, uint32_t* slots_out, uint32_t* rng, bool last,
                          const Staged& b, cudaStream_t st)
{
#define LG_WF_STAGED(W, T, K) staged_bounce_t<W, T, K>(s, job, n, in, order, out, keys_out, slots_out, rng, last, b, st)
    if (job.stack_safe)
        return job.width == 4 ? (job.watertight ? LG_WF_STAGED(4, true, false) : LG_WF_STAGED(4, false, false))
                              : (job.watertight ? LG_WF_STAGED(2, true, false) : LG_WF_STAGED(2, false, false));
    return job.width == 4 ? (job.watertight ? LG_WF_STAGED(4, true, true) : LG_WF_STAGED(4, false, true))
                          : (job.watertight ? LG_WF_STAGED(2, true, true) : LG_WF_STAGED(2, false, true));
#undef LG_WF_STAGED
}
}  // namespace

size_t wavefront_scratch_bytes(int n_pixels, int n_lights)
{
    const size_t n = (size_t)(n_pixels > 0 ? n_pixels : 1);
    // scenes with more lights than kWfStagedLights run the one-thread-per-ray bounce and need no per-light buffers
    const size_t nl = (n_lights > kWfStagedLights) ? 0 : (size_t)(n_lights > 0 ? n_lights : 1);
    const size_t a = 256;
    auto up = [&](size_t b) { return (b + a - 1) / a * a; };
    return 2 * up(n * sizeof(WfRay)) + 5 * up(n * sizeof(uint32_t)) + up(radix_sort_scratch_bytes(n)) +
           up(n * sizeof(int4)) + up(3 * n * sizeof(float4)) + 3 * up(nl * n * sizeof(float4)) +
           up(nl * n * sizeof(int)) + up(2 * sizeof(unsigned long long)) + a;
}

cudaError_t launch_wavefront_frame(const DevScene& s, const DevCam& cam, const WavefrontJob& job, void* scratch,
                                   size_t scratch_bytes, cudaStream_t st)
{
    const int n = cam.width * cam.height;
    if (n <= 0 || job.spp <= 0) return cudaSuccess;
    const int nl = s.n_points + 1;
    if (scratch_bytes < wavefront_scratch_bytes(n, nl)) return cudaErrorInvalidValue;
    const bool staged = !job.counters && nl <= kWfStagedLights;
    const size_t snl = staged ? (size_t)nl : 0;  // per-light buffers only for the staged launch
    const size_t a = 256;
    auto up = [&](size_t b) { return (b + a - 1) / a * a; };
    char* p = (char*)(((uintptr_t)scratch + a - 1) & ~(uintptr_t)(a - 1));
    WfRay* rays[2];
    uint32_t *keys[2], *slots[2];
    rays[0] = (WfRay*)p; p += up((size_t)n * sizeof(WfRay));
    rays[1] = (WfRay*)p; p += up((size_t)n * sizeof(WfRay));
    keys[0] = (uint32_t*)p; p += up((size_t)n * sizeof(uint32_t));
    keys[1] = (uint32_t*)p; p += up((size_t)n * sizeof(uint32_t));
    slots[0] = (uint32_t*)p; p += up((size_t)n * sizeof(uint32_t));
    slots[1] = (uint32_t*)p; p += up((size_t)n * sizeof(uint32_t));
    uint32_t* rng = (uint32_t*)p; p += up((size_t)n * sizeof(uint32_t));
    const RadixSortScratch rs = radix_sort_bind(p, (size_t)n);
    p += up(radix_sort_scratch_bytes((size_t)n));
    Staged sb;
    sb.hit = (int4*)p; p += up((size_t)n * sizeof(int4));
    sb.surf = (float4*)p; p += up(3 * (size_t)n * sizeof(float4));
    sb.so = (float4*)p; p += up(snl * n * sizeof(float4));
    sb.sd = (float4*)p; p += up(snl * n * sizeof(float4));
    sb.sc = (float4*)p; p += up(snl * n * sizeof(float4));
    sb.occ = (int*)p; p += up(snl * n * sizeof(int));
    sb.work = (unsigned long long*)p;
    const int blocks = (n + kWfThreads - 1) / kWfThreads;
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < job.spp && e == cudaSuccess; ++k)
    {
        int cur = 0;
        wf_primary_kernel<<<blocks, kWfThreads, 0, st>>>(cam, job.sample_base + k, rays[cur], keys[cur], slots[cur], rng);
        e = cudaGetLastError();
        if (e == cudaSuccess && job.sort) e = radix_sort_pairs(keys[cur], slots[cur], (size_t)n, 0, 32, rs, st);
        for (int b = 0; b <= job.max_bounces && e == cudaSuccess; ++b)
        {
            const bool last = b == job.max_bounces;
            // counting runs the one-thread-per-ray launch, which counts as it traverses; so do scenes with many
            // lights (the staged launch's per-light buffers grow with them)
            e = staged ? staged_bounce(s, job, n, rays[cur], slots[cur], rays[cur ^ 1], keys[cur ^ 1], slots[cur ^ 1], rng,
                                       last, sb, st)
                       : bounce(s, job.width, job.watertight, job.counters != nullptr, n, rays[cur], slots[cur],
                                job.accum, rays[cur ^ 1], keys[cur ^ 1], slots[cur ^ 1], rng, last, job.counters, st);
            if (last || e != cudaSuccess) break;
            if (job.sort) e = radix_sort_pairs(keys[cur ^ 1], slots[cur ^ 1], (size_t)n, 0, 32, rs, st);
            cur ^= 1;
        }
    }
    return e;
}
}  // namespace lg
