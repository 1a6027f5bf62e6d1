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
}  // namespace

size_t wavefront_scratch_bytes(int n_pixels)
{
    const size_t n = (size_t)(n_pixels > 0 ? n_pixels : 1);
    const size_t a = 256;
    auto up = [&](size_t b) { return (b + a - 1) / a * a; };
    return 2 * up(n * sizeof(WfRay)) + 5 * up(n * sizeof(uint32_t)) + up(radix_sort_scratch_bytes(n)) + a;
}

cudaError_t launch_wavefront_frame(const DevScene& s, const DevCam& cam, const WavefrontJob& job, void* scratch,
                                   size_t scratch_bytes, cudaStream_t st)
{
    const int n = cam.width * cam.height;
    if (n <= 0 || job.spp <= 0) return cudaSuccess;
    if (scratch_bytes < wavefront_scratch_bytes(n)) return cudaErrorInvalidValue;
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
            e = bounce(s, job.width, job.watertight, job.counters != nullptr, n, rays[cur], slots[cur], job.accum,
                       rays[cur ^ 1], keys[cur ^ 1], slots[cur ^ 1], rng, last, job.counters, st);
            if (last || e != cudaSuccess) break;
            if (job.sort) e = radix_sort_pairs(keys[cur ^ 1], slots[cur ^ 1], (size_t)n, 0, 32, rs, st);
            cur ^= 1;
        }
    }
    return e;
}
}  // namespace lg
