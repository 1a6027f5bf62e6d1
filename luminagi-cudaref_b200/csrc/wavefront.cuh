// wavefront.cuh -- the ray-sorted render (see wavefront.cu).
#pragma once
#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "trace.cuh"

namespace lg
{
// One ray of the wavefront, 48 bytes: origin (w = pixel index bits),
// direction (w = 1 alive / 0 dead), throughput.
struct alignas(16) WfRay
{
    float4 o, d, thr;
};
static_assert(sizeof(WfRay) == 48, "WfRay is three float4s");

struct WavefrontJob
{
    int spp, max_bounces, sample_base;
    bool sort;                 // false: rays stay in pixel order (the same launches without the sorts)
    int width;                 // traversal records: 4 or 2
    bool watertight;
    float* accum;              // W*H*3, added to
    RenderCounters* counters;  // optional: counts rays and record/triangle visits (one-thread-per-ray launches)
    // the staged launches (when not counting): persistent traversal grid and schedule
    int sm_count;
    int refill;                // idle lanes of a warp that trigger a refill from the ray list, 1..32 (8)
    int quorum;                // leaf postponement quorum, as for the persistent trace kernel
    bool stack_safe;           // the records' stack bound fits: traversal without push checks
};

// Device scratch for a frame of n_pixels with n_lights lights (the sun and
// the point lights): two ray buffers, keys, slots, RNG states, the radix
// sort's buffers, and the staged bounce's hits, surfaces, shadow rays and
// occlusion flags.
size_t wavefront_scratch_bytes(int n_pixels, int n_lights);

// Queues every launch of one frame on `stream`: per sample, camera rays,
// sort, then per bounce a trace launch and a sort of the next rays.
cudaError_t launch_wavefront_frame(const DevScene& s, const DevCam& cam, const WavefrontJob& job, void* scratch,
                                   size_t scratch_bytes, cudaStream_t stream);
}  // namespace lg
