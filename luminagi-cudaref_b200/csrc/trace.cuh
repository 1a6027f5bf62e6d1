// trace.cuh -- device scene layout and launchers of the path tracer.
#pragma once
#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "lumina.h"
#include "vecmath.h"

namespace lg
{
// One record per internal BVH node holding both children's boxes (64 B,
// four 16-byte loads).  Child links: >= 0 internal record index, < 0 leaf
// ~index into the leaf table.
struct alignas(16) WideNode
{
    float4 xy0;  // child 0: min.x, max.x, min.y, max.y
    float4 xy1;  // child 1: min.x, max.x, min.y, max.y
    float4 z01;  // child 0 min.z, max.z, child 1 min.z, max.z
    int4 link;   // link0, link1, unused, unused
};
static_assert(sizeof(WideNode) == 64, "WideNode is one 64-byte record");

// A 4-wide record: up to four children of a render-tree node, their boxes
// quantized to 8 bits per plane on a per-record grid (64 B, two 32-byte
// loads).  Per axis a the grid has origin o[a] and a power-of-two step
// step[a]; child k's min plane is o[a] + q * step[a] for q = byte k of
// qlo[a], its max plane likewise from qhi[a].  Quantized planes lie at least
// one step outside the child's exact box, so every ray that enters the exact
// box enters the quantized one.  An absent child has qlo = 255, qhi = 0 (an
// inverted box) and a link to an empty leaf, so even a test that let it
// through costs one visit of a leaf with no triangles.  Links as in WideNode.
struct alignas(32) Wide4Node
{
    float o[3];
    float step[3];
    uint32_t qlo[3];
    uint32_t qhi[3];
    int link[4];
};
static_assert(sizeof(Wide4Node) == 64, "Wide4Node is two 32-byte halves");

// Intersection record of one triangle: kTriVec float4s, v0 (w = material
// bits), e1 = v1 - v0, e2 = v2 - v0 (v0, v1, v2 in watertight mode), then
// padding, so a record starts on a 32-byte boundary when kTriVec == 4.
constexpr int kTriVec = 4;

// Entries of a ray's traversal stack (per thread, local memory; entries a
// traversal does not reach cost nothing).
constexpr int kTraceStack = 96;

struct DevScene
{
    const Wide4Node* nodes4;   // 4-wide records (used when width == 4)
    int root4;
    int n4;                    // number of 4-wide records
    int leaf_inline;           // 4-wide leaf links carry (first, count); see wide4_kernel
    const WideNode* nodes;
    const int2* leaves;        // (first triangle, count)
    const float4* tv;          // kTriVec per triangle: v0 (w = material bits), e1 = v1-v0, e2 = v2-v0
    const lg_triangle* tris;   // shading data (normals), BVH order
    const float4* mats;        // albedo
    const unsigned long long* texs;  // per material: diffuse texture object or 0; nullptr when none is set
    const lg_point_light* points;
    int n_points;
    int root;                  // root link (0 = internal record 0, < 0 = leaf)
    lg_dir_light sun;
    // Set to 1 by any traversal that had to drop a stack push (the tree is
    // deeper than the stack allows and the image would be incomplete).  It
    // stays set until the host reads and clears it; the store only runs on
    // overflow, so the check costs nothing otherwise.
    unsigned* fault;
};

struct DevCam
{
    vec3 pos, fwd, left, up;
    float tanHalfFov, aspect;
    int width, height;
};

struct RenderCounters
{
    unsigned long long closest_rays;
    unsigned long long shadow_rays;
    unsigned long long stack_overflows;
    unsigned long long node_fetches;  // WideNode records read (64 B each)
    unsigned long long tri_tests;     // ray/triangle tests (48 B of v0/e1/e2 each)
    unsigned long long leaf_fetches;  // leaf-table entries read (8 B each)
};

// One frame of a batched launch: its camera and sampling, its accumulator,
// and the number of the first of its (pixel, chunk) work items, which follow
// the previous job's.
struct BatchJob
{
    DevCam cam;
    unsigned long long item_begin;
    float* accum;  // W*H*3, added to
    int spp, max_bounces, sample_base, n_chunks, tiles_x, n_tiles;
};

struct TraceJob
{
    int spp, max_bounces, sample_base;
    int n_chunks;          // ceil(spp / 8)
    int tiles_x, n_tiles;  // 8 x 4 pixel tiles
    float* accum;          // W*H*3, added to
    double* accum64;       // optional
    unsigned long long* work64;  // work counter (zeroed by the launcher)
    int blocks_per_sm;     // persistent grid: resident blocks per SM (0 = as many as fit)
    int refill_threshold;  // finished rays in a warp that trigger the path logic, 1..32
    int leaf_quorum;       // lanes still searching for a leaf below which the warp tests held leaves, 0..31
    int top_records;       // 4-wide records (the first in BFS order) each block keeps in shared memory, 0 = none
    int stack_safe;        // 1: the records' stack bound fits kTraceStack, launch without push checks
    RenderCounters* counters;  // optional
    // batched launch (launch_trace_batch): every field above except work64 is taken from jobs[]
    const BatchJob* jobs;
    int n_jobs;
    unsigned long long total_items;
};

// Camera set-up of RenderSceneCUDA (pathtracer.cu:654-663); tanf runs on the host as there.
DevCam make_dev_cam(const lg_camera& c);

// Converts the reference node array (BFS) to WideNode records + leaf table.
// Scratch: 2 * n_nodes ints.  Returns the root link through *root (device
// write of one int; caller copies back) -- done inside the launcher.
cudaError_t build_wide_nodes(const lg_bvh_node* d_nodes, int n_nodes, WideNode* d_wide, int2* d_leaves,
                             int* d_scratch, int* root_host, int* n_internal_host, int* n_leaves_host,
                             cudaStream_t stream);
// Collapses the binary BVH (BFS order) into 4-wide records, top-down: a
// record starts from its node's two children and repeatedly opens the
// internal child of largest surface area until it has four; the internal
// children are the next records.  Records are numbered by the BFS rank of
// their nodes (deterministic).  Must follow build_wide_nodes on the same
// scratch (it reuses the leaf numbering).  Scratch: 11 * n_nodes + 256 ints.
// null_leaf: the index of a leaf-table entry (0, 0) for absent children.
// stack4_host / stack2_host: the most traversal-stack entries any ray can
// need over the 4-wide records (the largest sum, over a root-to-record path,
// of each record's child count less one: a visit stacks at most the hit
// children it does not enter, and entries above a popped one are gone) and
// over the 2-wide ones (the deepest internal node's depth + 1).
cudaError_t build_wide4_nodes(const lg_bvh_node* d_nodes, int n_nodes, int n_tris, int null_leaf, Wide4Node* d_wide4,
                              int* d_scratch, int* root4_host, int* n4_host, int* leaf_inline_host,
                              int* stack4_host, int* stack2_host, cudaStream_t stream);
// Intersection records, 3 float4 per triangle (w of the first = material):
// (v0, v1-v0, v2-v0) for Moller-Trumbore, (v0, v1, v2) for the watertight test.
cudaError_t prepare_triangles(const lg_triangle* d_tris, int n, float4* d_tv, bool watertight, cudaStream_t stream);

cudaError_t launch_trace(const DevScene& s, const DevCam& cam, const TraceJob& job, bool count, int sm_count,
                         int width, bool watertight, cudaStream_t stream);
// Several frames (cameras, spp, bounces) in one persistent launch; job.jobs
// (device) describes them, job.work64 is the shared work counter.
cudaError_t launch_trace_batch(const DevScene& s, const TraceJob& job, int sm_count, int width, bool watertight,
                               cudaStream_t stream);
// Primary-hit G-buffer (albedo, encoded normal, box-normalised position), W*H*3 bytes each.
cudaError_t launch_gbuffer(const DevScene& s, const DevCam& cam, vec3 bbMin, vec3 bbInvExtent, uint8_t* d_albedo,
                           uint8_t* d_normal, uint8_t* d_worldpos, int width, bool watertight, cudaStream_t stream);
cudaError_t launch_tonemap(const float* d_accum, uint8_t* d_rgb, long long n_values, float inv_spp,
                           cudaStream_t stream);
cudaError_t launch_accum64_to_32(const double* d_acc64, float* d_acc32, long long n_values, cudaStream_t stream);
}  // namespace lg
