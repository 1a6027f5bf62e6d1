/* lgoracle.h -- TEST INFRASTRUCTURE ONLY: the CPU oracle's C interface.
 *
 * Plain-C restatement of the reference render path (LuminaGI-CudaRef
 * src/bvh.cpp and src/pathtracer.cu).  Used by tests/ and bench.py's CPU
 * baseline as the checker; never linked into the product library.
 * Parity pinned against the reference's own sources compiled in
 * oracle/_ref/libref.so (tests/test_oracle.py).
 */
#ifndef LGORACLE_H
#define LGORACLE_H
#include <stdint.h>

typedef struct { float v[3][3]; float n[3][3]; float uv[3][2]; int material; } lgo_tri;        /* 100 B */
typedef struct { float bbMin[3]; float bbMax[3]; int left, right, firstTri, triCount; } lgo_node; /* 40 B */
typedef struct { float pos[3]; float color[3]; float intensity; float radius; } lgo_point;
typedef struct { float dir[3]; float color[3]; float intensity; } lgo_dir;
typedef struct {
    float pos[3]; float cameraToWorld[16]; float fovYDeg, aspect, nearZ, farZ; int imageWidth, imageHeight;
} lgo_camera;

/* Ray counters gathered while tracing. */
typedef struct {
    uint64_t closest_rays;  /* closest-hit rays (camera + bounce) */
    uint64_t shadow_rays;   /* shadow rays actually traced */
    uint64_t node_visits;   /* BVH nodes popped and box-tested */
    uint64_t tri_tests;     /* ray/triangle tests */
} lgo_counters;

/* BVH build; returns the node count (<= 2n-1).  perm[i] = original index of
 * the triangle at sorted position i (ties in Morton code broken by original
 * index).  tris_out receives the reordered triangles; codes_out (optional)
 * the sorted Morton codes. */
int lgo_build_bvh(const lgo_tri* tris, int n, lgo_node* nodes_out, int* perm, lgo_tri* tris_out, uint32_t* codes_out);

/* Morton code of one triangle given the scene bounds (bvh.cpp:185-191). */
uint32_t lgo_morton_of(const lgo_tri* t, const float scene_min[3], const float ext[3]);
void lgo_scene_bounds(const lgo_tri* tris, int n, float mn[3], float ext[3]);

/* Per-pixel accumulate over rows row_start, row_start+row_step, ...
 * accum (W*H*3) is added to.  counters may be NULL. */
int lgo_render(const lgo_node* nodes, const lgo_tri* tris, const float* mat_albedo, int n_mats,
               const lgo_point* points, int n_points, const lgo_dir* sun, const lgo_camera* cam, int spp,
               int max_bounces, int row_start, int row_step, int threads, float* accum, lgo_counters* counters);

/* accumulate_kernel's tonemap (pathtracer.cu:413-429). */
void lgo_tonemap(const float* accum, uint8_t* rgb, int n_pixels, float inv_spp);

#endif
