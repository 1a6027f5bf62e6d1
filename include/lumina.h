/* lumina.h -- C ABI of liblumina.so, the B200 render path.
 *
 * Plain C: pointers, sizes and POD structs only.  Every call returns LG_OK (0)
 * or a negative LG_ERR_* status and never exits the process (the reference
 * calls exit(1) on any CUDA error, pathtracer.cu:17-20); lg_last_error()
 * returns the calling thread's last message.
 *
 * Record layouts match the reference's C++ structs byte for byte
 * (include/scene.h:6-56, include/bvh.h:7-16), so a Scene's vectors can be
 * passed straight through.
 *
 * Entry points and the reference interface each one replaces:
 *   lg_scene_load_json      LoadSceneJSON                 src/scene_loader.cpp:26-138
 *   lg_build_bvh            BuildBVH                      src/bvh.cpp:164-211
 *   lg_build_bvh_device     BuildBVH, device-resident in/out
 *   lg_renderer_*, lg_render RenderSceneCUDA              src/pathtracer.cu:581-757
 *   lg_render_sorted        RenderSceneCUDASorted         src/pathtracer.cu:759-909 (cuda_ref --sort)
 *   lg_render_batch         cuda_ref --batch job loop     src/main.cpp:158-190
 *   lg_tonemap_device       tonemap_kernel                src/pathtracer.cu:413-429
 *   lg_look_at              overwrite_camera              src/main.cpp:29-59
 *   lg_write_png            stbi_write_png call sites     src/main.cpp:214-226
 *   lg_unet_*               ml/train.py:37-75 UNet and its Adam/L1 step (ml/train.py:184-201)
 */
#ifndef LUMINA_H
#define LUMINA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LG_OK 0
#define LG_ERR_INVALID (-1)     /* bad argument or scene content */
#define LG_ERR_CUDA (-2)        /* CUDA runtime error (message in lg_last_error) */
#define LG_ERR_IO (-3)          /* file could not be opened / written */
#define LG_ERR_PARSE (-4)       /* malformed scene.json */
#define LG_ERR_NOMEM (-5)       /* host or device allocation failed */
#define LG_ERR_DEVICE (-6)      /* a kernel reported an error flag (stack or queue overflow, wait limit) */
#define LG_ERR_CAPACITY (-7)    /* output buffer too small */

typedef struct { float v[3][3]; float n[3][3]; float uv[3][2]; int32_t material; } lg_triangle;   /* 100 B */
typedef struct { float bbMin[3]; float bbMax[3]; int32_t left, right, firstTri, triCount; } lg_bvh_node; /* 40 B */
typedef struct { float pos[3]; float color[3]; float intensity; float radius; } lg_point_light;
typedef struct { float dir[3]; float color[3]; float intensity; } lg_dir_light;
typedef struct {
    float pos[3];
    float camera_to_world[16]; /* rows 0/1/2 = forward/left/up, row 3 = position */
    float fov_y_deg, aspect, near_z, far_z;
    int32_t width, height;
} lg_camera;

/* A scene as plain arrays (host memory unless a call says otherwise). */
typedef struct {
    lg_camera camera;
    lg_dir_light sun;
    const lg_triangle* tris;
    int32_t n_tris;
    const float* mat_albedo;   /* 3 floats per material */
    const float* mat_emissive; /* 3 floats per material, may be NULL */
    int32_t n_mats;
    const lg_point_light* points;
    int32_t n_points;
    const lg_dir_light* directionals; /* parsed and kept; not used for shading (as in the reference) */
    int32_t n_directionals;
} lg_scene_desc;

const char* lg_last_error(void);
int lg_version(void);

/* ---- scene.json (drop-in for LoadSceneJSON) ---- */
typedef struct lg_scene lg_scene;
/* flags: bit0 = print the reference's "[scene] loaded ..." summary to stdout.
 * threads: host threads for parsing the triangle array (<= 0: all cores).
 * A binary scene file (lg_scene_save_bin; first bytes "LGSCENE1") is
 * recognised by its magic and loaded without text parsing. */
int lg_scene_load_json(const char* path, int flags, int threads, lg_scene** out);
int lg_scene_create(const lg_scene_desc* desc, lg_scene** out); /* deep copy */
int lg_scene_describe(const lg_scene* s, lg_scene_desc* out);   /* pointers stay owned by s */
int lg_scene_set_camera(lg_scene* s, const lg_camera* cam);
int lg_scene_save_json(const lg_scene* s, const char* path);
/* Binary scene file: the scene.json content with every record in its memory
 * layout (Triangle records verbatim), for fast ingest. */
int lg_scene_save_bin(const lg_scene* s, const char* path);
/* Material texture path (may be ""), owned by s. */
const char* lg_scene_texture(const lg_scene* s, int material);
/* Sets a material's texture path (the JSON "diffuse_tex" value). */
int lg_scene_set_texture(lg_scene* s, int material, const char* path);
void lg_scene_destroy(lg_scene* s);

/* ---- images ----
 * lg_image_load: stbi_load(path, &w, &h, &n, 4) as load_texture_to_device
 * uses it (src/pathtracer.cu:553-560), for PNG files (every colour type, bit
 * depth and interlace mode): 8-bit RGBA, top row first.  *rgba8 is released
 * with lg_image_free. */
int lg_image_load(const char* path, int32_t* w, int32_t* h, uint8_t** rgba8);
void lg_image_free(uint8_t* rgba8);

/* overwrite_camera (src/main.cpp:29-59): forward = normalize(target-pos),
 * left = normalize(-fy, fx, 0) (fallback +Y), up = forward x left.
 * Leaves cam unchanged when |target-pos| < 1e-8. */
void lg_look_at(lg_camera* cam, const float pos[3], const float target[3]);

/* ---- BVH (drop-in for BuildBVH) ----
 * Builds on the current CUDA device.  nodes_out must hold max(2*n_tris-1, 1)
 * nodes.  perm_out[i] (optional) = input index of the triangle placed at i;
 * tris_out (optional, may equal tris) receives the reordered triangles.
 * n_tris == 0 gives *n_nodes_out = 0. */
int lg_build_bvh(const lg_triangle* tris, int32_t n_tris, lg_bvh_node* nodes_out, int32_t* n_nodes_out,
                 int32_t* perm_out, lg_triangle* tris_out);
/* Same with device pointers on `stream` (a cudaStream_t, may be NULL).
 * d_tris_out may be NULL.  Scratch is taken from a per-device pool that
 * grows on demand. */
int lg_build_bvh_device(const lg_triangle* d_tris, int32_t n_tris, lg_bvh_node* d_nodes_out, int32_t* n_nodes_out,
                        int32_t* d_perm_out, lg_triangle* d_tris_out, void* stream);

/* No counterpart in the reference.  lg_build_bvh_device for callers that may
 * not allocate device memory (an engine's frame loop that cannot take the
 * synchronisation of cudaMalloc/cudaFree, or a host that reserves all device
 * memory through its own allocator).  Same arguments and results; the
 * scratch is a fixed array in device memory that the library holds on every
 * GPU that loads it, so at most LG_NOALLOC_MAX_TRIS triangles are accepted
 * (larger inputs return LG_ERR_CAPACITY).  The first call on a device looks
 * up the array's address for that device.
 * Under lazy module loading (CUDA's default since 12.2) that first call is
 * also when the array is loaded and its 14 MB are taken from the device, so
 * a host that reserves all device memory for its own allocator should make
 * one call on each device before it does (or set CUDA_MODULE_LOADING=EAGER).
 * Every call synchronises `stream` before it returns: it reads the node count
 * back to the host.  All calls share the one array: calls whose work overlaps
 * on the GPU (other threads, other streams) race and must be serialised by
 * the caller. */
#define LG_NOALLOC_MAX_TRIS 65536
int lg_build_bvh_device_noalloc(const lg_triangle* d_tris, int32_t n_tris, lg_bvh_node* d_nodes_out,
                                int32_t* n_nodes_out, int32_t* d_perm_out, lg_triangle* d_tris_out, void* stream);

/* ---- path tracer ---- */
typedef struct lg_renderer lg_renderer;

#define LG_RENDER_ACCUM64 1u   /* keep an FP64 per-pixel accumulator (judge images) */
#define LG_RENDER_NO_RAY_SORT 2u /* lg_render_sorted only: same launches, rays left in pixel order */

typedef struct {
    int32_t spp;           /* samples per pixel (chunks of 8 share one RNG stream, as in the reference) */
    int32_t max_bounces;
    int32_t sample_base;   /* first sample index (continues a progressive render); normally 0 */
    uint32_t flags;        /* LG_RENDER_* */
} lg_render_opts;

typedef struct {
    float kernel_ms;       /* device time of the trace + tonemap launches */
    /* The rest is filled only while counting is on (lg_renderer_set_counting). */
    uint64_t closest_rays; /* closest-hit rays traced (camera + bounce) */
    uint64_t shadow_rays;  /* shadow rays traced */
    uint64_t node_fetches; /* 64-byte two-child BVH records read */
    uint64_t tri_tests;    /* ray/triangle tests (48 bytes of vertex data each) */
    uint64_t leaf_fetches; /* 8-byte leaf-table entries read */
} lg_render_stats;

int lg_renderer_create(int device, lg_renderer** out);
void lg_renderer_destroy(lg_renderer* r);
/* Upload a scene and build its BVH on the device (triangles are reordered on
 * the device; host arrays are not modified).  Every triangle's material index
 * must lie in [0, n_mats): it is checked on the device after the upload, and
 * a bad one returns LG_ERR_INVALID naming the first such triangle, with the
 * renderer left without a scene (renders then miss everywhere) until the
 * next successful call.  The same holds for lg_renderer_set_scene_bvh. */
int lg_renderer_set_scene(lg_renderer* r, const lg_scene_desc* scene);
/* Upload a scene whose triangles are already in BVH order with its node array. */
int lg_renderer_set_scene_bvh(lg_renderer* r, const lg_scene_desc* scene, const lg_bvh_node* nodes, int32_t n_nodes);
/* Copy back the device BVH (nodes_out may be NULL to query the count). */
int lg_renderer_get_bvh(lg_renderer* r, lg_bvh_node* nodes_out, int32_t* n_nodes, lg_triangle* tris_out);
int lg_renderer_set_counting(lg_renderer* r, int enable);
/* Traversal records: 4 (default; up to four descendants per 64-byte record,
 * their boxes quantized to 8 bits per plane and rounded outwards) or 2 (one
 * binary node per 64-byte record, exact boxes and the reference's slab test).
 * Both traverse the same render tree. */
int lg_renderer_set_bvh_width(lg_renderer* r, int width);
/* The tree the traversal records are built from.  lg_renderer_get_bvh still
 * returns the scene's BuildBVH tree unchanged, and every mode reports hits
 * by BuildBVH's triangle order; any BVH over the same triangles gives the
 * same closest hits (up to exact ties in t).
 * LG_RENDER_TREE_BUILDBVH keeps BuildBVH's Morton-split topology.
 * LG_RENDER_TREE_PLOC regroups BuildBVH's leaves (triangle ranges) by PLOC
 * (Meister and Bittner, HPG 2018): agglomerative clustering by union surface
 * area, on the GPU, which makes traversal open fewer boxes.  A tree PLOC
 * cannot regroup (leaves sharing a first triangle) keeps its own topology.
 * LG_RENDER_TREE_PLOC_TRIANGLES (default) clusters the triangles themselves
 * by PLOC, one triangle per leaf (2T - 1 nodes): tighter leaves, 2.5x fewer
 * triangle tests per ray.
 * get_render_tree reports the mode in use. */
#define LG_RENDER_TREE_BUILDBVH 0
#define LG_RENDER_TREE_PLOC 1
#define LG_RENDER_TREE_PLOC_TRIANGLES 2
int lg_renderer_set_render_tree(lg_renderer* r, int mode);
int lg_renderer_get_render_tree(lg_renderer* r, int32_t* mode_used);
/* Ray/triangle test.  LG_ISECT_MOLLER_TRUMBORE (default) is the reference's
 * ray_tri (src/pathtracer.cu:82-107) and the parity mode.
 * LG_ISECT_WATERTIGHT is the watertight test of Woop, Benthin and Wald (JCGT
 * 2013): no ray passes between triangles that share an edge or a vertex;
 * results differ from the reference on the pixels whose rays graze edges. */
#define LG_ISECT_MOLLER_TRUMBORE 0
#define LG_ISECT_WATERTIGHT 1
int lg_renderer_set_intersection(lg_renderer* r, int mode);
/* Autotuner of the persistent trace launch: renders `cam` at spp/max_bounces
 * with 1..4 resident blocks per SM, keeps the fastest for later frames and
 * reports it (and its kernel time) through the optional outputs. */
int lg_renderer_autotune(lg_renderer* r, const lg_camera* cam, int spp, int max_bounces, int32_t* blocks_per_sm,
                         float* ms);
/* Ray refill of the persistent trace launch.  A warp steps its lanes' ray
 * traversals one BVH record or leaf at a time; once `threshold` of its 32
 * lanes have finished their rays, those lanes shade and start their next
 * ray while the others keep traversing.  32 waits for the whole warp (one
 * warp-wide traversal per path step).  Images do not depend on it. */
#define LG_REFILL_DEFAULT 12
int lg_renderer_set_refill_threshold(lg_renderer* r, int threshold);
int lg_renderer_get_refill_threshold(const lg_renderer* r);
/* Leaf postponement of the persistent trace launch.  A lane that reaches a
 * BVH leaf holds it and keeps visiting records; the warp tests the held
 * leaves together once at most `quorum` of its lanes are still looking for
 * one (0 = all lanes hold a leaf or are done).  Images do not depend on it. */
#define LG_LEAF_QUORUM_DEFAULT 12
int lg_renderer_set_leaf_quorum(lg_renderer* r, int quorum);
int lg_renderer_get_leaf_quorum(const lg_renderer* r);
/* Shared-memory copy of the top of the BVH: each block of the persistent
 * trace launch copies the first `n` 4-wide records (BFS order: the top levels,
 * which every ray visits first) into shared memory at start and reads them
 * from there (64 B each; at most LG_TOP_RECORDS_MAX, 0 = off).  The
 * reference stages its first 255 binary nodes the same way
 * (src/pathtracer.cu:44-50, 338-342).  Images do not depend on it. */
/* Persisting-L2 access window (the reference's CUDAREF_L2_PIN knob,
 * src/pathtracer.cu:675-693): with enable, the renderer's launches mark their
 * accesses to the 4-wide BVH records as persisting in L2 (up to the device's
 * persisting maximum, which this call also sets aside for the process).
 * Images do not depend on it.  The C++ RenderSceneCUDA drop-in turns it on
 * when the environment has CUDAREF_L2_PIN=1, as the reference does. */
int lg_renderer_set_l2_window(lg_renderer* r, int enable);
/* No counterpart in the reference (whose traversal drops pushes past its
 * 64-entry stack without a word, src/pathtracer.cu:142, 184).  The most
 * traversal-stack entries any ray can need over the current scene's records
 * (computed when they are built: per root-to-record path, the sum of each
 * record's children less one) and the stack's capacity.  When the bound fits,
 * frames are traced without per-push checks; otherwise every push is checked
 * and one that does not fit makes the render return LG_ERR_DEVICE. */
int lg_renderer_get_stack_bound(const lg_renderer* r, int32_t* bound, int32_t* capacity);
#define LG_TOP_RECORDS_DEFAULT 0
#define LG_TOP_RECORDS_MAX 1024
int lg_renderer_set_top_records(lg_renderer* r, int n);
int lg_renderer_get_top_records(const lg_renderer* r);
/* Autotuner of the trace schedule: renders `cam` at spp/max_bounces with each
 * pair of refill threshold (8, 12, 16, 24) and leaf quorum (4, 8, 12, 16),
 * keeps the fastest pair for later frames and reports it (and its kernel
 * time) through the optional outputs.  Images do not depend on the choice
 * beyond exact ties. */
int lg_renderer_autotune_schedule(lg_renderer* r, const lg_camera* cam, int spp, int max_bounces,
                                  int32_t* refill, int32_t* quorum, float* ms);
/* Diffuse texture of one material (load_texture_to_device + sample_albedo,
 * src/pathtracer.cu:553-579, 274-282): w x h RGBA8 host pixels, sampled as
 * sRGB with bilinear filtering and wrapping at uv (u, 1 - v).  rgba8 = NULL
 * removes it.  Setting a scene clears every texture. */
int lg_renderer_set_texture(lg_renderer* r, int material, const uint8_t* rgba8, int32_t w, int32_t h);
/* Loads each material's "diffuse_tex" from asset_root + "/" + path
 * (RenderSceneCUDA, src/pathtracer.cu:597-613); files that cannot be read
 * count as missing.  s must be the scene the renderer holds. */
int lg_renderer_load_textures(lg_renderer* r, const lg_scene* s, const char* asset_root, int32_t* loaded,
                              int32_t* missing);
/* Render one frame.  rgb8 (W*H*3 bytes) and accum (W*H*3 floats, sum over
 * samples as RenderSceneCUDA's accumulator) are host buffers; either may be
 * NULL.  accum64 (W*H*3 doubles) requires LG_RENDER_ACCUM64. */
int lg_render(lg_renderer* r, const lg_camera* cam, const lg_render_opts* opts, uint8_t* rgb8, float* accum,
              double* accum64, lg_render_stats* stats);
/* Device-output variant: results stay in device buffers owned by the
 * renderer until the next call; pointers are returned (any may be NULL). */
int lg_render_device(lg_renderer* r, const lg_camera* cam, const lg_render_opts* opts, void* stream,
                     const uint8_t** d_rgb8, const float** d_accum, const double** d_accum64);
/* The reference's ray-sorted render (RenderSceneCUDASorted,
 * src/pathtracer.cu:431-547 and 759-909; the CLI's --sort), with its own
 * estimator: per sample, a camera ray per pixel seeded (px*1973 + py*9277 +
 * (sample_base + sample)*26699) | 1; the rays sorted stably by a 30-bit
 * Morton code of their direction; per bounce every live ray traced, its
 * throughput x direct light (sun and point lights, a shadow ray each) added
 * to its pixel, and its next ray (cosine-weighted, no Russian roulette)
 * sorted again.  Draws after the camera jitter come from the RNG state of
 * the ray's sorted slot, as in the reference, so the sort order is part of
 * the image.  opts->flags may hold LG_RENDER_NO_RAY_SORT (rays stay in pixel
 * order: the same launches without the sorts, a different image of the same
 * estimator).  rgb8 / accum: host buffers as lg_render; stats->kernel_ms is
 * the device time of every launch of the frame. */
int lg_render_sorted(lg_renderer* r, const lg_camera* cam, const lg_render_opts* opts, uint8_t* rgb8, float* accum,
                     lg_render_stats* stats);
/* n_jobs frames (per-job camera, size, spp, bounces, sample_base) traced in
 * ONE persistent launch: the (pixel, chunk of 8 samples) items of all frames
 * share one work counter, so the GPU stays full across frames.  The job-table
 * upload, clears, trace and tonemaps are replayed from a CUDA graph while the
 * frame sizes and spp repeat.  rgb8_out receives the frames one after another
 * (sum of W*H*3 bytes, host).  ms_per_job: the launch's device time
 * apportioned to the frames by work items.  Same images as lg_render per job. */
int lg_render_batch(lg_renderer* r, const lg_camera* cams, const lg_render_opts* opts, int32_t n_jobs,
                    uint8_t* rgb8_out, float* ms_per_job);

/* gbuffer_kernel (src/pathtracer.cu:366-411): primary hit through each pixel
 * centre; albedo, normal*0.5+0.5 and world position normalised by the BVH root
 * box, each W*H*3 bytes (host buffers, any may be NULL).  Misses give albedo 0,
 * normal (128,128,255), position 0. */
int lg_render_gbuffer(lg_renderer* r, const lg_camera* cam, uint8_t* albedo, uint8_t* normal, uint8_t* worldpos);

/* tonemap_kernel: rgb8 = (u8)(sqrt(clamp(accum*inv_spp, 0, 1)) * 255). */
int lg_tonemap_device(const float* d_accum, uint8_t* d_rgb8, int64_t n_pixels, float inv_spp, void* stream);

/* ---- denoiser (reference ml/train.py:37-75 UNet, 3- or 12-channel in / 3-channel out) ----
 * BF16 tcgen05 convolutions with FP32 accumulation; FP32 master parameters in
 * the reference's state_dict order (d1.net.0.weight, d1.net.0.bias,
 * d1.net.2.weight, ..., u1.net.2.bias, tail.weight, tail.bias).  base must be
 * 32; in_ch is 3 (the reference's default) or up to 16 -- 12 is train.py's
 * --gbuffer variant, colour + albedo + normal + position stacked as channels
 * (train.py:112-119); the residual uses x[:, :3].  Images are FP32 NCHW; H
 * and W must be multiples of 8 (tools/denoise.py pads before calling the model).
 * mode 0 is the reference network: LeakyReLU(0.1), nearest upsampling, input
 * in [0,1], out = clamp(x[:, :3] + tail, 0, 1).  Mode bits select the
 * configuration-4 variant the reference does not ship:
 *   LG_UNET_RELU      ReLU activations;
 *   LG_UNET_BILINEAR  bilinear 2x upsampling (align_corners=False);
 *   LG_UNET_LOG_HDR   HDR radiance in and out: the network sees log1p(x), the
 *                     residual is taken in log space, out = expm1(max(y, 0));
 *                     its training loss is L1 between max(y, 0) and log1p(target).
 * LG_UNET_HDR_VARIANT = all three. */
#define LG_UNET_RELU 1
#define LG_UNET_BILINEAR 2
#define LG_UNET_LOG_HDR 4
#define LG_UNET_HDR_VARIANT 7
typedef struct lg_unet lg_unet;
int lg_unet_create(int base, int in_ch, int mode, lg_unet** out);
void lg_unet_destroy(lg_unet* u);
int64_t lg_unet_num_params(const lg_unet* u);
int lg_unet_set_params(lg_unet* u, const float* params, int64_t n);
int lg_unet_get_params(lg_unet* u, float* params, int64_t n);
/* y = clamp(x[:, :3] + tail(...), 0, 1) (mode 0); host buffers, x n*in_ch*h*w and y n*3*h*w floats. */
int lg_unet_forward(lg_unet* u, const float* x, int n, int h, int w, float* y);
/* Same on device buffers, ordered on `stream` (a cudaStream_t; NULL = synchronous). */
int lg_unet_forward_device(lg_unet* u, const float* d_x, int n, int h, int w, float* d_y, void* stream);
/* Training (reference ml/train.py:184-201): mean L1 loss of the network output
 * against target, backward pass on the tensor cores, and one Adam step
 * (betas 0.9/0.999, eps 1e-8, bias correction, as torch.optim.Adam) on the
 * FP32 master parameters.  d_x: device FP32 NCHW n x in_ch x h x w;
 * d_target: n x 3 x h x w.
 * *loss_out (may be NULL) receives the loss before the update. */
int lg_unet_train_step(lg_unet* u, const float* d_x, const float* d_target, int n, int h, int w, float lr,
                       float* loss_out);
/* The same step queued behind the work already on `stream` (the caller's
 * CUDA stream; the batch buffers may be written there just before), with
 * later work on `stream` ordered after it, and without waiting for the
 * device: a training loop runs ahead of the GPU instead of stopping twice
 * per step.  n times the batch's mean L1 loss is added to *d_loss_sum (a
 * device float, may be NULL), so summing over an epoch's batches gives the
 * loss summed over its images.  A wait timeout inside the step is reported
 * by the next call that waits for the device (lg_unet_sync,
 * lg_unet_train_step, lg_unet_loss_grad). */
int lg_unet_train_step_async(lg_unet* u, const float* d_x, const float* d_target, int n, int h, int w, float lr,
                             float* d_loss_sum, void* stream);
/* Waits for every step queued on the network; LG_ERR_DEVICE if one of its
 * tensor-core kernels gave up a wait. */
int lg_unet_sync(lg_unet* u);
/* The loss and the gradient of every parameter (host, state_dict order)
 * without updating them. */
int lg_unet_loss_grad(lg_unet* u, const float* d_x, const float* d_target, int n, int h, int w, float* grads,
                      float* loss_out);
/* One Adam step with the gradients of the last lg_unet_loss_grad call. */
int lg_unet_adam_apply(lg_unet* u, float lr);
/* Clears the Adam moments and step count. */
int lg_unet_adam_reset(lg_unet* u);
/* No counterpart in the reference (which calls exit(1) on any CUDA error,
 * src/pathtracer.cu:17-20).  Checks the failure path of the tensor-core
 * kernels: a probe kernel waits, with the same bounded wait they use, on an
 * mbarrier that nothing arrives at; after limit_ns (1 us .. 2 s) it sets the
 * network's error word as a convolution whose wait ran out would, and the
 * call returns LG_ERR_DEVICE ("... wait timeout 3").  Nothing is left in
 * flight, so the network stays usable: the next call clears the word. */
int lg_unet_wait_selftest(lg_unet* u, int64_t limit_ns);
/* Autotuner: for each of the 14 convolutions (and, with
 * LG_UNET_TUNE_BACKWARD, the 16 input-gradient convolutions of training)
 * times every compiled tile shape (output channels per CTA, input channels
 * per K-block, pipeline stages) with each of the kernels (0: one tile per
 * CTA; 1: persistent and warp-specialised; 2: persistent with the layer's
 * weights resident in shared memory, for layers with one output block whose
 * weights fit beside the pipeline; 3: as 2 on 4-row tiles; 4: as 3 with the
 * three row taps of each column tap packed side by side into one MMA's N,
 * for 32 and 64 output channels, input tiles loaded in 8-pixel runs; 5: as 4
 * on 8-row tiles; 6 and 7: packed row taps with the weights streamed, 4- and
 * 8-row tiles; all give bit-identical results)
 * inside real passes at n x h x w and keeps the fastest; weights are
 * repacked to match.  tiles_out (may be NULL)
 * receives 30 (bn, kc, stages, kernel) quadruples, forward layers first.
 * The Adam state is reset.  Until then (or lg_unet_set_tiles) the forward
 * convolutions use the choice this autotuner made at batch 8, 1728x864 on
 * B200, and the input-gradient convolutions a per-shape default. */
#define LG_UNET_TUNE_BACKWARD 1
int lg_unet_autotune(lg_unet* u, int n, int h, int w, int flags, int32_t* tiles_out);
/* Sets the 30 tile choices directly, in lg_unet_autotune's format; e.g. to
 * reuse a tuning result without timing.  (0, 0, 0, p) is the default shape on
 * the kernel p selects (0: one tile per CTA, 1: persistent; 2 only with an
 * explicit shape compiled for it). */
int lg_unet_set_tiles(lg_unet* u, const int32_t* tiles);
/* Folded upsampling (on by default): in inference passes of a network with
 * nearest upsampling, u3a, u2a and u1a read the upsampled half of their input
 * as the lower level's output repeated along x only, and sum the row taps
 * that meet the same low-resolution row (even output rows: ky1 + ky2, odd:
 * ky0 + ky1), where their tile has that form (kernel choices 6 and 7 with at
 * most 64 output channels per CTA).  Same network function; the folded
 * weights are rounded to BF16 after the sum, so outputs differ from the
 * unfolded pass by BF16 rounding.  Training passes never fold.  on = 0 turns
 * it off (e.g. to compare against the unfolded pass). */
int lg_unet_set_fold_upsampling(lg_unet* u, int on);
/* One 3x3 convolution layer on device buffers in the channel-blocked BF16
 * layout ((n*C/8 + c/8)*H + y)*W + x)*8 + c%8: epilogue 0 writes act(conv+b)
 * into channels [out_coff, out_coff+cout) of d_out (and, if d_out2, the 2x2
 * max-pooled result into d_out2); epilogue 1 writes it 2x upsampled (nearest).
 * Weights are FP32 [cout][cin_real][3][3]; cin >= cin_real is the blocked
 * input's channel count (multiple of 16). */
int lg_conv3x3_device(const void* d_in, int n, int cin, int h, int w, const float* d_w, int cin_real,
                      const float* d_b, int cout, float slope, int epilogue, void* d_out, int out_c, int out_coff,
                      void* d_out2, int out2_c, int out2_coff, void* stream);
/* FP32 NCHW <-> channel-blocked BF16 (cpad channels, zero padded). */
int lg_to_blocked_bf16(const float* d_x, int n, int c, int h, int w, void* d_out, int cpad, void* stream);
int lg_from_blocked_bf16(const void* d_in, int n, int c, int h, int w, float* d_out, void* stream);

/* ---- image plumbing between renderer and denoiser (device buffers) ---- */
/* n frames of h*w*3 bytes (HWC) -> FP32 NCHW u8/255 (ml/train.py:102-103). */
int lg_rgb8_to_f32(const uint8_t* d_rgb, int n, int h, int w, float* d_out, void* stream);
/* FP32 NCHW -> h*w*3 bytes per frame: (u8)(clip(v,0,1)*255 + 0.5) (tools/denoise.py:51). */
int lg_f32_to_rgb8(const float* d_in, int n, int h, int w, uint8_t* d_rgb, void* stream);
/* n accumulators (h*w*3 sums over samples, HWC) * inv_spp -> FP32 NCHW linear
 * radiance (the HDR denoiser's input). */
int lg_accum_to_f32(const float* d_accum, int n, int h, int w, float inv_spp, float* d_out, void* stream);
/* FP32 NCHW linear radiance -> h*w*3 bytes (HWC) with tonemap_kernel's formula
 * (u8)(sqrt(clamp(v, 0, 1)) * 255). */
int lg_f32_tonemap_rgb8(const float* d_in, int n, int h, int w, uint8_t* d_rgb, void* stream);
/* n_crops square crops (crop x crop, all 3 channels) of FP32 NCHW images
 * (n_images x 3 x h x w) at host-given (img_idx, ys, xs) into d_out
 * (n_crops x 3 x crop x crop).  With stream NULL the call returns when the
 * crops are written; with a stream it only queues the copy there. */
int lg_gather_crops(const float* d_images, int n_images, int h, int w, const int32_t* img_idx, const int32_t* ys,
                    const int32_t* xs, int n_crops, int crop, float* d_out, void* stream);

/* ---- measurement ----
 * No counterpart in the reference.  Read bandwidth of one memory level on
 * `device`, in GB/s, for roofline denominators: level 2 reads a `bytes`
 * buffer (choose one that fits in L2) `passes` times with L2-only loads;
 * level 1 has every block read the same `bytes` region (at most 48 KB)
 * `passes` times through the read-only L1 path.  Allocates and frees its
 * own buffers; synchronous. */
int lg_measure_read_bandwidth(int device, int level, int64_t bytes, int passes, double* gbs);

/* ---- image output ---- */
int lg_write_png(const char* path, int32_t w, int32_t h, const uint8_t* rgb8);
int lg_write_hdr(const char* path, int32_t w, int32_t h, const float* rgb32);

#ifdef __cplusplus
}
#endif
#endif
