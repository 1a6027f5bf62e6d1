// capi.cu -- the extern "C" boundary (include/lumina.h) and the C++ drop-ins
// BuildBVH (include/bvh.h) and RenderSceneCUDA (reference pathtracer.cu:581-757).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "bvh.h"
#include "common.h"
#include "lbvh.cuh"
#include "render_tree.cuh"
#include "scene.h"
#include "trace.cuh"
#include "wavefront.cuh"

namespace lg
{
bool load_scene_file(const std::string& path, Scene& out, bool verbose, int threads, std::string& err);
bool save_scene_file(const Scene& sc, const std::string& path, int threads);
bool save_scene_bin(const Scene& sc, const std::string& path);
bool write_png(const char* path, int w, int h, const uint8_t* rgb);
bool write_hdr(const char* path, int w, int h, const float* rgb);
bool decode_png(const char* path, int& w, int& h, std::vector<uint8_t>& rgba, std::string& err);

namespace
{
thread_local std::string g_err;
}

int set_error(int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}
void clear_error() { g_err.clear(); }

// Growable device buffer.
struct DevBuf
{
    void* p = nullptr;
    size_t bytes = 0;
    int reserve(size_t b)
    {
        if (b <= bytes) return LG_OK;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess)
        {
            p = nullptr;
            return set_error(LG_ERR_NOMEM, "cudaMalloc(%zu): %s", b, cudaGetErrorString(e));
        }
        bytes = b;
        return LG_OK;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T>
    T* as() const { return (T*)p; }
};

// Per-device scratch for the pointer-level BVH entry points.
struct DeviceScratch
{
    std::mutex mu;
    DevBuf buf;
};
DeviceScratch& device_scratch(int dev)
{
    static DeviceScratch pool[64];
    return pool[dev & 63];
}

// Lowest index of a triangle whose material index is outside [0, n_mats) into *first_bad (atomic minimum).
__global__ void material_check_kernel(const lg_triangle* __restrict__ t, int n, int n_mats, int* __restrict__ first_bad)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int m = t[i].material;
    if (m < 0 || m >= n_mats) atomicMin(first_bad, i);
}
}  // namespace lg

using namespace lg;

struct lg_scene
{
    Scene s;
    std::vector<float> albedo, emissive;  // flattened views for lg_scene_describe
};

struct lg_renderer
{
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool counting = false;
    // scene
    int n_tris = 0, n_nodes = 0, n_mats = 0, n_points = 0, root = 0, root4 = 0;
    int bvh_width = 4;  // traversal records: 4-wide (default) or the 2-wide form
    int leaf_inline = 0;  // 4-wide leaf links carry (first, count)
    int tree_mode = LG_RENDER_TREE_PLOC_TRIANGLES;  // tree the traversal records are built from
    int tree_used = -1;                   // the mode actually built (PLOC falls back to the BuildBVH tree)
    DevBuf rnodes, rt_scratch;            // render tree (depth order) and its build scratch
    bool watertight = false;  // ray/triangle test: Moller-Trumbore (the reference's) or watertight
    int trace_blocks_per_sm = 0;  // persistent trace grid (0 = occupancy maximum); see lg_renderer_autotune
    int trace_refill = LG_REFILL_DEFAULT;  // finished rays per warp that trigger the path logic (1..32)
    int trace_quorum = LG_LEAF_QUORUM_DEFAULT;  // searching lanes below which a warp tests its held leaves (0..31)
    int trace_top = LG_TOP_RECORDS_DEFAULT;     // 4-wide records each trace block keeps in shared memory
    int n4 = 0;                                 // 4-wide records of the current scene
    int stack4 = 1 << 30, stack2 = 1 << 30;     // traversal-stack bounds of the records (build_wide4_nodes)
    bool l2_window = false;                     // persisting-L2 access window over the 4-wide records
    lg_bvh_node root_node{};  // host copy of the BVH root (scene box for the G-buffer)
    DevBuf gbuf;              // G-buffer images (3 x W*H*3 bytes)
    // Traversal-stack overflow word (DevScene::fault) and its pinned host
    // copy, refreshed by an asynchronous copy after every trace launch.
    DevBuf fault;
    unsigned* fault_host = nullptr;
    DevBuf matchk;  // first triangle with a material index outside [0, n_mats), checked on the device
    DevBuf wf_scratch;  // ray-sorted render: rays, keys, slots, RNG states, sort buffers
    // diffuse textures, per material (load_texture_to_device, pathtracer.cu:553-579)
    std::vector<cudaArray_t> tex_arrays;
    std::vector<unsigned long long> tex_objs;  // cudaTextureObject_t, 0 = untextured
    DevBuf texs;                               // device copy of tex_objs
    int n_textured = 0;
    lg_dir_light sun{};
    DevBuf tris, tris_in, nodes, wide, wide4, leaves, tv, mats, points, scratch;
    // frame
    DevBuf accum, accum64, rgb, work, counters;
    int fw = 0, fh = 0;
    // batched launches: job table (pinned host copy + device), frames, and the
    // CUDA graph of the last batch shape (job table upload, clears, trace, tonemaps)
    DevBuf batch_jobs, batch_acc, batch_rgb;
    BatchJob* batch_host = nullptr;
    int batch_host_cap = 0;
    cudaGraphExec_t batch_exec = nullptr;
    std::vector<long long> batch_key;
    long long scene_gen = 0;  // bumped by every change a captured launch depends on
};

namespace
{
struct DeviceGuard
{
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

int apply_l2_window(lg_renderer* r);

int validate_scene(const lg_scene_desc* d)
{
    if (!d) return set_error(LG_ERR_INVALID, "scene is NULL");
    if (d->n_tris < 0 || d->n_mats < 0 || d->n_points < 0) return set_error(LG_ERR_INVALID, "negative count");
    if (d->n_tris > 0 && !d->tris) return set_error(LG_ERR_INVALID, "tris is NULL");
    if (d->n_mats > 0 && !d->mat_albedo) return set_error(LG_ERR_INVALID, "mat_albedo is NULL");
    if (d->n_points > 0 && !d->points) return set_error(LG_ERR_INVALID, "points is NULL");
    // material indices are checked on the device after the upload (check_materials): a host loop over the
    // 100-byte records touches the whole array, 105 MB at 1.05M triangles, about 10 ms of one core
    return LG_OK;
}

// Queues the check of the uploaded triangles' material indices (d_tris, device).
int queue_material_check(lg_renderer* r, const lg_triangle* d_tris, int n, int n_mats)
{
    LG_TRY(r->matchk.reserve(256));
    LG_TRY_CUDA(cudaMemsetAsync(r->matchk.p, 0x7f, sizeof(int), r->stream));  // 0x7f7f7f7f: none
    if (n > 0)
    {
        material_check_kernel<<<(n + 255) / 256, 256, 0, r->stream>>>(d_tris, n, n_mats, (int*)r->matchk.p);
        LG_TRY_CUDA(cudaGetLastError());
    }
    return LG_OK;
}

// After the scene's set-up: a bad material index leaves the renderer without a scene and is reported with the
// caller's triangle (host copy d).
int take_material_check(lg_renderer* r, const lg_scene_desc* d)
{
    int first = 0;
    LG_TRY_CUDA(cudaMemcpyAsync(&first, r->matchk.p, sizeof(int), cudaMemcpyDeviceToHost, r->stream));
    LG_TRY_CUDA(cudaStreamSynchronize(r->stream));
    if (first >= 0 && first < d->n_tris)
    {
        r->n_tris = 0;
        r->n_nodes = 0;
        r->root = 0;
        return set_error(LG_ERR_INVALID, "triangle %d has material %d outside [0,%d)", first, d->tris[first].material,
                         d->n_mats);
    }
    return LG_OK;
}

void clear_textures(lg_renderer* r)
{
    for (unsigned long long t : r->tex_objs)
        if (t) cudaDestroyTextureObject((cudaTextureObject_t)t);
    for (cudaArray_t a : r->tex_arrays)
        if (a) cudaFreeArray(a);
    r->tex_objs.assign((size_t)r->n_mats, 0ull);
    r->tex_arrays.assign((size_t)r->n_mats, nullptr);
    r->n_textured = 0;
}

int upload_common(lg_renderer* r, const lg_scene_desc* d)
{
    if (r->stream) cudaStreamSynchronize(r->stream);
    r->n_mats = d->n_mats;
    ++r->scene_gen;
    clear_textures(r);  // a new scene starts untextured
    r->n_points = d->n_points;
    r->sun = d->sun;
    std::vector<float4> m((size_t)std::max(d->n_mats, 1));
    for (int i = 0; i < d->n_mats; ++i)
        m[(size_t)i] = make_float4(d->mat_albedo[3 * i], d->mat_albedo[3 * i + 1], d->mat_albedo[3 * i + 2], 0.0f);
    LG_TRY(r->mats.reserve(m.size() * sizeof(float4)));
    LG_TRY_CUDA(cudaMemcpyAsync(r->mats.p, m.data(), m.size() * sizeof(float4), cudaMemcpyHostToDevice, r->stream));
    LG_TRY(r->points.reserve((size_t)std::max(d->n_points, 1) * sizeof(lg_point_light)));
    if (d->n_points)
        LG_TRY_CUDA(cudaMemcpyAsync(r->points.p, d->points, (size_t)d->n_points * sizeof(lg_point_light),
                                    cudaMemcpyHostToDevice, r->stream));
    return LG_OK;
}

// Traversal records (2- and 4-wide) from the render tree tree_mode selects
// (render_tree.cu): PLOC over the triangles, PLOC over the BuildBVH tree's
// leaves, or that tree itself.
int build_records(lg_renderer* r)
{
    const int nbvh = r->n_nodes;
    const size_t cap = std::max((size_t)nbvh, 2 * (size_t)r->n_tris);  // nodes of any render tree
    LG_TRY(r->wide.reserve(cap * sizeof(WideNode)));
    LG_TRY(r->leaves.reserve((cap + 1) * sizeof(int2)));  // + the empty leaf of absent 4-wide children
    LG_TRY(r->rnodes.reserve(cap * sizeof(lg_bvh_node)));
    LG_TRY(r->rt_scratch.reserve(render_tree_scratch_bytes(nbvh, r->n_tris)));
    int mode = r->tree_mode;
    int rc = build_render_tree(r->nodes.as<lg_bvh_node>(), nbvh, r->tris.as<lg_triangle>(), r->n_tris, mode,
                               r->rnodes.as<lg_bvh_node>(), r->rt_scratch.p, r->rt_scratch.bytes, r->stream);
    if (rc != LG_OK && mode != LG_RENDER_TREE_BUILDBVH)
    {
        // e.g. leaves whose triangle ranges share a first triangle: keep the given topology
        mode = LG_RENDER_TREE_BUILDBVH;
        rc = build_render_tree(r->nodes.as<lg_bvh_node>(), nbvh, r->tris.as<lg_triangle>(), r->n_tris, mode,
                               r->rnodes.as<lg_bvh_node>(), r->rt_scratch.p, r->rt_scratch.bytes, r->stream);
    }
    LG_TRY(rc);
    r->tree_used = mode;
    const int n = render_tree_nodes(nbvh, r->n_tris, mode);
    const size_t nb = (size_t)n / 1024 + 1;
    size_t need = ((size_t)n * 11 + 2 * nb + 256) * sizeof(int);
    LG_TRY(r->scratch.reserve(need));
    LG_TRY(r->wide4.reserve(((size_t)n / 2 + 1) * sizeof(Wide4Node)));
    int root = 0, ni = 0, nl = 0, root4 = 0, n4 = 0;
    LG_TRY_CUDA(build_wide_nodes(r->rnodes.as<lg_bvh_node>(), n, r->wide.as<WideNode>(), r->leaves.as<int2>(),
                                 r->scratch.as<int>(), &root, &ni, &nl, r->stream));
    int leaf_inline = 0;
    static const int2 kEmptyLeaf = {0, 0};
    LG_TRY_CUDA(cudaMemcpyAsync(r->leaves.as<int2>() + nl, &kEmptyLeaf, sizeof(int2), cudaMemcpyHostToDevice,
                                r->stream));
    LG_TRY_CUDA(build_wide4_nodes(r->rnodes.as<lg_bvh_node>(), n, r->n_tris, nl, r->wide4.as<Wide4Node>(),
                                  r->scratch.as<int>(), &root4, &n4, &leaf_inline, &r->stack4, &r->stack2, r->stream));
    LG_TRY_CUDA(cudaStreamSynchronize(r->stream));
    r->leaf_inline = leaf_inline;
    r->root4 = root4;
    r->n4 = root4 >= 0 ? n4 : 0;
    r->root = root;
    ++r->scene_gen;
    return r->l2_window ? apply_l2_window(r) : LG_OK;
}

// Traversal records + intersection records from the device node/triangle arrays.
int finish_scene(lg_renderer* r)
{
    if (r->n_nodes == 0) { r->root = 0; return LG_OK; }
    LG_TRY(r->tv.reserve((size_t)r->n_tris * kTriVec * sizeof(float4)));
    LG_TRY(build_records(r));
    LG_TRY_CUDA(cudaMemcpyAsync(&r->root_node, r->nodes.p, sizeof(lg_bvh_node), cudaMemcpyDeviceToHost, r->stream));
    LG_TRY_CUDA(prepare_triangles(r->tris.as<lg_triangle>(), r->n_tris, r->tv.as<float4>(), r->watertight, r->stream));
    LG_TRY_CUDA(cudaStreamSynchronize(r->stream));
    return LG_OK;
}

int ensure_frame(lg_renderer* r, int w, int h, bool acc64)
{
    const size_t n = (size_t)w * h * 3;
    LG_TRY(r->accum.reserve(n * sizeof(float)));
    LG_TRY(r->rgb.reserve(n));
    if (acc64) LG_TRY(r->accum64.reserve(n * sizeof(double)));
    LG_TRY(r->work.reserve(256));
    LG_TRY(r->counters.reserve(sizeof(RenderCounters)));
    r->fw = w;
    r->fh = h;
    return LG_OK;
}

DevScene dev_scene(const lg_renderer* r)
{
    DevScene s;
    s.nodes = r->wide.as<WideNode>();
    s.leaves = r->leaves.as<int2>();
    s.tv = r->tv.as<float4>();
    s.tris = r->tris.as<lg_triangle>();
    s.mats = r->mats.as<float4>();
    s.texs = r->n_textured ? r->texs.as<unsigned long long>() : nullptr;
    s.points = r->points.as<lg_point_light>();
    s.n_points = r->n_points;
    s.root = r->root;
    s.nodes4 = r->wide4.as<Wide4Node>();
    s.root4 = r->root4;
    s.n4 = r->n4;
    s.leaf_inline = r->leaf_inline;
    s.sun = r->sun;
    s.fault = r->fault.as<unsigned>();
    return s;
}

// The renderer stream's access-policy window: with l2_window, accesses of
// its launches to the 4-wide records (up to the device's persisting-L2
// maximum) are marked persisting, and the context's persisting L2 set-aside
// is raised to that size (a per-process setting, released at exit);
// otherwise no window.
int apply_l2_window(lg_renderer* r)
{
    cudaStreamAttrValue attr{};
    if (r->l2_window && r->n4 > 0)
    {
        int maxp = 0;
        LG_TRY_CUDA(cudaDeviceGetAttribute(&maxp, cudaDevAttrMaxPersistingL2CacheSize, r->device));
        int maxw = 0;
        LG_TRY_CUDA(cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxAccessPolicyWindowSize, r->device));
        const size_t bytes = std::min({(size_t)r->n4 * sizeof(Wide4Node), (size_t)maxp, (size_t)maxw});
        LG_TRY_CUDA(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, bytes));
        attr.accessPolicyWindow.base_ptr = r->wide4.p;
        attr.accessPolicyWindow.num_bytes = bytes;
        attr.accessPolicyWindow.hitRatio = 1.0f;
        attr.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        attr.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    }
    LG_TRY_CUDA(cudaStreamSetAttribute(r->stream, cudaStreamAttributeAccessPolicyWindow, &attr));
    return LG_OK;
}

// True when no traversal over the current records can need more than the
// traversal stack's entries (the bound build_wide4_nodes computed), so the
// trace launches may leave out the per-push check.
bool stack_safe(const lg_renderer* r)
{
    return (r->bvh_width == 4 ? r->stack4 : r->stack2) <= kTraceStack;
}

// Queues a copy of the device fault word into its pinned host copy, after
// the launches already on `st`.
cudaError_t post_fault(lg_renderer* r, cudaStream_t st)
{
    return cudaMemcpyAsync(r->fault_host, r->fault.p, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
}

// Reports a traversal-stack overflow recorded by a finished launch and clears
// the word.  The fast path reads the pinned copy only; a set word is rare, and
// then the stream is drained first so no copy still in flight can set it again.
int take_fault(lg_renderer* r)
{
    if (!*(volatile unsigned*)r->fault_host) return LG_OK;
    LG_TRY_CUDA(cudaStreamSynchronize(r->stream));
    LG_TRY_CUDA(cudaMemsetAsync(r->fault.p, 0, sizeof(unsigned), r->stream));
    LG_TRY_CUDA(cudaStreamSynchronize(r->stream));
    *(volatile unsigned*)r->fault_host = 0u;
    return set_error(LG_ERR_DEVICE,
                     "traversal stack overflow: the BVH is deeper than the %d-entry traversal stack holds, so "
                     "some subtrees were skipped and the image is incomplete",
                     kTraceStack);
}

int render_into_device(lg_renderer* r, const lg_camera* cam, const lg_render_opts* o, lg_render_stats* stats)
{
    if (!r || !cam || !o) return set_error(LG_ERR_INVALID, "NULL argument");
    if (cam->width <= 0 || cam->height <= 0) return set_error(LG_ERR_INVALID, "image size %dx%d", cam->width, cam->height);
    if (o->spp < 0 || o->max_bounces < 0) return set_error(LG_ERR_INVALID, "spp/bounces must be >= 0");
    const bool acc64 = (o->flags & LG_RENDER_ACCUM64) != 0;
    LG_TRY(ensure_frame(r, cam->width, cam->height, acc64));
    const long long nval = (long long)cam->width * cam->height * 3;
    LG_TRY_CUDA(cudaMemsetAsync(r->accum.p, 0, (size_t)nval * sizeof(float), r->stream));
    if (acc64) LG_TRY_CUDA(cudaMemsetAsync(r->accum64.p, 0, (size_t)nval * sizeof(double), r->stream));
    if (r->counting) LG_TRY_CUDA(cudaMemsetAsync(r->counters.p, 0, sizeof(RenderCounters), r->stream));
    LG_TRY_CUDA(cudaEventRecord(r->ev0, r->stream));
    if (o->spp > 0 && r->n_nodes > 0)
    {
        const DevScene s = dev_scene(r);
        TraceJob job;
        job.spp = o->spp;
        job.max_bounces = o->max_bounces;
        job.sample_base = o->sample_base;
        job.n_chunks = (o->spp + 7) / 8;
        job.tiles_x = (cam->width + 7) / 8;
        job.n_tiles = job.tiles_x * ((cam->height + 3) / 4);
        job.accum = r->accum.as<float>();
        job.accum64 = acc64 ? r->accum64.as<double>() : nullptr;
        job.work64 = r->work.as<unsigned long long>();
        job.counters = r->counting ? r->counters.as<RenderCounters>() : nullptr;
        job.blocks_per_sm = r->trace_blocks_per_sm;
        job.refill_threshold = r->trace_refill;
        job.leaf_quorum = r->trace_quorum;
        job.top_records = r->trace_top;
        job.stack_safe = stack_safe(r);
        LG_TRY_CUDA(launch_trace(s, make_dev_cam(*cam), job, r->counting, r->sm_count, r->bvh_width, r->watertight,
                                 r->stream));
    }
    const float inv = 1.0f / (float)o->spp;
    LG_TRY_CUDA(launch_tonemap(r->accum.as<float>(), r->rgb.as<uint8_t>(), nval, inv, r->stream));
    LG_TRY_CUDA(cudaEventRecord(r->ev1, r->stream));
    LG_TRY_CUDA(post_fault(r, r->stream));
    if (stats)
    {
        LG_TRY_CUDA(cudaStreamSynchronize(r->stream));
        LG_TRY(take_fault(r));
        float ms = 0.0f;
        LG_TRY_CUDA(cudaEventElapsedTime(&ms, r->ev0, r->ev1));
        stats->kernel_ms = ms;
        stats->closest_rays = stats->shadow_rays = 0;
        stats->node_fetches = stats->tri_tests = stats->leaf_fetches = 0;
        if (r->counting)
        {
            RenderCounters c;
            LG_TRY_CUDA(cudaMemcpy(&c, r->counters.p, sizeof c, cudaMemcpyDeviceToHost));
            stats->closest_rays = c.closest_rays;
            stats->shadow_rays = c.shadow_rays;
            stats->node_fetches = c.node_fetches;
            stats->tri_tests = c.tri_tests;
            stats->leaf_fetches = c.leaf_fetches;
            if (c.stack_overflows)
                return set_error(LG_ERR_DEVICE, "traversal stack overflowed %llu times", c.stack_overflows);
        }
    }
    return LG_OK;
}
}  // namespace

extern "C" {

const char* lg_last_error(void) { return g_err.c_str(); }
int lg_version(void) { return 100; }

// ---- scene ----
int lg_scene_load_json(const char* path, int flags, int threads, lg_scene** out)
{
    if (!path || !out) return set_error(LG_ERR_INVALID, "NULL argument");
    *out = nullptr;
    lg_scene* s = new (std::nothrow) lg_scene();
    if (!s) return set_error(LG_ERR_NOMEM, "out of memory");
    std::string err;
    if (!load_scene_file(path, s->s, (flags & 1) != 0, threads, err))
    {
        delete s;
        return g_err.find("failed to open") != std::string::npos ? LG_ERR_IO : LG_ERR_PARSE;
    }
    *out = s;
    return LG_OK;
}

int lg_scene_create(const lg_scene_desc* d, lg_scene** out)
{
    if (!d || !out) return set_error(LG_ERR_INVALID, "NULL argument");
    lg_scene* s = new (std::nothrow) lg_scene();
    if (!s) return set_error(LG_ERR_NOMEM, "out of memory");
    CameraDesc& c = s->s.camera;
    std::memcpy(c.pos, d->camera.pos, sizeof c.pos);
    std::memcpy(c.cameraToWorld, d->camera.camera_to_world, sizeof c.cameraToWorld);
    c.fovYDeg = d->camera.fov_y_deg;
    c.aspect = d->camera.aspect;
    c.nearZ = d->camera.near_z;
    c.farZ = d->camera.far_z;
    c.imageWidth = d->camera.width;
    c.imageHeight = d->camera.height;
    std::memcpy(&s->s.sun, &d->sun, sizeof(lg_dir_light));
    s->s.triangles.resize((size_t)std::max(d->n_tris, 0));
    if (d->n_tris > 0) std::memcpy(s->s.triangles.data(), d->tris, (size_t)d->n_tris * sizeof(Triangle));
    for (int i = 0; i < d->n_mats; ++i)
    {
        Material m;
        for (int k = 0; k < 3; ++k)
        {
            m.albedo[k] = d->mat_albedo[3 * i + k];
            m.emissive[k] = d->mat_emissive ? d->mat_emissive[3 * i + k] : 0.0f;
        }
        s->s.materials.push_back(m);
    }
    s->s.points.resize((size_t)std::max(d->n_points, 0));
    if (d->n_points > 0) std::memcpy(s->s.points.data(), d->points, (size_t)d->n_points * sizeof(PointLight));
    s->s.directionals.resize((size_t)std::max(d->n_directionals, 0));
    if (d->n_directionals > 0)
        std::memcpy(s->s.directionals.data(), d->directionals, (size_t)d->n_directionals * sizeof(DirectionalLight));
    *out = s;
    return LG_OK;
}

int lg_scene_describe(const lg_scene* cs, lg_scene_desc* d)
{
    if (!cs || !d) return set_error(LG_ERR_INVALID, "NULL argument");
    lg_scene* s = const_cast<lg_scene*>(cs);
    const CameraDesc& c = s->s.camera;
    std::memcpy(d->camera.pos, c.pos, sizeof c.pos);
    std::memcpy(d->camera.camera_to_world, c.cameraToWorld, sizeof c.cameraToWorld);
    d->camera.fov_y_deg = c.fovYDeg;
    d->camera.aspect = c.aspect;
    d->camera.near_z = c.nearZ;
    d->camera.far_z = c.farZ;
    d->camera.width = c.imageWidth;
    d->camera.height = c.imageHeight;
    std::memcpy(&d->sun, &s->s.sun, sizeof(lg_dir_light));
    d->tris = reinterpret_cast<const lg_triangle*>(s->s.triangles.data());
    d->n_tris = (int32_t)s->s.triangles.size();
    s->albedo.resize(s->s.materials.size() * 3);
    s->emissive.resize(s->s.materials.size() * 3);
    for (size_t i = 0; i < s->s.materials.size(); ++i)
        for (int k = 0; k < 3; ++k)
        {
            s->albedo[3 * i + k] = s->s.materials[i].albedo[k];
            s->emissive[3 * i + k] = s->s.materials[i].emissive[k];
        }
    d->mat_albedo = s->albedo.data();
    d->mat_emissive = s->emissive.data();
    d->n_mats = (int32_t)s->s.materials.size();
    d->points = reinterpret_cast<const lg_point_light*>(s->s.points.data());
    d->n_points = (int32_t)s->s.points.size();
    d->directionals = reinterpret_cast<const lg_dir_light*>(s->s.directionals.data());
    d->n_directionals = (int32_t)s->s.directionals.size();
    return LG_OK;
}

int lg_scene_set_camera(lg_scene* s, const lg_camera* cam)
{
    if (!s || !cam) return set_error(LG_ERR_INVALID, "NULL argument");
    CameraDesc& c = s->s.camera;
    std::memcpy(c.pos, cam->pos, sizeof c.pos);
    std::memcpy(c.cameraToWorld, cam->camera_to_world, sizeof c.cameraToWorld);
    c.fovYDeg = cam->fov_y_deg;
    c.aspect = cam->aspect;
    c.nearZ = cam->near_z;
    c.farZ = cam->far_z;
    c.imageWidth = cam->width;
    c.imageHeight = cam->height;
    return LG_OK;
}

int lg_scene_save_json(const lg_scene* s, const char* path)
{
    if (!s || !path) return set_error(LG_ERR_INVALID, "NULL argument");
    if (!save_scene_file(s->s, path, 0)) return set_error(LG_ERR_IO, "cannot write %s", path);
    return LG_OK;
}

int lg_scene_save_bin(const lg_scene* s, const char* path)
{
    if (!s || !path) return set_error(LG_ERR_INVALID, "NULL argument");
    if (!save_scene_bin(s->s, path)) return set_error(LG_ERR_IO, "cannot write %s", path);
    return LG_OK;
}

const char* lg_scene_texture(const lg_scene* s, int material)
{
    if (!s || material < 0 || material >= (int)s->s.materials.size()) return "";
    return s->s.materials[(size_t)material].diffuseTex.c_str();
}

int lg_scene_set_texture(lg_scene* s, int material, const char* path)
{
    if (!s || !path) return set_error(LG_ERR_INVALID, "NULL argument");
    if (material < 0 || material >= (int)s->s.materials.size())
        return set_error(LG_ERR_INVALID, "material %d out of range", material);
    s->s.materials[(size_t)material].diffuseTex = path;
    return LG_OK;
}

void lg_scene_destroy(lg_scene* s) { delete s; }

// ---- images ----
int lg_image_load(const char* path, int32_t* w, int32_t* h, uint8_t** rgba8)
{
    if (!path || !w || !h || !rgba8) return set_error(LG_ERR_INVALID, "NULL argument");
    *rgba8 = nullptr;
    std::vector<uint8_t> px;
    std::string err;
    int iw = 0, ih = 0;
    if (!decode_png(path, iw, ih, px, err))
        return set_error(err == "cannot open" ? LG_ERR_IO : LG_ERR_PARSE, "%s: %s", path, err.c_str());
    uint8_t* out = (uint8_t*)std::malloc(px.size());
    if (!out) return set_error(LG_ERR_NOMEM, "out of memory");
    std::memcpy(out, px.data(), px.size());
    *w = iw;
    *h = ih;
    *rgba8 = out;
    return LG_OK;
}

void lg_image_free(uint8_t* rgba8) { std::free(rgba8); }

// overwrite_camera (reference main.cpp:29-59).
void lg_look_at(lg_camera* cam, const float pos[3], const float tgt[3])
{
    float fx = tgt[0] - pos[0];
    float fy = tgt[1] - pos[1];
    float fz = tgt[2] - pos[2];
    float fl = std::sqrt(fx * fx + fy * fy + fz * fz);
    if (fl < 1e-8f) return;
    fx /= fl;
    fy /= fl;
    fz /= fl;
    float lx = -fy, ly = fx, lz = 0.0f;
    float ll = std::sqrt(lx * lx + ly * ly + lz * lz);
    if (ll < 1e-6f) { lx = 0; ly = 1; lz = 0; ll = 1; }
    lx /= ll;
    ly /= ll;
    lz /= ll;
    float ux = fy * lz - fz * ly;
    float uy = fz * lx - fx * lz;
    float uz = fx * ly - fy * lx;
    float* m = cam->camera_to_world;
    m[0] = fx; m[1] = fy; m[2] = fz; m[3] = 0;
    m[4] = lx; m[5] = ly; m[6] = lz; m[7] = 0;
    m[8] = ux; m[9] = uy; m[10] = uz; m[11] = 0;
    m[12] = pos[0]; m[13] = pos[1]; m[14] = pos[2]; m[15] = 1;
    cam->pos[0] = pos[0];
    cam->pos[1] = pos[1];
    cam->pos[2] = pos[2];
}

// ---- BVH ----
int lg_build_bvh_device(const lg_triangle* d_tris, int32_t n_tris, lg_bvh_node* d_nodes_out, int32_t* n_nodes_out,
                        int32_t* d_perm_out, lg_triangle* d_tris_out, void* stream)
{
    if (!n_nodes_out || (n_tris > 0 && (!d_tris || !d_nodes_out))) return set_error(LG_ERR_INVALID, "NULL argument");
    int dev = 0;
    LG_TRY_CUDA(cudaGetDevice(&dev));
    DeviceScratch& ds = device_scratch(dev);
    std::lock_guard<std::mutex> lk(ds.mu);
    const bool tmp = d_tris_out == nullptr || d_tris_out == d_tris;
    LG_TRY(ds.buf.reserve(lbvh_scratch_bytes(n_tris, tmp)));
    int count = 0;
    LG_TRY(lbvh_build(d_tris, n_tris, d_nodes_out, &count, d_perm_out, d_tris_out, ds.buf.p, ds.buf.bytes,
                      (cudaStream_t)stream));
    *n_nodes_out = count;
    return LG_OK;
}

int lg_build_bvh(const lg_triangle* tris, int32_t n, lg_bvh_node* nodes_out, int32_t* n_nodes_out, int32_t* perm_out,
                 lg_triangle* tris_out)
{
    if (!n_nodes_out || n < 0 || (n > 0 && (!tris || !nodes_out))) return set_error(LG_ERR_INVALID, "bad argument");
    if (n == 0) { *n_nodes_out = 0; return LG_OK; }
    lg_triangle* d_in = nullptr;
    lg_triangle* d_out = nullptr;
    lg_bvh_node* d_nodes = nullptr;
    int32_t* d_perm = nullptr;
    int rc = LG_OK;
    int32_t count = 0;
    const size_t tb = (size_t)n * sizeof(lg_triangle);
    cudaStream_t st = nullptr;
    auto fail = [&](cudaError_t e, const char* what) {
        rc = set_error(LG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) { fail(e, "stream"); goto done; }
    if ((e = cudaMalloc(&d_in, tb)) != cudaSuccess) { fail(e, "cudaMalloc"); goto done; }
    if ((e = cudaMalloc(&d_out, tb)) != cudaSuccess) { fail(e, "cudaMalloc"); goto done; }
    if ((e = cudaMalloc(&d_nodes, (size_t)(2 * n - 1) * sizeof(lg_bvh_node))) != cudaSuccess) { fail(e, "cudaMalloc"); goto done; }
    if ((e = cudaMalloc(&d_perm, (size_t)n * sizeof(int32_t))) != cudaSuccess) { fail(e, "cudaMalloc"); goto done; }
    if ((e = cudaMemcpyAsync(d_in, tris, tb, cudaMemcpyHostToDevice, st)) != cudaSuccess) { fail(e, "H2D"); goto done; }
    rc = lg_build_bvh_device(d_in, n, d_nodes, &count, d_perm, d_out, st);
    if (rc != LG_OK) goto done;
    if ((e = cudaMemcpyAsync(nodes_out, d_nodes, (size_t)count * sizeof(lg_bvh_node), cudaMemcpyDeviceToHost, st)) != cudaSuccess) { fail(e, "D2H"); goto done; }
    if (perm_out && (e = cudaMemcpyAsync(perm_out, d_perm, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, st)) != cudaSuccess) { fail(e, "D2H"); goto done; }
    if (tris_out && (e = cudaMemcpyAsync(tris_out, d_out, tb, cudaMemcpyDeviceToHost, st)) != cudaSuccess) { fail(e, "D2H"); goto done; }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) { fail(e, "sync"); goto done; }
    *n_nodes_out = count;
done:
    cudaFree(d_in);
    cudaFree(d_out);
    cudaFree(d_nodes);
    cudaFree(d_perm);
    if (st) cudaStreamDestroy(st);
    return rc;
}

// ---- renderer ----
int lg_renderer_create(int device, lg_renderer** out)
{
    if (!out) return set_error(LG_ERR_INVALID, "NULL argument");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return set_error(LG_ERR_CUDA, "no CUDA device: %s", e != cudaSuccess ? cudaGetErrorString(e) : "count 0");
    if (device < 0 || device >= ndev) return set_error(LG_ERR_INVALID, "device %d out of range", device);
    DeviceGuard g(device);
    lg_renderer* r = new (std::nothrow) lg_renderer();
    if (!r) return set_error(LG_ERR_NOMEM, "out of memory");
    r->device = device;
    cudaDeviceGetAttribute(&r->sm_count, cudaDevAttrMultiProcessorCount, device);
    if ((e = cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&r->ev0)) != cudaSuccess || (e = cudaEventCreate(&r->ev1)) != cudaSuccess ||
        (e = cudaMallocHost((void**)&r->fault_host, sizeof(unsigned))) != cudaSuccess)
    {
        lg_renderer_destroy(r);
        return set_error(LG_ERR_CUDA, "renderer init: %s", cudaGetErrorString(e));
    }
    *r->fault_host = 0u;
    if (r->fault.reserve(sizeof(unsigned)) != LG_OK ||
        (e = cudaMemsetAsync(r->fault.p, 0, sizeof(unsigned), r->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(r->stream)) != cudaSuccess)
    {
        lg_renderer_destroy(r);
        return set_error(LG_ERR_CUDA, "renderer init: fault word: %s", cudaGetErrorString(e));
    }
    *out = r;
    return LG_OK;
}

void lg_renderer_destroy(lg_renderer* r)
{
    if (!r) return;
    DeviceGuard g(r->device);
    if (r->stream) cudaStreamSynchronize(r->stream);
    r->n_mats = 0;
    clear_textures(r);
    r->texs.release();
    r->gbuf.release();
    if (r->batch_exec) cudaGraphExecDestroy(r->batch_exec);
    if (r->batch_host) cudaFreeHost(r->batch_host);
    if (r->fault_host) cudaFreeHost(r->fault_host);
    r->fault.release();
    r->matchk.release();
    for (DevBuf* b : {&r->batch_jobs, &r->batch_acc, &r->batch_rgb, &r->rnodes, &r->rt_scratch, &r->wf_scratch})
        b->release();
    for (DevBuf* b : {&r->tris, &r->tris_in, &r->nodes, &r->wide, &r->wide4, &r->leaves, &r->tv, &r->mats, &r->points,
                      &r->scratch, &r->accum, &r->accum64, &r->rgb, &r->work, &r->counters})
        b->release();
    if (r->ev0) cudaEventDestroy(r->ev0);
    if (r->ev1) cudaEventDestroy(r->ev1);
    if (r->stream) cudaStreamDestroy(r->stream);
    delete r;
}

int lg_renderer_set_scene(lg_renderer* r, const lg_scene_desc* d)
{
    if (!r) return set_error(LG_ERR_INVALID, "NULL renderer");
    LG_TRY(validate_scene(d));
    DeviceGuard g(r->device);
    const int n = d->n_tris;
    r->n_tris = n;
    LG_TRY(upload_common(r, d));
    LG_TRY(r->tris.reserve((size_t)std::max(n, 1) * sizeof(lg_triangle)));
    LG_TRY(r->tris_in.reserve((size_t)std::max(n, 1) * sizeof(lg_triangle)));
    LG_TRY(r->nodes.reserve((size_t)std::max(2 * n - 1, 1) * sizeof(lg_bvh_node)));
    if (n > 0)
        LG_TRY_CUDA(cudaMemcpyAsync(r->tris_in.p, d->tris, (size_t)n * sizeof(lg_triangle), cudaMemcpyHostToDevice,
                                    r->stream));
    LG_TRY(queue_material_check(r, r->tris_in.as<lg_triangle>(), n, d->n_mats));
    LG_TRY(r->scratch.reserve(lbvh_scratch_bytes(n, false)));
    int count = 0;
    LG_TRY(lbvh_build(r->tris_in.as<lg_triangle>(), n, r->nodes.as<lg_bvh_node>(), &count, nullptr,
                      r->tris.as<lg_triangle>(), r->scratch.p, r->scratch.bytes, r->stream));
    r->n_nodes = count;
    LG_TRY(finish_scene(r));
    return take_material_check(r, d);
}

int lg_renderer_set_scene_bvh(lg_renderer* r, const lg_scene_desc* d, const lg_bvh_node* nodes, int32_t n_nodes)
{
    if (!r) return set_error(LG_ERR_INVALID, "NULL renderer");
    LG_TRY(validate_scene(d));
    if (n_nodes < 0 || (n_nodes > 0 && !nodes)) return set_error(LG_ERR_INVALID, "bad node array");
    if (d->n_tris > 0 && n_nodes == 0) return set_error(LG_ERR_INVALID, "triangles without a BVH");
    for (int i = 0; i < n_nodes; ++i)
    {
        const lg_bvh_node& nd = nodes[i];
        if (nd.triCount > 0)
        {
            if (nd.firstTri < 0 || (long long)nd.firstTri + nd.triCount > d->n_tris)
                return set_error(LG_ERR_INVALID, "node %d: triangle range outside the scene", i);
        }
        else if (nd.triCount < 0 || nd.left <= i || nd.right <= i || nd.left >= n_nodes || nd.right >= n_nodes)
            return set_error(LG_ERR_INVALID, "node %d: child links must point forward inside the array", i);
    }
    DeviceGuard g(r->device);
    r->n_tris = d->n_tris;
    r->n_nodes = n_nodes;
    LG_TRY(upload_common(r, d));
    LG_TRY(r->tris.reserve((size_t)std::max(d->n_tris, 1) * sizeof(lg_triangle)));
    LG_TRY(r->nodes.reserve((size_t)std::max(n_nodes, 1) * sizeof(lg_bvh_node)));
    if (d->n_tris)
        LG_TRY_CUDA(cudaMemcpyAsync(r->tris.p, d->tris, (size_t)d->n_tris * sizeof(lg_triangle),
                                    cudaMemcpyHostToDevice, r->stream));
    LG_TRY(queue_material_check(r, r->tris.as<lg_triangle>(), d->n_tris, d->n_mats));
    if (n_nodes)
        LG_TRY_CUDA(cudaMemcpyAsync(r->nodes.p, nodes, (size_t)n_nodes * sizeof(lg_bvh_node), cudaMemcpyHostToDevice,
                                    r->stream));
    LG_TRY(finish_scene(r));
    return take_material_check(r, d);
}

int lg_renderer_get_bvh(lg_renderer* r, lg_bvh_node* nodes_out, int32_t* n_nodes, lg_triangle* tris_out)
{
    if (!r || !n_nodes) return set_error(LG_ERR_INVALID, "NULL argument");
    DeviceGuard g(r->device);
    *n_nodes = r->n_nodes;
    if (nodes_out && r->n_nodes)
        LG_TRY_CUDA(cudaMemcpyAsync(nodes_out, r->nodes.p, (size_t)r->n_nodes * sizeof(lg_bvh_node),
                                    cudaMemcpyDeviceToHost, r->stream));
    if (tris_out && r->n_tris)
        LG_TRY_CUDA(cudaMemcpyAsync(tris_out, r->tris.p, (size_t)r->n_tris * sizeof(lg_triangle),
                                    cudaMemcpyDeviceToHost, r->stream));
    LG_TRY_CUDA(cudaStreamSynchronize(r->stream));
    return LG_OK;
}

int lg_renderer_set_bvh_width(lg_renderer* r, int width)
{
    if (!r) return set_error(LG_ERR_INVALID, "NULL renderer");
    if (width != 2 && width != 4) return set_error(LG_ERR_INVALID, "BVH width must be 2 or 4");
    r->bvh_width = width;
    return LG_OK;
}

int lg_renderer_set_texture(lg_renderer* r, int material, const uint8_t* rgba8, int32_t w, int32_t h)
{
    if (!r) return set_error(LG_ERR_INVALID, "NULL renderer");
    if (material < 0 || material >= r->n_mats) return set_error(LG_ERR_INVALID, "material %d out of range", material);
    if (rgba8 && (w <= 0 || h <= 0)) return set_error(LG_ERR_INVALID, "texture size %dx%d", w, h);
    DeviceGuard g(r->device);
    LG_TRY_CUDA(cudaStreamSynchronize(r->stream));
    const size_t m = (size_t)material;
    if (r->tex_objs[m])
    {
        cudaDestroyTextureObject((cudaTextureObject_t)r->tex_objs[m]);
        cudaFreeArray(r->tex_arrays[m]);
        r->tex_objs[m] = 0;
        r->tex_arrays[m] = nullptr;
        --r->n_textured;
    }
    if (rgba8)
    {
        // uchar4 array read as sRGB, normalised float, bilinear, wrapping (pathtracer.cu:562-576).
        cudaChannelFormatDesc fmt = cudaCreateChannelDesc<uchar4>();
        cudaArray_t arr = nullptr;
        LG_TRY_CUDA(cudaMallocArray(&arr, &fmt, (size_t)w, (size_t)h));
        cudaError_t e = cudaMemcpy2DToArray(arr, 0, 0, rgba8, (size_t)w * 4, (size_t)w * 4, (size_t)h,
                                            cudaMemcpyHostToDevice);
        cudaResourceDesc res{};
        res.resType = cudaResourceTypeArray;
        res.res.array.array = arr;
        cudaTextureDesc td{};
        td.addressMode[0] = cudaAddressModeWrap;
        td.addressMode[1] = cudaAddressModeWrap;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeNormalizedFloat;
        td.normalizedCoords = 1;
        td.sRGB = 1;
        cudaTextureObject_t obj = 0;
        if (e == cudaSuccess) e = cudaCreateTextureObject(&obj, &res, &td, nullptr);
        if (e != cudaSuccess)
        {
            cudaFreeArray(arr);
            return set_error(LG_ERR_CUDA, "texture upload: %s", cudaGetErrorString(e));
        }
        r->tex_arrays[m] = arr;
        r->tex_objs[m] = (unsigned long long)obj;
        ++r->n_textured;
    }
    ++r->scene_gen;
    LG_TRY(r->texs.reserve((size_t)std::max(r->n_mats, 1) * sizeof(unsigned long long)));
    LG_TRY_CUDA(cudaMemcpy(r->texs.p, r->tex_objs.data(), (size_t)r->n_mats * sizeof(unsigned long long),
                           cudaMemcpyHostToDevice));
    return LG_OK;
}

int lg_renderer_load_textures(lg_renderer* r, const lg_scene* s, const char* asset_root, int32_t* loaded,
                              int32_t* missing)
{
    if (!r || !s || !asset_root) return set_error(LG_ERR_INVALID, "NULL argument");
    if ((int)s->s.materials.size() != r->n_mats)
        return set_error(LG_ERR_INVALID, "scene has %zu materials, renderer %d", s->s.materials.size(), r->n_mats);
    int nl = 0, nm = 0;
    for (int m = 0; m < r->n_mats; ++m)
    {
        const std::string& rel = s->s.materials[(size_t)m].diffuseTex;
        if (rel.empty()) continue;
        const std::string full = std::string(asset_root) + "/" + rel;
        int32_t w = 0, h = 0;
        uint8_t* px = nullptr;
        if (lg_image_load(full.c_str(), &w, &h, &px) != LG_OK)
        {
            ++nm;
            continue;
        }
        const int rc = lg_renderer_set_texture(r, m, px, w, h);
        lg_image_free(px);
        LG_TRY(rc);
        ++nl;
    }
    if (loaded) *loaded = nl;
    if (missing) *missing = nm;
    return LG_OK;
}

int lg_renderer_set_intersection(lg_renderer* r, int mode)
{
    if (!r) return set_error(LG_ERR_INVALID, "NULL renderer");
    if (mode != LG_ISECT_MOLLER_TRUMBORE && mode != LG_ISECT_WATERTIGHT)
        return set_error(LG_ERR_INVALID, "intersection mode must be 0 (Moller-Trumbore) or 1 (watertight)");
    const bool wt = mode == LG_ISECT_WATERTIGHT;
    if (wt == r->watertight) return LG_OK;
    DeviceGuard g(r->device);
    r->watertight = wt;
    ++r->scene_gen;
    if (r->n_tris > 0)
    {
        LG_TRY_CUDA(prepare_triangles(r->tris.as<lg_triangle>(), r->n_tris, r->tv.as<float4>(), wt, r->stream));
        LG_TRY_CUDA(cudaStreamSynchronize(r->stream));
    }
    return LG_OK;
}

int lg_renderer_autotune(lg_renderer* r, const lg_camera* cam, int spp, int max_bounces, int32_t* blocks_per_sm_out,
                         float* ms_out)
{
    if (!r || !cam || spp <= 0 || max_bounces < 0) return set_error(LG_ERR_INVALID, "bad argument");
    DeviceGuard g(r->device);
    const int saved = r->trace_blocks_per_sm;
    const bool counting = r->counting;
    r->counting = false;
    int best = 0;
    float best_ms = 1e30f;
    int rc = LG_OK;
    // Candidates: 1 .. 4 resident 256-thread blocks per SM (the kernel's register budget allows 4).
    for (int bps = 1; bps <= 4 && rc == LG_OK; ++bps)
    {
        r->trace_blocks_per_sm = bps;
        float ms = 1e30f;
        for (int rep = 0; rep < 3 && rc == LG_OK; ++rep)
        {
            lg_render_opts o{spp, max_bounces, 0, 0};
            lg_render_stats st{};
            rc = render_into_device(r, cam, &o, &st);
            if (rc == LG_OK && rep > 0) ms = std::min(ms, st.kernel_ms);
        }
        if (rc == LG_OK && ms < best_ms)
        {
            best_ms = ms;
            best = bps;
        }
    }
    r->counting = counting;
    r->trace_blocks_per_sm = rc == LG_OK ? best : saved;
    if (rc != LG_OK) return rc;
    if (blocks_per_sm_out) *blocks_per_sm_out = best;
    if (ms_out) *ms_out = best_ms;
    return LG_OK;
}

int lg_renderer_autotune_schedule(lg_renderer* r, const lg_camera* cam, int spp, int max_bounces,
                                  int32_t* refill_out, int32_t* quorum_out, float* ms_out)
{
    if (!r || !cam || spp <= 0 || max_bounces < 0) return set_error(LG_ERR_INVALID, "bad argument");
    DeviceGuard g(r->device);
    const int saved_refill = r->trace_refill, saved_quorum = r->trace_quorum;
    const bool counting = r->counting;
    r->counting = false;
    // Candidates around the engine-scene optimum (refill 12, quorum 12); one
    // untimed render, then the fastest of two timed ones per pair.
    static const int kRefill[] = {8, 12, 16, 24};
    static const int kQuorum[] = {4, 8, 12, 16};
    int best_refill = saved_refill, best_quorum = saved_quorum;
    float best_ms = 1e30f;
    int rc = LG_OK;
    for (int fi = 0; fi < 4 && rc == LG_OK; ++fi)
        for (int qi = 0; qi < 4 && rc == LG_OK; ++qi)
        {
            r->trace_refill = kRefill[fi];
            r->trace_quorum = kQuorum[qi];
            float ms = 1e30f;
            for (int rep = 0; rep < 3 && rc == LG_OK; ++rep)
            {
                lg_render_opts o{spp, max_bounces, 0, 0};
                lg_render_stats st{};
                rc = render_into_device(r, cam, &o, &st);
                if (rc == LG_OK && rep > 0) ms = std::min(ms, st.kernel_ms);
            }
            if (rc == LG_OK && ms < best_ms)
            {
                best_ms = ms;
                best_refill = kRefill[fi];
                best_quorum = kQuorum[qi];
            }
        }
    r->counting = counting;
    r->trace_refill = rc == LG_OK ? best_refill : saved_refill;
    r->trace_quorum = rc == LG_OK ? best_quorum : saved_quorum;
    if (rc != LG_OK) return rc;
    if (refill_out) *refill_out = best_refill;
    if (quorum_out) *quorum_out = best_quorum;
    if (ms_out) *ms_out = best_ms;
    return LG_OK;
}

int lg_renderer_set_refill_threshold(lg_renderer* r, int threshold)
{
    if (!r) return set_error(LG_ERR_INVALID, "NULL renderer");
    if (threshold < 1 || threshold > 32) return set_error(LG_ERR_INVALID, "refill threshold must be 1..32");
    r->trace_refill = threshold;
    return LG_OK;
}

int lg_renderer_get_refill_threshold(const lg_renderer* r)
{
    if (!r) return set_error(LG_ERR_INVALID, "NULL renderer");
    return r->trace_refill;
}

int lg_renderer_set_leaf_quorum(lg_renderer* r, int quorum)
{
    if (!r) return set_error(LG_ERR_INVALID, "NULL renderer");
    if (quorum < 0 || quorum > 31) return set_error(LG_ERR_INVALID, "leaf quorum must be 0..31");
    r->trace_quorum = quorum;
    return LG_OK;
}

int lg_renderer_get_leaf_quorum(const lg_renderer* r)
{
    if (!r) return set_error(LG_ERR_INVALID, "NULL renderer");
    return r->trace_quorum;
}

int lg_renderer_get_stack_bound(const lg_renderer* r, int32_t* bound, int32_t* capacity)
{
    if (!r || !bound || !capacity) return set_error(LG_ERR_INVALID, "NULL argument");
    *bound = r->n_nodes ? (r->bvh_width == 4 ? r->stack4 : r->stack2) : 0;
    *capacity = kTraceStack;
    return LG_OK;
}

int lg_renderer_set_l2_window(lg_renderer* r, int enable)
{
    if (!r) return set_error(LG_ERR_INVALID, "NULL renderer");
    DeviceGuard g(r->device);
    r->l2_window = enable != 0;
    ++r->scene_gen;  // captured batch graphs carry the stream's window
    return apply_l2_window(r);
}

int lg_renderer_set_top_records(lg_renderer* r, int n)
{
    if (!r) return set_error(LG_ERR_INVALID, "NULL renderer");
    if (n < 0 || n > LG_TOP_RECORDS_MAX) return set_error(LG_ERR_INVALID, "top records must be 0..%d", LG_TOP_RECORDS_MAX);
    r->trace_top = n;
    return LG_OK;
}

int lg_renderer_get_top_records(const lg_renderer* r)
{
    if (!r) return set_error(LG_ERR_INVALID, "NULL renderer");
    return r->trace_top;
}

int lg_renderer_set_render_tree(lg_renderer* r, int mode)
{
    if (!r) return set_error(LG_ERR_INVALID, "NULL renderer");
    if (mode != LG_RENDER_TREE_BUILDBVH && mode != LG_RENDER_TREE_PLOC && mode != LG_RENDER_TREE_PLOC_TRIANGLES)
        return set_error(LG_ERR_INVALID,
                         "render tree mode must be 0 (BuildBVH topology), 1 (PLOC over its leaves) or 2 (PLOC over "
                         "triangles)");
    if (mode == r->tree_mode) return LG_OK;
    DeviceGuard g(r->device);
    r->tree_mode = mode;
    if (r->n_nodes == 0) return LG_OK;
    LG_TRY_CUDA(cudaStreamSynchronize(r->stream));
    return build_records(r);
}

int lg_renderer_get_render_tree(lg_renderer* r, int32_t* mode_used)
{
    if (!r || !mode_used) return set_error(LG_ERR_INVALID, "NULL argument");
    *mode_used = r->tree_used;
    return LG_OK;
}

int lg_renderer_set_counting(lg_renderer* r, int enable)
{
    if (!r) return set_error(LG_ERR_INVALID, "NULL renderer");
    r->counting = enable != 0;
    return LG_OK;
}

int lg_render(lg_renderer* r, const lg_camera* cam, const lg_render_opts* o, uint8_t* rgb8, float* accum,
              double* accum64, lg_render_stats* stats)
{
    if (!r) return set_error(LG_ERR_INVALID, "NULL renderer");
    DeviceGuard g(r->device);
    if (accum64 && !(o && (o->flags & LG_RENDER_ACCUM64)))
        return set_error(LG_ERR_INVALID, "accum64 output needs LG_RENDER_ACCUM64");
    lg_render_stats local{};
    LG_TRY(render_into_device(r, cam, o, stats ? stats : &local));
    const size_t nval = (size_t)cam->width * cam->height * 3;
    if (rgb8) LG_TRY_CUDA(cudaMemcpyAsync(rgb8, r->rgb.p, nval, cudaMemcpyDeviceToHost, r->stream));
    if (accum) LG_TRY_CUDA(cudaMemcpyAsync(accum, r->accum.p, nval * sizeof(float), cudaMemcpyDeviceToHost, r->stream));
    if (accum64)
        LG_TRY_CUDA(cudaMemcpyAsync(accum64, r->accum64.p, nval * sizeof(double), cudaMemcpyDeviceToHost, r->stream));
    LG_TRY_CUDA(cudaStreamSynchronize(r->stream));
    return LG_OK;
}

int lg_render_device(lg_renderer* r, const lg_camera* cam, const lg_render_opts* o, void* stream,
                     const uint8_t** d_rgb8, const float** d_accum, const double** d_accum64)
{
    if (!r) return set_error(LG_ERR_INVALID, "NULL renderer");
    DeviceGuard g(r->device);
    // An overflow in an earlier asynchronous frame is reported here.
    LG_TRY(take_fault(r));
    // Order the renderer's stream after the caller's stream.
    if (stream)
    {
        cudaEvent_t ev;
        LG_TRY_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        cudaEventRecord(ev, (cudaStream_t)stream);
        cudaStreamWaitEvent(r->stream, ev, 0);
        cudaEventDestroy(ev);
    }
    LG_TRY(render_into_device(r, cam, o, nullptr));
    if (stream)
    {
        cudaEvent_t ev;
        LG_TRY_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        cudaEventRecord(ev, r->stream);
        cudaStreamWaitEvent((cudaStream_t)stream, ev, 0);
        cudaEventDestroy(ev);
    }
    else
    {
        LG_TRY_CUDA(cudaStreamSynchronize(r->stream));
        LG_TRY(take_fault(r));
    }
    if (d_rgb8) *d_rgb8 = r->rgb.as<uint8_t>();
    if (d_accum) *d_accum = r->accum.as<float>();
    if (d_accum64) *d_accum64 = (o->flags & LG_RENDER_ACCUM64) ? r->accum64.as<double>() : nullptr;
    return LG_OK;
}

int lg_render_sorted(lg_renderer* r, const lg_camera* cam, const lg_render_opts* o, uint8_t* rgb8, float* accum,
                     lg_render_stats* stats)
{
    if (!r || !cam || !o) return set_error(LG_ERR_INVALID, "NULL argument");
    if (cam->width <= 0 || cam->height <= 0) return set_error(LG_ERR_INVALID, "image size %dx%d", cam->width, cam->height);
    if ((long long)cam->width * cam->height > (1ll << 30)) return set_error(LG_ERR_INVALID, "image too large");
    if (o->spp < 0 || o->max_bounces < 0) return set_error(LG_ERR_INVALID, "spp/bounces must be >= 0");
    if (o->flags & LG_RENDER_ACCUM64) return set_error(LG_ERR_INVALID, "the ray-sorted render has no FP64 accumulator");
    DeviceGuard g(r->device);
    LG_TRY(take_fault(r));
    LG_TRY(ensure_frame(r, cam->width, cam->height, false));
    const int npix = cam->width * cam->height;
    const long long nval = (long long)npix * 3;
    LG_TRY(r->wf_scratch.reserve(wavefront_scratch_bytes(npix, r->n_points + 1)));
    LG_TRY_CUDA(cudaMemsetAsync(r->accum.p, 0, (size_t)nval * sizeof(float), r->stream));
    if (r->counting) LG_TRY_CUDA(cudaMemsetAsync(r->counters.p, 0, sizeof(RenderCounters), r->stream));
    LG_TRY_CUDA(cudaEventRecord(r->ev0, r->stream));
    if (o->spp > 0 && r->n_nodes > 0)
    {
        WavefrontJob job;
        job.spp = o->spp;
        job.max_bounces = o->max_bounces;
        job.sample_base = o->sample_base;
        job.sort = (o->flags & LG_RENDER_NO_RAY_SORT) == 0;
        job.width = r->bvh_width;
        job.watertight = r->watertight;
        job.accum = r->accum.as<float>();
        job.counters = r->counting ? r->counters.as<RenderCounters>() : nullptr;
        job.sm_count = r->sm_count;
        job.refill = 8;  // ray-list traversals: refill at 8 idle lanes (64-spp engine frame: 4 and 16 are 2-4% slower)
        job.quorum = r->trace_quorum;
        job.stack_safe = stack_safe(r);
        LG_TRY_CUDA(launch_wavefront_frame(dev_scene(r), make_dev_cam(*cam), job, r->wf_scratch.p,
                                           r->wf_scratch.bytes, r->stream));
    }
    LG_TRY_CUDA(launch_tonemap(r->accum.as<float>(), r->rgb.as<uint8_t>(), nval, 1.0f / (float)o->spp, r->stream));
    LG_TRY_CUDA(cudaEventRecord(r->ev1, r->stream));
    LG_TRY_CUDA(post_fault(r, r->stream));
    if (rgb8) LG_TRY_CUDA(cudaMemcpyAsync(rgb8, r->rgb.p, (size_t)nval, cudaMemcpyDeviceToHost, r->stream));
    if (accum) LG_TRY_CUDA(cudaMemcpyAsync(accum, r->accum.p, (size_t)nval * sizeof(float), cudaMemcpyDeviceToHost, r->stream));
    LG_TRY_CUDA(cudaStreamSynchronize(r->stream));
    LG_TRY(take_fault(r));
    if (stats)
    {
        float ms = 0.0f;
        LG_TRY_CUDA(cudaEventElapsedTime(&ms, r->ev0, r->ev1));
        *stats = lg_render_stats{};
        stats->kernel_ms = ms;
        if (r->counting)
        {
            RenderCounters c;
            LG_TRY_CUDA(cudaMemcpy(&c, r->counters.p, sizeof c, cudaMemcpyDeviceToHost));
            stats->closest_rays = c.closest_rays;
            stats->shadow_rays = c.shadow_rays;
            stats->node_fetches = c.node_fetches;
            stats->tri_tests = c.tri_tests;
            stats->leaf_fetches = c.leaf_fetches;
        }
    }
    return LG_OK;
}

int lg_render_batch(lg_renderer* r, const lg_camera* cams, const lg_render_opts* opts, int32_t n_jobs,
                    uint8_t* rgb8_out, float* ms_per_job)
{
    if (!r || !cams || !opts || n_jobs < 0) return set_error(LG_ERR_INVALID, "bad argument");
    if (n_jobs == 0) return LG_OK;
    DeviceGuard g(r->device);
    // Every frame's (pixel, chunk of 8 samples) items in one persistent launch,
    // numbered frame after frame; frames go to consecutive accumulators.
    std::vector<size_t> acc_off((size_t)n_jobs + 1, 0);
    unsigned long long items = 0;
    std::vector<unsigned long long> item_begin((size_t)n_jobs);
    std::vector<long long> key;
    key.reserve((size_t)n_jobs * 3 + 4);
    for (int j = 0; j < n_jobs; ++j)
    {
        const lg_camera& c = cams[j];
        const lg_render_opts& o = opts[j];
        if (c.width <= 0 || c.height <= 0) return set_error(LG_ERR_INVALID, "job %d: image size %dx%d", j, c.width, c.height);
        if (o.spp < 0 || o.max_bounces < 0) return set_error(LG_ERR_INVALID, "job %d: spp/bounces must be >= 0", j);
        if (o.flags & LG_RENDER_ACCUM64) return set_error(LG_ERR_INVALID, "job %d: FP64 accumulators are per-frame only", j);
        acc_off[(size_t)j + 1] = acc_off[(size_t)j] + (size_t)c.width * c.height * 3;
        item_begin[(size_t)j] = items;
        const unsigned long long tiles = (unsigned long long)((c.width + 7) / 8) * ((c.height + 3) / 4);
        items += tiles * (unsigned long long)((o.spp + 7) / 8) * 32ull;
        key.push_back(c.width);
        key.push_back(c.height);
        key.push_back(o.spp);
    }
    const size_t nval = acc_off[(size_t)n_jobs];
    LG_TRY(r->batch_acc.reserve(nval * sizeof(float)));
    LG_TRY(r->batch_rgb.reserve(nval));
    LG_TRY(r->batch_jobs.reserve((size_t)n_jobs * sizeof(BatchJob)));
    LG_TRY(r->work.reserve(256));
    if (r->batch_host_cap < n_jobs)
    {
        if (r->batch_host) cudaFreeHost(r->batch_host);
        r->batch_host = nullptr;
        r->batch_host_cap = 0;
        LG_TRY_CUDA(cudaMallocHost((void**)&r->batch_host, (size_t)n_jobs * sizeof(BatchJob)));
        r->batch_host_cap = n_jobs;
    }
    // The job table is written into pinned memory that the graph copies from.
    LG_TRY_CUDA(cudaStreamSynchronize(r->stream));
    for (int j = 0; j < n_jobs; ++j)
    {
        BatchJob& b = r->batch_host[j];
        b.cam = make_dev_cam(cams[j]);
        b.item_begin = item_begin[(size_t)j];
        b.accum = r->batch_acc.as<float>() + acc_off[(size_t)j];
        b.spp = opts[j].spp;
        b.max_bounces = opts[j].max_bounces;
        b.sample_base = opts[j].sample_base;
        b.n_chunks = (opts[j].spp + 7) / 8;
        b.tiles_x = (cams[j].width + 7) / 8;
        b.n_tiles = b.tiles_x * ((cams[j].height + 3) / 4);
    }
    // The graph depends on the frame shapes, the scene records, the buffers and the trace options.
    const void* deps[] = {r->batch_acc.p, r->batch_rgb.p, r->batch_jobs.p, r->batch_host, r->wide.p, r->wide4.p,
                          r->tv.p,        r->tris.p,      r->mats.p,       r->texs.p,     r->points.p, r->work.p};
    for (const void* p : deps) key.push_back((long long)(uintptr_t)p);
    key.push_back(r->bvh_width * 2 + (r->watertight ? 1 : 0));
    key.push_back(r->trace_blocks_per_sm);
    key.push_back(r->trace_refill);
    key.push_back(r->trace_quorum);
    key.push_back(r->trace_top);
    key.push_back(r->scene_gen);
    if (key != r->batch_key || !r->batch_exec)
    {
        if (r->batch_exec) cudaGraphExecDestroy(r->batch_exec);
        r->batch_exec = nullptr;
        r->batch_key.clear();
        cudaStream_t st = r->stream;
        LG_TRY_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaMemcpyAsync(r->batch_jobs.p, r->batch_host, (size_t)n_jobs * sizeof(BatchJob),
                                        cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(r->batch_acc.p, 0, nval * sizeof(float), st);
        if (e == cudaSuccess && r->n_nodes > 0 && items > 0)
        {
            TraceJob job{};
            job.work64 = r->work.as<unsigned long long>();
            job.jobs = r->batch_jobs.as<BatchJob>();
            job.n_jobs = n_jobs;
            job.total_items = items;
            job.blocks_per_sm = r->trace_blocks_per_sm;
            job.refill_threshold = r->trace_refill;
            job.leaf_quorum = r->trace_quorum;
            job.top_records = r->trace_top;
            job.stack_safe = stack_safe(r);
            e = launch_trace_batch(dev_scene(r), job, r->sm_count, r->bvh_width, r->watertight, st);
        }
        for (int j = 0; j < n_jobs && e == cudaSuccess; ++j)
            e = launch_tonemap(r->batch_acc.as<float>() + acc_off[(size_t)j], r->batch_rgb.as<uint8_t>() + acc_off[(size_t)j],
                               (long long)(acc_off[(size_t)j + 1] - acc_off[(size_t)j]), 1.0f / (float)opts[j].spp, st);
        if (e == cudaSuccess) e = post_fault(r, st);
        cudaGraph_t graph = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(st, &graph);
        if (e == cudaSuccess) e = ec;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&r->batch_exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (e != cudaSuccess)
        {
            r->batch_exec = nullptr;
            return set_error(LG_ERR_CUDA, "batched render graph: %s", cudaGetErrorString(e));
        }
        r->batch_key = key;
    }
    LG_TRY_CUDA(cudaEventRecord(r->ev0, r->stream));
    LG_TRY_CUDA(cudaGraphLaunch(r->batch_exec, r->stream));
    LG_TRY_CUDA(cudaEventRecord(r->ev1, r->stream));
    if (rgb8_out) LG_TRY_CUDA(cudaMemcpyAsync(rgb8_out, r->batch_rgb.p, nval, cudaMemcpyDeviceToHost, r->stream));
    LG_TRY_CUDA(cudaStreamSynchronize(r->stream));
    LG_TRY(take_fault(r));
    if (ms_per_job)
    {
        // One launch serves all frames: its time is apportioned by work items.
        float ms = 0.0f;
        LG_TRY_CUDA(cudaEventElapsedTime(&ms, r->ev0, r->ev1));
        for (int j = 0; j < n_jobs; ++j)
        {
            const unsigned long long nj = (j + 1 < n_jobs ? item_begin[(size_t)j + 1] : items) - item_begin[(size_t)j];
            ms_per_job[j] = items ? ms * (float)((double)nj / (double)items) : ms / (float)n_jobs;
        }
    }
    return LG_OK;
}

int lg_render_gbuffer(lg_renderer* r, const lg_camera* cam, uint8_t* albedo, uint8_t* normal, uint8_t* worldpos)
{
    if (!r || !cam) return set_error(LG_ERR_INVALID, "NULL argument");
    if (cam->width <= 0 || cam->height <= 0) return set_error(LG_ERR_INVALID, "image size %dx%d", cam->width, cam->height);
    DeviceGuard g(r->device);
    const size_t n = (size_t)cam->width * cam->height * 3;
    LG_TRY(r->gbuf.reserve(3 * n));
    uint8_t* base = r->gbuf.as<uint8_t>();
    if (r->n_nodes == 0)
    {
        // nothing to hit: every pixel is a miss
        LG_TRY_CUDA(cudaMemsetAsync(base, 0, 3 * n, r->stream));
        std::vector<uint8_t> miss(n);
        for (size_t i = 0; i < n; i += 3) { miss[i] = 128; miss[i + 1] = 128; miss[i + 2] = 255; }
        LG_TRY_CUDA(cudaMemcpyAsync(base + n, miss.data(), n, cudaMemcpyHostToDevice, r->stream));
    }
    else
    {
        // Scene box from the BVH root, inverse extent clamped at 1e-6 (pathtracer.cu:728-734).
        const lg_bvh_node& root = r->root_node;
        const vec3 bbMin = v3(root.bbMin[0], root.bbMin[1], root.bbMin[2]);
        const vec3 ext = vsub(v3(root.bbMax[0], root.bbMax[1], root.bbMax[2]), bbMin);
        const vec3 inv = v3(1.0f / std::max(ext.x, 1e-6f), 1.0f / std::max(ext.y, 1e-6f), 1.0f / std::max(ext.z, 1e-6f));
        LG_TRY_CUDA(launch_gbuffer(dev_scene(r), make_dev_cam(*cam), bbMin, inv, base, base + n, base + 2 * n,
                                   r->bvh_width, r->watertight, r->stream));
        LG_TRY_CUDA(post_fault(r, r->stream));
    }
    if (albedo) LG_TRY_CUDA(cudaMemcpyAsync(albedo, base, n, cudaMemcpyDeviceToHost, r->stream));
    if (normal) LG_TRY_CUDA(cudaMemcpyAsync(normal, base + n, n, cudaMemcpyDeviceToHost, r->stream));
    if (worldpos) LG_TRY_CUDA(cudaMemcpyAsync(worldpos, base + 2 * n, n, cudaMemcpyDeviceToHost, r->stream));
    LG_TRY_CUDA(cudaStreamSynchronize(r->stream));
    LG_TRY(take_fault(r));
    return LG_OK;
}

int lg_tonemap_device(const float* d_accum, uint8_t* d_rgb8, int64_t n_pixels, float inv_spp, void* stream)
{
    if ((!d_accum || !d_rgb8) && n_pixels > 0) return set_error(LG_ERR_INVALID, "NULL argument");
    LG_TRY_CUDA(launch_tonemap(d_accum, d_rgb8, (long long)n_pixels * 3, inv_spp, (cudaStream_t)stream));
    return LG_OK;
}

int lg_write_png(const char* path, int32_t w, int32_t h, const uint8_t* rgb8)
{
    if (!path || !rgb8) return set_error(LG_ERR_INVALID, "NULL argument");
    if (!write_png(path, w, h, rgb8)) return set_error(LG_ERR_IO, "failed to write %s", path);
    return LG_OK;
}

int lg_write_hdr(const char* path, int32_t w, int32_t h, const float* rgb32)
{
    if (!path || !rgb32) return set_error(LG_ERR_INVALID, "NULL argument");
    if (!write_hdr(path, w, h, rgb32)) return set_error(LG_ERR_IO, "failed to write %s", path);
    return LG_OK;
}

}  // extern "C"

// ---- C++ drop-ins ----
void BuildBVH(Scene& scene, Bvh& out)
{
    out.nodes.clear();
    out.rootIdx = 0;
    const int n = (int)scene.triangles.size();
    if (n == 0) return;
    out.nodes.resize((size_t)(2 * n - 1));
    int count = 0;
    lg_triangle* tris = reinterpret_cast<lg_triangle*>(scene.triangles.data());
    int rc = lg_build_bvh(tris, n, reinterpret_cast<lg_bvh_node*>(out.nodes.data()), &count, nullptr, tris);
    if (rc != LG_OK)
    {
        std::fprintf(stderr, "BuildBVH: %s\n", lg_last_error());
        out.nodes.clear();
        return;
    }
    out.nodes.resize((size_t)count);
}

namespace
{
lg_camera camera_of(const Scene& s)
{
    lg_camera c;
    std::memcpy(c.pos, s.camera.pos, sizeof c.pos);
    std::memcpy(c.camera_to_world, s.camera.cameraToWorld, sizeof c.camera_to_world);
    c.fov_y_deg = s.camera.fovYDeg;
    c.aspect = s.camera.aspect;
    c.near_z = s.camera.nearZ;
    c.far_z = s.camera.farZ;
    c.width = s.camera.imageWidth;
    c.height = s.camera.imageHeight;
    return c;
}
lg_scene_desc desc_of(const Scene& s, std::vector<float>& alb)
{
    lg_scene_desc d{};
    d.camera = camera_of(s);
    std::memcpy(&d.sun, &s.sun, sizeof d.sun);
    d.tris = reinterpret_cast<const lg_triangle*>(s.triangles.data());
    d.n_tris = (int32_t)s.triangles.size();
    alb.resize(s.materials.size() * 3);
    for (size_t i = 0; i < s.materials.size(); ++i)
        for (int k = 0; k < 3; ++k) alb[3 * i + k] = s.materials[i].albedo[k];
    d.mat_albedo = alb.data();
    d.n_mats = (int32_t)s.materials.size();
    d.points = reinterpret_cast<const lg_point_light*>(s.points.data());
    d.n_points = (int32_t)s.points.size();
    return d;
}

// A renderer holding `scene` with the caller's BVH and the scene's textures
// resolved against assetRoot, reported as the reference reports them
// (pathtracer.cu:597-613).  Returns LG_OK or the failing call's status.
int open_renderer(const Scene& scene, const Bvh& bvh, const std::string& assetRoot, lg_scene_desc& d,
                  std::vector<float>& alb, lg_renderer** out)
{
    d = desc_of(scene, alb);
    int dev = 0;
    cudaGetDevice(&dev);
    int rc = lg_renderer_create(dev, out);
    // CUDAREF_L2_PIN=1: the reference's knob for a persisting-L2 window over
    // the BVH (pathtracer.cu:675-693)
    const char* pin = std::getenv("CUDAREF_L2_PIN");
    if (rc == LG_OK && pin && std::atoi(pin)) rc = lg_renderer_set_l2_window(*out, 1);
    if (rc == LG_OK)
        rc = lg_renderer_set_scene_bvh(*out, &d, reinterpret_cast<const lg_bvh_node*>(bvh.nodes.data()),
                                       (int32_t)bvh.nodes.size());
    if (rc != LG_OK) return rc;
    int loaded = 0, missing = 0;
    for (size_t m = 0; m < scene.materials.size() && rc == LG_OK; ++m)
    {
        const std::string& rel = scene.materials[m].diffuseTex;
        if (rel.empty()) continue;
        const std::string full = assetRoot + "/" + rel;
        int32_t w = 0, h = 0;
        uint8_t* px = nullptr;
        if (lg_image_load(full.c_str(), &w, &h, &px) != LG_OK)
        {
            std::fprintf(stderr, "  texture not found: %s\n", full.c_str());
            ++missing;
            continue;
        }
        rc = lg_renderer_set_texture(*out, (int)m, px, w, h);
        lg_image_free(px);
        ++loaded;
    }
    std::printf("textures: %d loaded, %d missing (of %zu materials)\n", loaded, missing, scene.materials.size());
    return rc;
}
}  // namespace

// Same signature as the reference (declared in its main.cpp:19-24).  The
// G-buffer images are produced when all three outputs are given (as the
// reference does, pathtracer.cu:726-747).
void RenderSceneCUDA(const Scene& scene, const Bvh& bvh, const std::string& assetRoot, int spp, int maxBounces,
                     std::vector<uint8_t>& outRGB, int& outW, int& outH, std::vector<uint8_t>* outAlbedo,
                     std::vector<uint8_t>* outNormal, std::vector<uint8_t>* outWorldPos)
{
    outW = scene.camera.imageWidth;
    outH = scene.camera.imageHeight;
    outRGB.assign((size_t)outW * outH * 3, 0);
    for (auto* v : {outAlbedo, outNormal, outWorldPos})
        if (v) v->assign((size_t)outW * outH * 3, 0);
    std::vector<float> alb;
    lg_scene_desc d{};
    lg_renderer* r = nullptr;
    int rc = open_renderer(scene, bvh, assetRoot, d, alb, &r);
    lg_render_stats st{};
    if (rc == LG_OK)
    {
        lg_render_opts o{spp, maxBounces, 0, 0};
        lg_camera cam = d.camera;
        rc = lg_render(r, &cam, &o, outRGB.data(), nullptr, nullptr, &st);
    }
    if (rc != LG_OK) std::fprintf(stderr, "render failed: %s\n", lg_last_error());
    else
        std::printf("kernel: %.1f ms  (%d x %d, %d spp, %d bounces, %zu tris)\n", st.kernel_ms, outW, outH, spp,
                    maxBounces, scene.triangles.size());
    if (rc == LG_OK && outAlbedo && outNormal && outWorldPos)
    {
        lg_camera cam = d.camera;
        rc = lg_render_gbuffer(r, &cam, outAlbedo->data(), outNormal->data(), outWorldPos->data());
        if (rc != LG_OK) std::fprintf(stderr, "gbuffer failed: %s\n", lg_last_error());
    }
    lg_renderer_destroy(r);
}

// Same signature as the reference (declared in its main.cpp:25-27; defined
// at pathtracer.cu:759-909): the ray-sorted render, lg_render_sorted.
void RenderSceneCUDASorted(const Scene& scene, const Bvh& bvh, const std::string& assetRoot, int spp, int maxBounces,
                           std::vector<uint8_t>& outRGB, int& outW, int& outH)
{
    outW = scene.camera.imageWidth;
    outH = scene.camera.imageHeight;
    outRGB.assign((size_t)outW * outH * 3, 0);
    std::vector<float> alb;
    lg_scene_desc d{};
    lg_renderer* r = nullptr;
    int rc = open_renderer(scene, bvh, assetRoot, d, alb, &r);
    lg_render_stats st{};
    if (rc == LG_OK)
    {
        lg_render_opts o{spp, maxBounces, 0, 0};
        lg_camera cam = d.camera;
        rc = lg_render_sorted(r, &cam, &o, outRGB.data(), nullptr, &st);
    }
    if (rc != LG_OK) std::fprintf(stderr, "render failed: %s\n", lg_last_error());
    else
        std::printf("kernel (sorted): %.1f ms  (%d x %d, %d spp, %d bounces, %zu tris)\n", st.kernel_ms, outW, outH,
                    spp, maxBounces, scene.triangles.size());
    lg_renderer_destroy(r);
}
