// ref_harness.cu -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// Compiles the reference renderer's own source (src/pathtracer.cu of
// LuminaGI-CudaRef, included from the reference checkout at build time; no
// reference source is copied into this repository) twice over:
//   * its __device__ trace functions are re-annotated __host__ __device__ so
//     they also build for the CPU (OpenMP over rows) -- the CPU baseline and
//     the CPU render oracle;
//   * its accumulate_kernel / tonemap_kernel are launched on the GPU exactly
//     as RenderSceneCUDA does (pathtracer.cu:646-706), reading back the FP32
//     accumulator that RenderSceneCUDA itself never returns -- the GPU render
//     oracle ("reference design on B200").
// bvh.cpp and scene_loader.cpp are linked in unchanged and exposed through
// the extern "C" wrappers below.  Built by oracle/Makefile into oracle/_ref/.
//
// Only tests/, __graft_entry__.smoke() and bench.py (cpu_baseline leg and the
// reference arm) may load the resulting library.
#include <cuda_runtime.h>
#include <thrust/device_ptr.h>
#include <thrust/sort.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <omp.h>

// The reference samples textures with tex2D, which has no host version.
// Synthetic scenes are untextured (tex == 0), so the host side never calls it.
template <class T>
__host__ __device__ inline T lgref_tex2D(cudaTextureObject_t t, float x, float y)
{
#ifdef __CUDA_ARCH__
    return tex2D<T>(t, x, y);
#else
    (void)t; (void)x; (void)y;
    return T{};
#endif
}

#undef __device__
#define __device__ __host__ __location__(device)
#define tex2D lgref_tex2D
#include REF_PATHTRACER_CU
#undef tex2D
#undef __device__
#define __device__ __location__(device)

namespace
{
// Camera set-up as RenderSceneCUDA performs it (pathtracer.cu:654-663).
CameraGPU make_cam(const CameraDesc& c)
{
    CameraGPU cam{};
    cam.pos = vfrom(c.pos);
    const float* m = c.cameraToWorld;
    cam.fwd = v3(m[0], m[1], m[2]);
    cam.left = v3(m[4], m[5], m[6]);
    cam.up = v3(m[8], m[9], m[10]);
    cam.tanHalfFov = tanf(c.fovYDeg * 0.5f * 3.14159265358979f / 180.0f);
    cam.aspect = c.aspect;
    cam.width = c.imageWidth;
    cam.height = c.imageHeight;
    return cam;
}

std::vector<DeviceMaterial> make_mats(const float* albedo, const float* emissive, int nMats)
{
    std::vector<DeviceMaterial> m((size_t)nMats);
    for (int i = 0; i < nMats; ++i)
    {
        for (int k = 0; k < 3; ++k)
        {
            m[i].albedo[k] = albedo[3 * i + k];
            m[i].emissive[k] = emissive ? emissive[3 * i + k] : 0.0f;
        }
        m[i].tex = 0;
    }
    return m;
}
}  // namespace

extern "C" {

// ---- scene loader (reference src/scene_loader.cpp) ----
void* ref_scene_load(const char* path)
{
    Scene* s = new Scene();
    if (!LoadSceneJSON(path, *s)) { delete s; return nullptr; }
    return s;
}

void ref_scene_counts(void* h, int* nTris, int* nMats, int* nPoints, int* nDirs)
{
    const Scene* s = (const Scene*)h;
    *nTris = (int)s->triangles.size();
    *nMats = (int)s->materials.size();
    *nPoints = (int)s->points.size();
    *nDirs = (int)s->directionals.size();
}

void ref_scene_get(void* h, CameraDesc* cam, DirectionalLight* sun, Triangle* tris, float* matAlbedo,
                   float* matEmissive, PointLight* points, DirectionalLight* dirs)
{
    const Scene* s = (const Scene*)h;
    *cam = s->camera;
    *sun = s->sun;
    if (!s->triangles.empty()) std::memcpy(tris, s->triangles.data(), s->triangles.size() * sizeof(Triangle));
    for (size_t i = 0; i < s->materials.size(); ++i)
        for (int k = 0; k < 3; ++k)
        {
            matAlbedo[3 * i + k] = s->materials[i].albedo[k];
            matEmissive[3 * i + k] = s->materials[i].emissive[k];
        }
    for (size_t i = 0; i < s->points.size(); ++i) points[i] = s->points[i];
    for (size_t i = 0; i < s->directionals.size(); ++i) dirs[i] = s->directionals[i];
}

void ref_scene_free(void* h) { delete (Scene*)h; }

// ---- BVH (reference src/bvh.cpp:164-211, single-threaded as shipped) ----
// outTris receives scene.triangles after BuildBVH's in-place reorder.
int ref_build_bvh(const Triangle* tris, int n, BvhNode* outNodes, int cap, int* outCount, Triangle* outTris)
{
    Scene s;
    s.triangles.assign(tris, tris + n);
    Bvh b;
    BuildBVH(s, b);
    *outCount = (int)b.nodes.size();
    if ((int)b.nodes.size() > cap) return -1;
    if (!b.nodes.empty()) std::memcpy(outNodes, b.nodes.data(), b.nodes.size() * sizeof(BvhNode));
    if (outTris && n) std::memcpy(outTris, s.triangles.data(), (size_t)n * sizeof(Triangle));
    return 0;
}

// ---- CPU render: accumulate_kernel's per-pixel body (pathtracer.cu:349-363)
// replayed over rows rowStart, rowStart+rowStep, ... with OpenMP.
// accum must hold W*H*3 floats and is added to (not cleared).
int ref_trace_cpu(const BvhNode* nodes, const Triangle* tris, const float* matAlbedo, const float* matEmissive,
                  int nMats, const PointLight* points, int nPoints, const DirectionalLight* sun,
                  const CameraDesc* camDesc, int spp, int maxBounces, int rowStart, int rowStep, int threads,
                  float* accum)
{
    std::vector<DeviceMaterial> mats = make_mats(matAlbedo, matEmissive, nMats);
    DeviceScene s{};
    s.nodes = nodes;
    s.tris = tris;
    s.mats = mats.data();
    s.points = points;
    s.numPoints = nPoints;
    s.sun = *sun;
    const CameraGPU cam = make_cam(*camDesc);
    const int W = cam.width, H = cam.height;
    if (rowStep < 1) rowStep = 1;
    const int nRows = rowStart < H ? (H - rowStart + rowStep - 1) / rowStep : 0;
    if (threads > 0) omp_set_num_threads(threads);
    const int kChunk = 8;
#pragma omp parallel for schedule(dynamic, 1)
    for (int r = 0; r < nRows; ++r)
    {
        const int py = rowStart + r * rowStep;
        for (int px = 0; px < W; ++px)
        {
            for (int base = 0; base < spp; base += kChunk)
            {
                const int thisLaunch = (spp - base < kChunk) ? (spp - base) : kChunk;
                uint32_t rng = (uint32_t)(px * 1973 + py * 9277 + base * 26699) | 1u;
                vec3 sum = v3(0, 0, 0);
                for (int k = 0; k < thisLaunch; ++k)
                {
                    float jx = randf(rng);
                    float jy = randf(rng);
                    Ray ray = primary_ray(cam, px, py, jx, jy);
                    sum = vadd(sum, trace_path(s, nullptr, ray, maxBounces, rng));
                }
                const size_t i = ((size_t)py * W + px) * 3;
                accum[i + 0] += sum.x;
                accum[i + 1] += sum.y;
                accum[i + 2] += sum.z;
            }
        }
    }
    return 0;
}

int ref_omp_max_threads(void) { return omp_get_max_threads(); }

// ---- textures: per-material file paths used by the GPU entry points below
// (load_texture_to_device, pathtracer.cu:553-579, on each non-empty path).
static std::vector<std::string> g_texPaths;

void ref_set_textures(int nMats, const char* const* paths)
{
    g_texPaths.assign((size_t)(nMats > 0 ? nMats : 0), std::string());
    for (int i = 0; i < nMats && paths; ++i)
        if (paths[i]) g_texPaths[(size_t)i] = paths[i];
}

// stbi_load(path, &w, &h, &n, 4) as the reference calls it; *out is freed with ref_image_free.
int ref_image_load(const char* path, int* w, int* h, unsigned char** out)
{
    int n = 0;
    *out = stbi_load(path, w, h, &n, 4);
    return *out ? 0 : 1;
}

void ref_image_free(unsigned char* p) { stbi_image_free(p); }

// ---- GPU render with the reference kernels, launched as RenderSceneCUDA
// launches them.  The node buffer is padded to at least 255 nodes because
// accumulate_kernel stages nodes[0..254] into shared memory unconditionally
// (pathtracer.cu:341-342).  accumHost (W*H*3 floats) and rgbHost (W*H*3
// bytes) may be null.  Returns 0 or a CUDA error code.
int ref_render_gpu(const BvhNode* nodes, int nNodes, const Triangle* tris, int nTris, const float* matAlbedo,
                   const float* matEmissive, int nMats, const PointLight* points, int nPoints,
                   const DirectionalLight* sun, const CameraDesc* camDesc, int spp, int maxBounces,
                   float* accumHost, uint8_t* rgbHost, float* kernelMs)
{
#define RCHK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { rc = (int)e_; goto done; } } while (0)
    int rc = 0;
    std::vector<DeviceMaterial> mats = make_mats(matAlbedo, matEmissive, nMats);
    std::vector<cudaArray_t> texArrays((size_t)(nMats > 0 ? nMats : 0), nullptr);
    for (int i = 0; i < nMats && i < (int)g_texPaths.size(); ++i)
        if (!g_texPaths[(size_t)i].empty() && !load_texture_to_device(g_texPaths[(size_t)i], texArrays[(size_t)i], mats[(size_t)i].tex))
            mats[(size_t)i].tex = 0;
    const CameraGPU cam = make_cam(*camDesc);
    const int W = cam.width, H = cam.height;
    const int nPad = nNodes < kShmemBvhNodes ? kShmemBvhNodes : nNodes;
    BvhNode* d_nodes = nullptr;
    Triangle* d_tris = nullptr;
    DeviceMaterial* d_mats = nullptr;
    PointLight* d_points = nullptr;
    float* d_accum = nullptr;
    uint8_t* d_image = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    DeviceScene s{};
    dim3 block(16, 16);
    dim3 grid((W + 15) / 16, (H + 15) / 16);
    RCHK(cudaMalloc(&d_nodes, (size_t)nPad * sizeof(BvhNode)));
    RCHK(cudaMemset(d_nodes, 0, (size_t)nPad * sizeof(BvhNode)));
    RCHK(cudaMemcpy(d_nodes, nodes, (size_t)nNodes * sizeof(BvhNode), cudaMemcpyHostToDevice));
    RCHK(cudaMalloc(&d_tris, (size_t)(nTris > 0 ? nTris : 1) * sizeof(Triangle)));
    if (nTris) RCHK(cudaMemcpy(d_tris, tris, (size_t)nTris * sizeof(Triangle), cudaMemcpyHostToDevice));
    RCHK(cudaMalloc(&d_mats, (size_t)(nMats > 0 ? nMats : 1) * sizeof(DeviceMaterial)));
    if (nMats) RCHK(cudaMemcpy(d_mats, mats.data(), (size_t)nMats * sizeof(DeviceMaterial), cudaMemcpyHostToDevice));
    if (nPoints)
    {
        RCHK(cudaMalloc(&d_points, (size_t)nPoints * sizeof(PointLight)));
        RCHK(cudaMemcpy(d_points, points, (size_t)nPoints * sizeof(PointLight), cudaMemcpyHostToDevice));
    }
    RCHK(cudaMalloc(&d_accum, (size_t)W * H * 3 * sizeof(float)));
    RCHK(cudaMemset(d_accum, 0, (size_t)W * H * 3 * sizeof(float)));
    RCHK(cudaMalloc(&d_image, (size_t)W * H * 3));
    s.nodes = d_nodes;
    s.tris = d_tris;
    s.mats = d_mats;
    s.points = d_points;
    s.numPoints = nPoints;
    s.sun = *sun;
    RCHK(cudaEventCreate(&t0));
    RCHK(cudaEventCreate(&t1));
    RCHK(cudaEventRecord(t0));
    for (int base = 0; base < spp; base += 8)
    {
        const int thisLaunch = (spp - base < 8) ? (spp - base) : 8;
        accumulate_kernel<<<grid, block>>>(s, cam, d_accum, thisLaunch, base, maxBounces);
        RCHK(cudaGetLastError());
    }
    tonemap_kernel<<<grid, block>>>(d_accum, d_image, W, H, 1.0f / (float)spp);
    RCHK(cudaGetLastError());
    RCHK(cudaEventRecord(t1));
    RCHK(cudaEventSynchronize(t1));
    if (kernelMs) RCHK(cudaEventElapsedTime(kernelMs, t0, t1));
    if (accumHost) RCHK(cudaMemcpy(accumHost, d_accum, (size_t)W * H * 3 * sizeof(float), cudaMemcpyDeviceToHost));
    if (rgbHost) RCHK(cudaMemcpy(rgbHost, d_image, (size_t)W * H * 3, cudaMemcpyDeviceToHost));
done:
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFree(d_nodes);
    cudaFree(d_tris);
    cudaFree(d_mats);
    cudaFree(d_points);
    cudaFree(d_accum);
    cudaFree(d_image);
    for (size_t i = 0; i < texArrays.size(); ++i)
        if (texArrays[i]) { cudaDestroyTextureObject(mats[i].tex); cudaFreeArray(texArrays[i]); }
    return rc;
#undef RCHK
}

// ---- The reference's ray-sorted render, launched as RenderSceneCUDASorted
// launches it (pathtracer.cu:838-890: per sample gen_primary_kernel, a
// thrust::sort_by_key of the rays by direction key, then per bounce
// trace_and_bounce_kernel and a sort of the next rays), reading back the FP32
// accumulator it never returns.  Untextured scenes; node buffer padded to
// 255 nodes because trace_and_bounce_kernel stages nodes[0..254] into shared
// memory (pathtracer.cu:492-494).
int ref_render_sorted_gpu(const BvhNode* nodes, int nNodes, const Triangle* tris, int nTris, const float* matAlbedo,
                          const float* matEmissive, int nMats, const PointLight* points, int nPoints,
                          const DirectionalLight* sun, const CameraDesc* camDesc, int spp, int maxBounces,
                          float* accumHost, uint8_t* rgbHost, float* kernelMs)
{
#define RCHK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { rc = (int)e_; goto done; } } while (0)
    int rc = 0;
    std::vector<DeviceMaterial> mats = make_mats(matAlbedo, matEmissive, nMats);
    const CameraGPU cam = make_cam(*camDesc);
    const int W = cam.width, H = cam.height, N = W * H;
    const int nPad = nNodes < kShmemBvhNodes ? kShmemBvhNodes : nNodes;
    BvhNode* d_nodes = nullptr;
    Triangle* d_tris = nullptr;
    DeviceMaterial* d_mats = nullptr;
    PointLight* d_points = nullptr;
    float* d_accum = nullptr;
    uint8_t* d_image = nullptr;
    SortedRay *d_raysA = nullptr, *d_raysB = nullptr;
    uint32_t *d_keysA = nullptr, *d_keysB = nullptr, *d_rng = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    DeviceScene s{};
    dim3 block2d(16, 16);
    dim3 grid2d((W + 15) / 16, (H + 15) / 16);
    const int grid1d = (N + 255) / 256;
    RCHK(cudaMalloc(&d_nodes, (size_t)nPad * sizeof(BvhNode)));
    RCHK(cudaMemset(d_nodes, 0, (size_t)nPad * sizeof(BvhNode)));
    RCHK(cudaMemcpy(d_nodes, nodes, (size_t)nNodes * sizeof(BvhNode), cudaMemcpyHostToDevice));
    RCHK(cudaMalloc(&d_tris, (size_t)(nTris > 0 ? nTris : 1) * sizeof(Triangle)));
    if (nTris) RCHK(cudaMemcpy(d_tris, tris, (size_t)nTris * sizeof(Triangle), cudaMemcpyHostToDevice));
    RCHK(cudaMalloc(&d_mats, (size_t)(nMats > 0 ? nMats : 1) * sizeof(DeviceMaterial)));
    if (nMats) RCHK(cudaMemcpy(d_mats, mats.data(), (size_t)nMats * sizeof(DeviceMaterial), cudaMemcpyHostToDevice));
    if (nPoints)
    {
        RCHK(cudaMalloc(&d_points, (size_t)nPoints * sizeof(PointLight)));
        RCHK(cudaMemcpy(d_points, points, (size_t)nPoints * sizeof(PointLight), cudaMemcpyHostToDevice));
    }
    RCHK(cudaMalloc(&d_accum, (size_t)N * 3 * sizeof(float)));
    RCHK(cudaMemset(d_accum, 0, (size_t)N * 3 * sizeof(float)));
    RCHK(cudaMalloc(&d_image, (size_t)N * 3));
    RCHK(cudaMalloc(&d_raysA, (size_t)N * sizeof(SortedRay)));
    RCHK(cudaMalloc(&d_raysB, (size_t)N * sizeof(SortedRay)));
    RCHK(cudaMalloc(&d_keysA, (size_t)N * sizeof(uint32_t)));
    RCHK(cudaMalloc(&d_keysB, (size_t)N * sizeof(uint32_t)));
    RCHK(cudaMalloc(&d_rng, (size_t)N * sizeof(uint32_t)));
    s.nodes = d_nodes;
    s.tris = d_tris;
    s.mats = d_mats;
    s.points = d_points;
    s.numPoints = nPoints;
    s.sun = *sun;
    RCHK(cudaEventCreate(&t0));
    RCHK(cudaEventCreate(&t1));
    RCHK(cudaEventRecord(t0));
    for (int sample = 0; sample < spp; ++sample)
    {
        gen_primary_kernel<<<grid2d, block2d>>>(cam, d_raysA, d_keysA, d_rng, sample);
        RCHK(cudaGetLastError());
        thrust::sort_by_key(thrust::device_ptr<uint32_t>(d_keysA), thrust::device_ptr<uint32_t>(d_keysA + N),
                            thrust::device_ptr<SortedRay>(d_raysA));
        for (int b = 0; b <= maxBounces; ++b)
        {
            const bool last = (b == maxBounces);
            trace_and_bounce_kernel<<<grid1d, 256>>>(s, d_raysA, (uint32_t)N, d_accum, last ? nullptr : d_raysB,
                                                      last ? nullptr : d_keysB, d_rng, last);
            RCHK(cudaGetLastError());
            if (last) break;
            thrust::sort_by_key(thrust::device_ptr<uint32_t>(d_keysB), thrust::device_ptr<uint32_t>(d_keysB + N),
                                thrust::device_ptr<SortedRay>(d_raysB));
            std::swap(d_raysA, d_raysB);
            std::swap(d_keysA, d_keysB);
        }
    }
    tonemap_kernel<<<grid2d, block2d>>>(d_accum, d_image, W, H, 1.0f / (float)spp);
    RCHK(cudaGetLastError());
    RCHK(cudaEventRecord(t1));
    RCHK(cudaEventSynchronize(t1));
    if (kernelMs) RCHK(cudaEventElapsedTime(kernelMs, t0, t1));
    if (accumHost) RCHK(cudaMemcpy(accumHost, d_accum, (size_t)N * 3 * sizeof(float), cudaMemcpyDeviceToHost));
    if (rgbHost) RCHK(cudaMemcpy(rgbHost, d_image, (size_t)N * 3, cudaMemcpyDeviceToHost));
done:
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFree(d_nodes);
    cudaFree(d_tris);
    cudaFree(d_mats);
    cudaFree(d_points);
    cudaFree(d_accum);
    cudaFree(d_image);
    cudaFree(d_raysA);
    cudaFree(d_raysB);
    cudaFree(d_keysA);
    cudaFree(d_keysB);
    cudaFree(d_rng);
    return rc;
#undef RCHK
}

// ---- G-buffer with the reference gbuffer_kernel, box from the root node as
// RenderSceneCUDA computes it (pathtracer.cu:726-747).  Node buffer padded as above.
int ref_gbuffer_gpu(const BvhNode* nodes, int nNodes, const Triangle* tris, int nTris, const float* matAlbedo,
                    const float* matEmissive, int nMats, const PointLight* points, int nPoints,
                    const DirectionalLight* sun, const CameraDesc* camDesc, uint8_t* albHost, uint8_t* nrmHost,
                    uint8_t* wpHost)
{
#define RCHK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { rc = (int)e_; goto done; } } while (0)
    int rc = 0;
    std::vector<DeviceMaterial> mats = make_mats(matAlbedo, matEmissive, nMats);
    std::vector<cudaArray_t> texArrays((size_t)(nMats > 0 ? nMats : 0), nullptr);
    for (int i = 0; i < nMats && i < (int)g_texPaths.size(); ++i)
        if (!g_texPaths[(size_t)i].empty() && !load_texture_to_device(g_texPaths[(size_t)i], texArrays[(size_t)i], mats[(size_t)i].tex))
            mats[(size_t)i].tex = 0;
    const CameraGPU cam = make_cam(*camDesc);
    const int W = cam.width, H = cam.height;
    const size_t imgBytes = (size_t)W * H * 3;
    const int nPad = nNodes < kShmemBvhNodes ? kShmemBvhNodes : nNodes;
    BvhNode* d_nodes = nullptr;
    Triangle* d_tris = nullptr;
    DeviceMaterial* d_mats = nullptr;
    PointLight* d_points = nullptr;
    uint8_t *d_alb = nullptr, *d_nrm = nullptr, *d_wp = nullptr;
    DeviceScene s{};
    dim3 block(16, 16);
    dim3 grid((W + 15) / 16, (H + 15) / 16);
    const BvhNode& root = nodes[0];
    vec3 bbMin = v3(root.bbMin[0], root.bbMin[1], root.bbMin[2]);
    vec3 bbMax = v3(root.bbMax[0], root.bbMax[1], root.bbMax[2]);
    vec3 ext = vsub(bbMax, bbMin);
    vec3 invExt = v3(1.0f / fmaxf(ext.x, 1e-6f), 1.0f / fmaxf(ext.y, 1e-6f), 1.0f / fmaxf(ext.z, 1e-6f));
    RCHK(cudaMalloc(&d_nodes, (size_t)nPad * sizeof(BvhNode)));
    RCHK(cudaMemset(d_nodes, 0, (size_t)nPad * sizeof(BvhNode)));
    RCHK(cudaMemcpy(d_nodes, nodes, (size_t)nNodes * sizeof(BvhNode), cudaMemcpyHostToDevice));
    RCHK(cudaMalloc(&d_tris, (size_t)(nTris > 0 ? nTris : 1) * sizeof(Triangle)));
    if (nTris) RCHK(cudaMemcpy(d_tris, tris, (size_t)nTris * sizeof(Triangle), cudaMemcpyHostToDevice));
    RCHK(cudaMalloc(&d_mats, (size_t)(nMats > 0 ? nMats : 1) * sizeof(DeviceMaterial)));
    if (nMats) RCHK(cudaMemcpy(d_mats, mats.data(), (size_t)nMats * sizeof(DeviceMaterial), cudaMemcpyHostToDevice));
    if (nPoints)
    {
        RCHK(cudaMalloc(&d_points, (size_t)nPoints * sizeof(PointLight)));
        RCHK(cudaMemcpy(d_points, points, (size_t)nPoints * sizeof(PointLight), cudaMemcpyHostToDevice));
    }
    RCHK(cudaMalloc(&d_alb, imgBytes));
    RCHK(cudaMalloc(&d_nrm, imgBytes));
    RCHK(cudaMalloc(&d_wp, imgBytes));
    s.nodes = d_nodes;
    s.tris = d_tris;
    s.mats = d_mats;
    s.points = d_points;
    s.numPoints = nPoints;
    s.sun = *sun;
    gbuffer_kernel<<<grid, block>>>(s, cam, bbMin, invExt, d_alb, d_nrm, d_wp);
    RCHK(cudaGetLastError());
    RCHK(cudaDeviceSynchronize());
    RCHK(cudaMemcpy(albHost, d_alb, imgBytes, cudaMemcpyDeviceToHost));
    RCHK(cudaMemcpy(nrmHost, d_nrm, imgBytes, cudaMemcpyDeviceToHost));
    RCHK(cudaMemcpy(wpHost, d_wp, imgBytes, cudaMemcpyDeviceToHost));
done:
    cudaFree(d_nodes);
    cudaFree(d_tris);
    cudaFree(d_mats);
    cudaFree(d_points);
    cudaFree(d_alb);
    cudaFree(d_nrm);
    cudaFree(d_wp);
    for (size_t i = 0; i < texArrays.size(); ++i)
        if (texArrays[i]) { cudaDestroyTextureObject(mats[i].tex); cudaFreeArray(texArrays[i]); }
    return rc;
#undef RCHK
}

}  // extern "C"
