// cuda_ref -- command-line renderer, drop-in for the reference's src/main.cpp.
//
//   cuda_ref <scene.json> [output.png] [--spp N] [--bounces N] [--asset-root DIR]
//            [-o out.png] [--cam-pos x y z --cam-target x y z] [--batch FILE]
//            [--sort] [--gbuffer] [--hdr out.hdr] [--device N]
//
// Flags, defaults (output/reference.png, 64 spp, 2 bounces), the batch file
// format ("out_png spp bounces camx camy camz tgtx tgty tgtz", '#' comments,
// malformed lines skipped), the stdout lines ("bvh: ...", "kernel: ...",
// "render: ...", "wrote ...", "[k/n] ... render=... ms") and the exit codes
// (1 usage, 2 scene load, 3 PNG write) follow main.cpp:93-229.  The scene is
// uploaded and its BVH built on the device once; batch jobs only change the
// camera.  --sort renders the single frame with the ray-sorted wavefront
// (lg_render_sorted, RenderSceneCUDASorted's semantics: per-sample seeding,
// no Russian roulette, rays sorted by direction between bounces) and prints
// "kernel (sorted): ..."; batch jobs ignore it, as main.cpp:158-190 does.
// Diffuse textures resolve against --asset-root (default: the scene file's
// grandparent directory, main.cpp:140-141).  --gbuffer also writes <stem>.albedo.png, <stem>.normal.png and
// <stem>.worldpos.png (main.cpp:177-184, 220-227).  --hdr additionally writes
// the linear radiance (accum / spp).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "lumina.h"

namespace
{
struct BatchJob
{
    std::string out_png;
    int spp = 0, bounces = 0;
    float cam_pos[3] = {0, 0, 0};
    float cam_tgt[3] = {0, 0, 0};
};

std::vector<BatchJob> read_batch_file(const std::string& path)
{
    std::vector<BatchJob> jobs;
    std::ifstream in(path);
    if (!in)
    {
        std::fprintf(stderr, "can't open batch file: %s\n", path.c_str());
        return jobs;
    }
    std::string line;
    while (std::getline(in, line))
    {
        auto hash = line.find('#');
        if (hash != std::string::npos) line.erase(hash);
        std::istringstream ss(line);
        BatchJob j;
        if (!(ss >> j.out_png >> j.spp >> j.bounces >> j.cam_pos[0] >> j.cam_pos[1] >> j.cam_pos[2] >> j.cam_tgt[0] >>
              j.cam_tgt[1] >> j.cam_tgt[2]))
            continue;
        jobs.push_back(j);
    }
    return jobs;
}

double ms_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// <dir>/<stem>.albedo.png etc. next to the colour image.
void write_gbuffer(lg_renderer* r, const lg_camera& cam, const std::string& png)
{
    const size_t n = (size_t)cam.width * cam.height * 3;
    std::vector<uint8_t> alb(n), nrm(n), wp(n);
    if (lg_render_gbuffer(r, &cam, alb.data(), nrm.data(), wp.data()) != LG_OK)
    {
        std::fprintf(stderr, "gbuffer: %s\n", lg_last_error());
        return;
    }
    std::filesystem::path p(png);
    const std::string stem = (p.parent_path() / p.stem()).string();
    lg_write_png((stem + ".albedo.png").c_str(), cam.width, cam.height, alb.data());
    lg_write_png((stem + ".normal.png").c_str(), cam.width, cam.height, nrm.data());
    lg_write_png((stem + ".worldpos.png").c_str(), cam.width, cam.height, wp.data());
}

// Diffuse textures from <assetRoot>/<diffuse_tex>, reported as RenderSceneCUDA
// does (pathtracer.cu:597-613); unreadable files leave the material untextured.
void load_textures(lg_renderer* r, lg_scene* scene, int n_mats, const std::string& assetRoot)
{
    int loaded = 0, missing = 0;
    for (int m = 0; m < n_mats; ++m)
    {
        const std::string rel = lg_scene_texture(scene, m);
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
        if (lg_renderer_set_texture(r, m, px, w, h) != LG_OK) std::fprintf(stderr, "%s\n", lg_last_error());
        else ++loaded;
        lg_image_free(px);
    }
    std::printf("textures: %d loaded, %d missing (of %d materials)\n", loaded, missing, n_mats);
}

void make_parent_dirs(const std::string& p)
{
    std::error_code ec;
    auto parent = std::filesystem::path(p).parent_path();
    if (!parent.empty()) std::filesystem::create_directories(parent, ec);
}
}  // namespace

int main(int argc, char** argv)
{
    const char* jsonPath = nullptr;
    std::string pngPath = "output/reference.png";
    std::string hdrPath;
    std::string assetRoot;
    std::string batchFile;
    int spp = 64, bounces = 2, device = 0;
    bool gbuffer = false, useSort = false;
    bool haveCamPos = false, haveCamTgt = false;
    float camPos[3] = {0, 0, 0}, camTgt[3] = {0, 0, 0};

    auto read_vec3 = [&](int& i, float out[3]) -> bool {
        if (i + 3 >= argc) return false;
        out[0] = (float)std::atof(argv[++i]);
        out[1] = (float)std::atof(argv[++i]);
        out[2] = (float)std::atof(argv[++i]);
        return true;
    };
    for (int i = 1; i < argc; ++i)
    {
        std::string a = argv[i];
        if (a == "--spp" && i + 1 < argc) spp = std::atoi(argv[++i]);
        else if (a == "--bounces" && i + 1 < argc) bounces = std::atoi(argv[++i]);
        else if (a == "--asset-root" && i + 1 < argc) assetRoot = argv[++i];
        else if (a == "-o" && i + 1 < argc) pngPath = argv[++i];
        else if (a == "--hdr" && i + 1 < argc) hdrPath = argv[++i];
        else if (a == "--device" && i + 1 < argc) device = std::atoi(argv[++i]);
        else if (a == "--sort") useSort = true;
        else if (a == "--gbuffer") gbuffer = true;
        else if (a == "--cam-pos") haveCamPos = read_vec3(i, camPos);
        else if (a == "--cam-target") haveCamTgt = read_vec3(i, camTgt);
        else if (a == "--batch" && i + 1 < argc) batchFile = argv[++i];
        else if (!a.empty() && a[0] != '-' && !jsonPath) jsonPath = argv[i];
        else if (!a.empty() && a[0] != '-') pngPath = argv[i];
    }
    if (!jsonPath)
    {
        std::fprintf(stderr, "usage: %s <scene.json> [output.png] [--spp N] [--bounces N] [--asset-root DIR]\n",
                     argv[0]);
        return 1;
    }

    lg_scene* scene = nullptr;
    if (lg_scene_load_json(jsonPath, 1, 0, &scene) != LG_OK) return 2;
    lg_scene_desc desc;
    lg_scene_describe(scene, &desc);
    if (assetRoot.empty()) assetRoot = std::filesystem::path(jsonPath).parent_path().parent_path().string();

    if (haveCamPos && haveCamTgt)
    {
        lg_look_at(&desc.camera, camPos, camTgt);
        std::printf("camera override: pos (%.2f,%.2f,%.2f) -> target (%.2f,%.2f,%.2f)\n", camPos[0], camPos[1],
                    camPos[2], camTgt[0], camTgt[1], camTgt[2]);
    }

    lg_renderer* r = nullptr;
    if (lg_renderer_create(device, &r) != LG_OK)
    {
        std::fprintf(stderr, "%s\n", lg_last_error());
        lg_scene_destroy(scene);
        return 4;
    }
    auto t_bvh0 = std::chrono::steady_clock::now();
    if (lg_renderer_set_scene(r, &desc) != LG_OK)
    {
        std::fprintf(stderr, "%s\n", lg_last_error());
        lg_renderer_destroy(r);
        lg_scene_destroy(scene);
        return 4;
    }
    const double bvh_ms = ms_since(t_bvh0);
    load_textures(r, scene, desc.n_mats, assetRoot);
    int32_t n_nodes = 0;
    lg_renderer_get_bvh(r, nullptr, &n_nodes, nullptr);
    const int W = desc.camera.width, H = desc.camera.height;
    std::vector<uint8_t> rgb((size_t)W * H * 3);
    int rc = 0;

    if (!batchFile.empty())
    {
        auto jobs = read_batch_file(batchFile);
        std::printf("batch: %zu jobs  (scene+bvh loaded once in %.1f ms)\n", jobs.size(), bvh_ms);
        for (size_t k = 0; k < jobs.size(); ++k)
        {
            const BatchJob& j = jobs[k];
            lg_camera cam = desc.camera;
            lg_look_at(&cam, j.cam_pos, j.cam_tgt);
            lg_render_opts o{j.spp, j.bounces, 0, 0};
            lg_render_stats st{};
            auto t0 = std::chrono::steady_clock::now();
            if (lg_render(r, &cam, &o, rgb.data(), nullptr, nullptr, &st) != LG_OK)
            {
                std::fprintf(stderr, "%s\n", lg_last_error());
                rc = 4;
                break;
            }
            std::printf("kernel: %.1f ms  (%d x %d, %d spp, %d bounces, %d tris)\n", st.kernel_ms, W, H, j.spp,
                        j.bounces, desc.n_tris);
            const double ms = ms_since(t0);
            make_parent_dirs(j.out_png);
            lg_write_png(j.out_png.c_str(), W, H, rgb.data());
            if (gbuffer) write_gbuffer(r, cam, j.out_png);
            std::printf("[%zu/%zu] %s  spp=%d  render=%.1f ms\n", k + 1, jobs.size(), j.out_png.c_str(), j.spp, ms);
        }
        lg_renderer_destroy(r);
        lg_scene_destroy(scene);
        return rc;
    }

    std::printf("bvh: %.1f ms (%d nodes)\n", bvh_ms, (int)n_nodes);
    std::vector<float> accum(hdrPath.empty() ? 0 : (size_t)W * H * 3);
    lg_render_opts o{spp, bounces, 0, 0};
    lg_render_stats st{};
    auto t2 = std::chrono::steady_clock::now();
    const int rrc = useSort ? lg_render_sorted(r, &desc.camera, &o, rgb.data(), hdrPath.empty() ? nullptr : accum.data(), &st)
                            : lg_render(r, &desc.camera, &o, rgb.data(), hdrPath.empty() ? nullptr : accum.data(), nullptr, &st);
    if (rrc != LG_OK)
    {
        std::fprintf(stderr, "%s\n", lg_last_error());
        lg_renderer_destroy(r);
        lg_scene_destroy(scene);
        return 4;
    }
    std::printf("kernel%s: %.1f ms  (%d x %d, %d spp, %d bounces, %d tris)\n", useSort ? " (sorted)" : "",
                st.kernel_ms, W, H, spp, bounces, desc.n_tris);
    std::printf("render: %.1f ms (%d x %d)\n", ms_since(t2), W, H);
    if (gbuffer)
    {
        make_parent_dirs(pngPath);
        write_gbuffer(r, desc.camera, pngPath);
    }
    lg_renderer_destroy(r);
    if (lg_write_png(pngPath.c_str(), W, H, rgb.data()) != LG_OK)
    {
        std::fprintf(stderr, "failed to write %s\n", pngPath.c_str());
        lg_scene_destroy(scene);
        return 3;
    }
    std::printf("wrote %s\n", pngPath.c_str());
    if (!hdrPath.empty())
    {
        const float inv = spp > 0 ? 1.0f / (float)spp : 0.0f;
        for (auto& v : accum) v *= inv;
        if (lg_write_hdr(hdrPath.c_str(), W, H, accum.data()) != LG_OK)
            std::fprintf(stderr, "failed to write %s\n", hdrPath.c_str());
        else std::printf("wrote %s\n", hdrPath.c_str());
    }
    lg_scene_destroy(scene);
    return 0;
}
