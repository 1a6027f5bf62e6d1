// scene.h -- world-space triangle soup, lights, materials and camera.
//
// Drop-in for the reference header include/scene.h:1-58.  Every struct keeps
// the reference's field order and size (Triangle is 100 bytes: 9 vertex floats,
// 9 normal floats, 6 uv floats and an int material) because host callers and
// the device kernels share these records byte for byte.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

struct CameraDesc
{
    float pos[3] = {0, 0, 0};
    float cameraToWorld[16] = {};  // rows 0/1/2 = forward / left / up, row 3 = position
    float fovYDeg = 60.0f;
    float aspect = 1.0f;
    float nearZ = 0.1f;
    float farZ = 1000.0f;
    int imageWidth = 1920;
    int imageHeight = 1080;
};

struct DirectionalLight
{
    float dir[3] = {0, 0, -1};  // direction the light travels
    float color[3] = {1, 1, 1};
    float intensity = 1.0f;
};

struct PointLight
{
    float pos[3] = {0, 0, 0};
    float color[3] = {1, 1, 1};
    float intensity = 1.0f;
    float radius = 1.0f;
};

struct Material
{
    float albedo[3] = {0.8f, 0.8f, 0.8f};
    float emissive[3] = {0, 0, 0};
    std::string diffuseTex;  // empty = untextured
};

struct Triangle
{
    float v[3][3];
    float n[3][3];
    float uv[3][2];
    int material = 0;
};
static_assert(sizeof(Triangle) == 100, "Triangle must stay 100 bytes (reference ABI)");

struct Scene
{
    CameraDesc camera;
    DirectionalLight sun;
    std::vector<DirectionalLight> directionals;
    std::vector<PointLight> points;
    std::vector<Material> materials;
    std::vector<Triangle> triangles;
};

// Parses a version-1 scene.json (reference src/scene_loader.cpp:26-138).
// Returns false and prints "[scene] ..." to stderr on any error.
bool LoadSceneJSON(const std::string& path, Scene& out);
