// vecmath.h -- small FP32 vector helpers shared by host code and CUDA kernels.
//
// Drop-in for the reference header include/vecmath.h:1-44: the same names
// (vec3, v3, vfrom, vadd, vsub, vmul, vhad, dot, cross, len, normalize, Ray,
// make_ray) with the same argument meaning, so code written against the
// reference compiles unchanged.  The arithmetic order of every helper is the
// one the reference uses (dot = x*x' + y*y' + z*z' left to right; normalize
// multiplies by 1/len and falls back to +Z below 1e-20), because the path
// tracer's parity with the reference renderer depends on it.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define LG_HD __host__ __device__ inline
#else
#define LG_HD inline
#endif

struct vec3 { float x, y, z; };

LG_HD vec3 v3(float x, float y, float z) { vec3 r; r.x = x; r.y = y; r.z = z; return r; }
LG_HD vec3 vfrom(const float p[3]) { return v3(p[0], p[1], p[2]); }
LG_HD vec3 vadd(vec3 a, vec3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
LG_HD vec3 vsub(vec3 a, vec3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
LG_HD vec3 vmul(vec3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
LG_HD vec3 vhad(vec3 a, vec3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
LG_HD float dot(vec3 a, vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
LG_HD vec3 cross(vec3 a, vec3 b)
{
    return v3(a.y * b.z - a.z * b.y,
              a.z * b.x - a.x * b.z,
              a.x * b.y - a.y * b.x);
}
LG_HD float len(vec3 a) { return sqrtf(dot(a, a)); }
LG_HD vec3 normalize(vec3 a)
{
    const float l = len(a);
    if (l > 1e-20f) return vmul(a, 1.0f / l);
    return v3(0.0f, 0.0f, 1.0f);
}

// A ray with its per-axis reciprocal direction (for slab tests).
struct Ray
{
    vec3 o, d;
    vec3 inv_d;
};

// Normalises d and precomputes 1/d, as the reference's make_ray does.
LG_HD Ray make_ray(vec3 o, vec3 d)
{
    Ray r;
    r.o = o;
    r.d = normalize(d);
    r.inv_d = v3(1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z);
    return r;
}
