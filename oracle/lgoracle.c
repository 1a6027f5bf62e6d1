/* lgoracle.c -- TEST INFRASTRUCTURE ONLY: CPU oracle for the render path.
 *
 * A plain-C restatement of LuminaGI-CudaRef's host BVH build (src/bvh.cpp)
 * and its device trace code (src/pathtracer.cu), written so every FP32
 * operation happens in the reference's order (build with
 * -ffp-contract=off).  It is the checker for this project's CUDA kernels in
 * tests/ and the CPU baseline in bench.py; the product never links it.
 *
 * Differences from the reference, on purpose:
 *   - the Morton sort breaks ties by original triangle index (a total order);
 *     the reference's std::sort leaves the order inside a run of equal codes
 *     to libstdc++'s introsort.  Node arrays do not depend on that order.
 *   - ray counters are gathered (the reference has none).
 * Pinned against the reference's own sources (oracle/_ref/libref.so) by
 * tests/test_oracle.py: BVH nodes bit-identical, accumulators bit-identical.
 */
#include "lgoracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* vector helpers (include/vecmath.h:9-44)                             */
/* ------------------------------------------------------------------ */
typedef struct { float x, y, z; } v3f;
typedef struct { v3f o, d, inv_d; } ray_t;

static v3f V(float x, float y, float z) { v3f r; r.x = x; r.y = y; r.z = z; return r; }
static v3f Vp(const float* p) { return V(p[0], p[1], p[2]); }
static v3f Vadd(v3f a, v3f b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3f Vsub(v3f a, v3f b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3f Vmul(v3f a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static v3f Vhad(v3f a, v3f b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static float Vdot(v3f a, v3f b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3f Vcross(v3f a, v3f b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static float Vlen(v3f a) { return sqrtf(Vdot(a, a)); }
static v3f Vnorm(v3f a)
{
    float l = Vlen(a);
    return (l > 1e-20f) ? Vmul(a, 1.0f / l) : V(0, 0, 1);
}
static ray_t make_ray(v3f o, v3f d)
{
    ray_t r;
    r.o = o;
    r.d = Vnorm(d);
    r.inv_d = V(1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z);
    return r;
}

/* ------------------------------------------------------------------ */
/* BVH build (src/bvh.cpp)                                             */
/* ------------------------------------------------------------------ */
/* bvh.cpp:14-21 */
static uint32_t spread3(uint32_t v)
{
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
/* bvh.cpp:23-32: clamp(f*1024, 0, 1023), truncate */
static uint32_t quant10(float f)
{
    f = f * 1024.0f;
    if (f < 0.0f) f = 0.0f;
    if (f > 1023.0f) f = 1023.0f;
    return (uint32_t)f;
}
static uint32_t morton3(float x, float y, float z)
{
    return (spread3(quant10(x)) << 2) | (spread3(quant10(y)) << 1) | spread3(quant10(z));
}
/* bvh.cpp:34-42: strict-less updates, first occurrence wins on ties */
static void fit(float mn[3], float mx[3], const float p[3])
{
    for (int k = 0; k < 3; ++k) if (p[k] < mn[k]) mn[k] = p[k];
    for (int k = 0; k < 3; ++k) if (p[k] > mx[k]) mx[k] = p[k];
}
/* bvh.cpp:44-52 */
static void fit_union(float mn[3], float mx[3], const float amn[3], const float amx[3])
{
    for (int k = 0; k < 3; ++k) if (amn[k] < mn[k]) mn[k] = amn[k];
    for (int k = 0; k < 3; ++k) if (amx[k] > mx[k]) mx[k] = amx[k];
}
/* bvh.cpp:54-65: lowest i in [first,last) with the mask bit set */
static int find_split(const uint32_t* code, int first, int last, uint32_t mask)
{
    int lo = first, hi = last;
    while (lo < hi)
    {
        int mid = lo + ((hi - lo) >> 1);
        if (code[mid] & mask) hi = mid; else lo = mid + 1;
    }
    return lo;
}

typedef struct { lgo_node* nodes; int count; const uint32_t* code; const lgo_tri* tris; } build_ctx;

/* bvh.cpp:75-120: preorder DFS, leaf at <= 4 triangles or when no bit splits */
static int build_recursive(build_ctx* c, int first, int last, int bit)
{
    int idx = c->count++;
    lgo_node* n = &c->nodes[idx];
    int count = last - first;
    int split = first;
    while (bit >= 0)
    {
        split = find_split(c->code, first, last, 1u << bit);
        if (split != first && split != last) break;
        --bit;
    }
    if (count <= 4 || bit < 0)
    {
        float mn[3] = {INFINITY, INFINITY, INFINITY};
        float mx[3] = {-INFINITY, -INFINITY, -INFINITY};
        n->left = -1; n->right = -1; n->firstTri = first; n->triCount = count;
        for (int i = first; i < last; ++i)
            for (int k = 0; k < 3; ++k) fit(mn, mx, c->tris[i].v[k]);
        memcpy(n->bbMin, mn, sizeof mn);
        memcpy(n->bbMax, mx, sizeof mx);
        return idx;
    }
    int L = build_recursive(c, first, split, bit - 1);
    int R = build_recursive(c, split, last, bit - 1);
    n = &c->nodes[idx];
    n->left = L; n->right = R; n->firstTri = -1; n->triCount = 0;
    memcpy(n->bbMin, c->nodes[L].bbMin, 3 * sizeof(float));
    memcpy(n->bbMax, c->nodes[L].bbMax, 3 * sizeof(float));
    fit_union(n->bbMin, n->bbMax, c->nodes[R].bbMin, c->nodes[R].bbMax);
    return idx;
}

/* bvh.cpp:122-162: renumber breadth-first, left child before right */
static void relayout_bfs(lgo_node* nodes, int n)
{
    int* oldToNew = (int*)malloc(sizeof(int) * n);
    int* order = (int*)malloc(sizeof(int) * n);
    lgo_node* tmp = (lgo_node*)malloc(sizeof(lgo_node) * n);
    int head = 0, tail = 0;
    order[tail++] = 0;
    oldToNew[0] = 0;
    while (head < tail)
    {
        int oi = order[head++];
        if (nodes[oi].triCount == 0)
        {
            oldToNew[nodes[oi].left] = tail; order[tail++] = nodes[oi].left;
            oldToNew[nodes[oi].right] = tail; order[tail++] = nodes[oi].right;
        }
    }
    for (int ni = 0; ni < n; ++ni)
    {
        lgo_node nn = nodes[order[ni]];
        if (nn.triCount == 0) { nn.left = oldToNew[nn.left]; nn.right = oldToNew[nn.right]; }
        tmp[ni] = nn;
    }
    memcpy(nodes, tmp, sizeof(lgo_node) * n);
    free(tmp); free(order); free(oldToNew);
}

/* bvh.cpp:170-178 */
void lgo_scene_bounds(const lgo_tri* tris, int n, float mn[3], float ext[3])
{
    float mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    mn[0] = mn[1] = mn[2] = INFINITY;
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) fit(mn, mx, tris[i].v[c]);
    for (int a = 0; a < 3; ++a)
    {
        ext[a] = mx[a] - mn[a];
        if (ext[a] <= 0.0f) ext[a] = 1.0f;
    }
}

/* bvh.cpp:185-190: centroid = (v0+v1+v2) * (1/3), normalised by the scene box */
uint32_t lgo_morton_of(const lgo_tri* t, const float mn[3], const float ext[3])
{
    const float third = 1.0f / 3.0f;
    float cx = (t->v[0][0] + t->v[1][0] + t->v[2][0]) * third;
    float cy = (t->v[0][1] + t->v[1][1] + t->v[2][1]) * third;
    float cz = (t->v[0][2] + t->v[1][2] + t->v[2][2]) * third;
    return morton3((cx - mn[0]) / ext[0], (cy - mn[1]) / ext[1], (cz - mn[2]) / ext[2]);
}

static const uint32_t* g_sort_codes;
static int cmp_code_index(const void* a, const void* b)
{
    int ia = *(const int*)a, ib = *(const int*)b;
    uint32_t ca = g_sort_codes[ia], cb = g_sort_codes[ib];
    if (ca != cb) return ca < cb ? -1 : 1;
    return (ia > ib) - (ia < ib);
}

/* bvh.cpp:164-211 */
int lgo_build_bvh(const lgo_tri* tris, int n, lgo_node* nodes_out, int* perm, lgo_tri* tris_out, uint32_t* codes_out)
{
    if (n <= 0) return 0;
    float mn[3], ext[3];
    lgo_scene_bounds(tris, n, mn, ext);
    uint32_t* code = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* sorted = (uint32_t*)malloc(sizeof(uint32_t) * n);
    int* order = (int*)malloc(sizeof(int) * n);
    for (int i = 0; i < n; ++i) { code[i] = lgo_morton_of(&tris[i], mn, ext); order[i] = i; }
    g_sort_codes = code;
    qsort(order, (size_t)n, sizeof(int), cmp_code_index);
    for (int i = 0; i < n; ++i)
    {
        sorted[i] = code[order[i]];
        tris_out[i] = tris[order[i]];
        if (perm) perm[i] = order[i];
        if (codes_out) codes_out[i] = sorted[i];
    }
    build_ctx c = {nodes_out, 0, sorted, tris_out};
    build_recursive(&c, 0, n, 29);
    relayout_bfs(nodes_out, c.count);
    free(code); free(sorted); free(order);
    return c.count;
}

/* ------------------------------------------------------------------ */
/* Path tracer (src/pathtracer.cu)                                     */
/* ------------------------------------------------------------------ */
typedef struct {
    const lgo_node* nodes; const lgo_tri* tris; const float* albedo;
    const lgo_point* points; int n_points; lgo_dir sun;
} scene_t;

typedef struct { v3f pos, fwd, left, up; float tanHalfFov, aspect; int width, height; } cam_t;

/* pathtracer.cu:61-80 */
static int ray_aabb(const ray_t* r, const float mn[3], const float mx[3], float tmax_in)
{
    float t0 = (mn[0] - r->o.x) * r->inv_d.x;
    float t1 = (mx[0] - r->o.x) * r->inv_d.x;
    float lo = fminf(t0, t1), hi = fmaxf(t0, t1);
    t0 = (mn[1] - r->o.y) * r->inv_d.y;
    t1 = (mx[1] - r->o.y) * r->inv_d.y;
    lo = fmaxf(lo, fminf(t0, t1));
    hi = fminf(hi, fmaxf(t0, t1));
    t0 = (mn[2] - r->o.z) * r->inv_d.z;
    t1 = (mx[2] - r->o.z) * r->inv_d.z;
    lo = fmaxf(lo, fminf(t0, t1));
    hi = fminf(hi, fmaxf(t0, t1));
    if (hi < fmaxf(lo, 0.0f) || lo > tmax_in) return 0;
    return 1;
}

/* pathtracer.cu:82-107: Moller-Trumbore, |det| < 1e-6 rejected, hit in (1e-6, tmax) */
static int ray_tri(const ray_t* r, const lgo_tri* t, float tmax, float* oT, float* oU, float* oV)
{
    const float kEps = 1e-6f;
    v3f v0 = Vp(t->v[0]);
    v3f e1 = Vsub(Vp(t->v[1]), v0);
    v3f e2 = Vsub(Vp(t->v[2]), v0);
    v3f p = Vcross(r->d, e2);
    float det = Vdot(e1, p);
    if (det > -kEps && det < kEps) return 0;
    float invDet = 1.0f / det;
    v3f s = Vsub(r->o, v0);
    float u = Vdot(s, p) * invDet;
    if (u < 0.0f || u > 1.0f) return 0;
    v3f q = Vcross(s, e1);
    float v = Vdot(r->d, q) * invDet;
    if (v < 0.0f || u + v > 1.0f) return 0;
    float tt = Vdot(e2, q) * invDet;
    if (tt <= kEps || tt >= tmax) return 0;
    *oT = tt; *oU = u; *oV = v;
    return 1;
}

/* pathtracer.cu:109-160: 64-entry stack, push left then right, no ordering */
static int traverse_closest(const scene_t* s, const ray_t* r, float tmax, float* oT, v3f* oN, lgo_counters* c)
{
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    float bestT = tmax, bestU = 0, bestV = 0;
    int bestTri = -1;
    c->closest_rays++;
    while (sp > 0)
    {
        const lgo_node* n = &s->nodes[stack[--sp]];
        c->node_visits++;
        if (!ray_aabb(r, n->bbMin, n->bbMax, bestT)) continue;
        if (n->triCount > 0)
        {
            for (int i = 0; i < n->triCount; ++i)
            {
                int ti = n->firstTri + i;
                float tt, uu, vv;
                c->tri_tests++;
                if (ray_tri(r, &s->tris[ti], bestT, &tt, &uu, &vv)) { bestT = tt; bestTri = ti; bestU = uu; bestV = vv; }
            }
        }
        else if (sp + 2 <= 64)
        {
            stack[sp++] = n->left;
            stack[sp++] = n->right;
        }
    }
    if (bestTri < 0) return -1;
    const lgo_tri* t = &s->tris[bestTri];
    float w = 1.0f - bestU - bestV;
    *oN = Vnorm(V(w * t->n[0][0] + bestU * t->n[1][0] + bestV * t->n[2][0],
                  w * t->n[0][1] + bestU * t->n[1][1] + bestV * t->n[2][1],
                  w * t->n[0][2] + bestU * t->n[1][2] + bestV * t->n[2][2]));
    *oT = bestT;
    return bestTri;
}

/* pathtracer.cu:162-191: any-hit */
static int traverse_occluded(const scene_t* s, const ray_t* r, float tmax, lgo_counters* c)
{
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    c->shadow_rays++;
    while (sp > 0)
    {
        const lgo_node* n = &s->nodes[stack[--sp]];
        c->node_visits++;
        if (!ray_aabb(r, n->bbMin, n->bbMax, tmax)) continue;
        if (n->triCount > 0)
        {
            for (int i = 0; i < n->triCount; ++i)
            {
                float tt, uu, vv;
                c->tri_tests++;
                if (ray_tri(r, &s->tris[n->firstTri + i], tmax, &tt, &uu, &vv)) return 1;
            }
        }
        else if (sp + 2 <= 64)
        {
            stack[sp++] = n->left;
            stack[sp++] = n->right;
        }
    }
    return 0;
}

/* pathtracer.cu:193-204 */
static uint32_t xorshift32(uint32_t* s)
{
    *s ^= *s << 13;
    *s ^= *s >> 17;
    *s ^= *s << 5;
    return *s;
}
static float randf(uint32_t* s) { return (float)(xorshift32(s) >> 8) * (1.0f / 16777216.0f); }

/* pathtracer.cu:206-214: Frisvad frame */
static void onb(v3f N, v3f* T, v3f* B)
{
    if (N.z < -0.99999f) { *T = V(0, -1, 0); *B = V(-1, 0, 0); return; }
    float a = 1.0f / (1.0f + N.z);
    float b = -N.x * N.y * a;
    *T = V(1.0f - N.x * N.x * a, b, -N.x);
    *B = V(b, 1.0f - N.y * N.y * a, -N.y);
}

/* pathtracer.cu:216-228 */
static v3f sample_cos_hemi(v3f N, uint32_t* rng)
{
    float u1 = randf(rng);
    float u2 = randf(rng);
    float r = sqrtf(u1);
    float phi = 2.0f * 3.14159265358979f * u2;
    float x = r * cosf(phi);
    float y = r * sinf(phi);
    float z = sqrtf(fmaxf(0.0f, 1.0f - u1));
    v3f T, B;
    onb(N, &T, &B);
    return Vnorm(Vadd(Vadd(Vmul(T, x), Vmul(B, y)), Vmul(N, z)));
}

/* pathtracer.cu:230-272: sun (shadow ray even at zero intensity) + point lights */
static v3f shade_direct(const scene_t* s, v3f P, v3f N, v3f albedo, lgo_counters* c)
{
    const float kShadowBias = 1e-3f;
    v3f color = V(0, 0, 0);
    {
        v3f toLight = Vnorm(Vmul(Vp(s->sun.dir), -1.0f));
        float ndotl = fmaxf(0.0f, Vdot(N, toLight));
        if (ndotl > 0.0f)
        {
            ray_t sh = make_ray(Vadd(P, Vmul(N, kShadowBias)), toLight);
            if (!traverse_occluded(s, &sh, 1e30f, c))
            {
                float I = s->sun.intensity * ndotl;
                color = Vadd(color, Vhad(albedo, Vmul(Vp(s->sun.color), I)));
            }
        }
    }
    for (int i = 0; i < s->n_points; ++i)
    {
        const lgo_point* L = &s->points[i];
        v3f toLightVec = Vsub(Vp(L->pos), P);
        float dist = Vlen(toLightVec);
        v3f toLight = Vmul(toLightVec, 1.0f / dist);
        float ndotl = fmaxf(0.0f, Vdot(N, toLight));
        if (ndotl <= 0.0f || dist >= L->radius * 3.0f) continue;
        ray_t sh = make_ray(Vadd(P, Vmul(N, kShadowBias)), toLight);
        if (traverse_occluded(s, &sh, dist - kShadowBias, c)) continue;
        float atten = fmaxf(0.0f, 1.0f - dist / L->radius);
        atten = atten * atten;
        float I = L->intensity * ndotl * atten;
        color = Vadd(color, Vhad(albedo, Vmul(Vp(L->color), I)));
    }
    return color;
}

/* pathtracer.cu:284-293 */
static ray_t primary_ray(const cam_t* cam, int px, int py, float jx, float jy)
{
    float ndcx = (2.0f * (px + jx) / cam->width) - 1.0f;
    float ndcy = 1.0f - (2.0f * (py + jy) / cam->height);
    float rx = ndcx * cam->aspect * cam->tanHalfFov;
    float ry = ndcy * cam->tanHalfFov;
    v3f dirCam = V(1.0f, -rx, ry);
    v3f dirWorld = Vadd(Vadd(Vmul(cam->fwd, dirCam.x), Vmul(cam->left, dirCam.y)), Vmul(cam->up, dirCam.z));
    return make_ray(cam->pos, dirWorld);
}

/* pathtracer.cu:295-331: emissive unused, no environment light, RR from bounce 1 */
static v3f trace_path(const scene_t* s, ray_t ray, int maxBounces, uint32_t* rng, lgo_counters* c)
{
    v3f L = V(0, 0, 0);
    v3f T = V(1, 1, 1);
    for (int bounce = 0; bounce <= maxBounces; ++bounce)
    {
        float hitT;
        v3f N;
        int tri = traverse_closest(s, &ray, 1e30f, &hitT, &N, c);
        if (tri < 0) break;
        if (Vdot(N, ray.d) > 0.0f) N = Vmul(N, -1.0f);
        v3f P = Vadd(ray.o, Vmul(ray.d, hitT));
        v3f albedo = Vp(&s->albedo[3 * s->tris[tri].material]);
        L = Vadd(L, Vhad(T, shade_direct(s, P, N, albedo, c)));
        if (bounce == maxBounces) break;
        if (bounce >= 1)
        {
            float q = fminf(0.95f, fmaxf(T.x, fmaxf(T.y, T.z)));
            if (randf(rng) > q) break;
            T = Vmul(T, 1.0f / q);
        }
        v3f nd = sample_cos_hemi(N, rng);
        ray = make_ray(Vadd(P, Vmul(N, 1e-3f)), nd);
        T = Vhad(T, albedo);
    }
    return L;
}

/* Camera set-up of RenderSceneCUDA (pathtracer.cu:654-663). */
static cam_t make_cam(const lgo_camera* c)
{
    cam_t k;
    const float* m = c->cameraToWorld;
    k.pos = Vp(c->pos);
    k.fwd = V(m[0], m[1], m[2]);
    k.left = V(m[4], m[5], m[6]);
    k.up = V(m[8], m[9], m[10]);
    k.tanHalfFov = tanf(c->fovYDeg * 0.5f * 3.14159265358979f / 180.0f);
    k.aspect = c->aspect;
    k.width = c->imageWidth;
    k.height = c->imageHeight;
    return k;
}

/* accumulate_kernel body (pathtracer.cu:349-363) for every chunk of 8 samples
 * (pathtracer.cu:699-704), over a subset of rows. */
int lgo_render(const lgo_node* nodes, const lgo_tri* tris, const float* mat_albedo, int n_mats,
               const lgo_point* points, int n_points, const lgo_dir* sun, const lgo_camera* camd, int spp,
               int max_bounces, int row_start, int row_step, int threads, float* accum, lgo_counters* counters)
{
    (void)n_mats;
    scene_t s;
    s.nodes = nodes; s.tris = tris; s.albedo = mat_albedo; s.points = points; s.n_points = n_points; s.sun = *sun;
    cam_t cam = make_cam(camd);
    const int W = cam.width, H = cam.height;
    if (row_step < 1) row_step = 1;
    const int n_rows = row_start < H ? (H - row_start + row_step - 1) / row_step : 0;
    uint64_t cr = 0, sr = 0, nv = 0, tt = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : cr, sr, nv, tt) num_threads(threads > 0 ? threads : 1)
    for (int r = 0; r < n_rows; ++r)
    {
        lgo_counters c = {0, 0, 0, 0};
        const int py = row_start + r * row_step;
        for (int px = 0; px < W; ++px)
        {
            for (int base = 0; base < spp; base += 8)
            {
                const int n_this = (spp - base < 8) ? (spp - base) : 8;
                uint32_t rng = ((uint32_t)px * 1973u + (uint32_t)py * 9277u + (uint32_t)base * 26699u) | 1u;
                v3f sum = V(0, 0, 0);
                for (int k = 0; k < n_this; ++k)
                {
                    float jx = randf(&rng);
                    float jy = randf(&rng);
                    ray_t ray = primary_ray(&cam, px, py, jx, jy);
                    sum = Vadd(sum, trace_path(&s, ray, max_bounces, &rng, &c));
                }
                size_t i = ((size_t)py * W + px) * 3;
                accum[i + 0] += sum.x;
                accum[i + 1] += sum.y;
                accum[i + 2] += sum.z;
            }
        }
        cr += c.closest_rays; sr += c.shadow_rays; nv += c.node_visits; tt += c.tri_tests;
    }
    if (counters)
    {
        counters->closest_rays = cr; counters->shadow_rays = sr;
        counters->node_visits = nv; counters->tri_tests = tt;
    }
    return 0;
}

/* pathtracer.cu:413-429: sqrt(clamp(acc/spp,0,1)) * 255, truncated */
void lgo_tonemap(const float* accum, uint8_t* rgb, int n_pixels, float inv_spp)
{
    for (long i = 0; i < (long)n_pixels * 3; ++i)
    {
        float v = sqrtf(fmaxf(0.0f, fminf(accum[i] * inv_spp, 1.0f)));
        rgb[i] = (uint8_t)(v * 255.0f);
    }
}
