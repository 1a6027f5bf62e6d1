// trace_dev.cuh -- device functions shared by the trace kernels (trace.cu)
// and the ray-sorted wavefront render (wavefront.cu): ray/box and
// ray/triangle tests, the traversal of the 4-wide and 2-wide records, the
// reference's RNG, camera, hemisphere sampling and light arithmetic.
// Included inside an unnamed namespace of namespace lg.
#pragma once

constexpr int kStack = kTraceStack;

// ---------------------------------------------------------------------------
// Ray queries
// ---------------------------------------------------------------------------
// Slab test of one box (pathtracer.cu:61-80); tmin_out = max(lo, 0).
__device__ __forceinline__ bool slab(const Ray& r, float mnx, float mxx, float mny, float mxy, float mnz, float mxz,
                                     float tmax_in, float& tmin_out)
{
    float t0 = (mnx - r.o.x) * r.inv_d.x;
    float t1 = (mxx - r.o.x) * r.inv_d.x;
    float lo = fminf(t0, t1), hi = fmaxf(t0, t1);
    t0 = (mny - r.o.y) * r.inv_d.y;
    t1 = (mxy - r.o.y) * r.inv_d.y;
    lo = fmaxf(lo, fminf(t0, t1));
    hi = fminf(hi, fmaxf(t0, t1));
    t0 = (mnz - r.o.z) * r.inv_d.z;
    t1 = (mxz - r.o.z) * r.inv_d.z;
    lo = fmaxf(lo, fminf(t0, t1));
    hi = fminf(hi, fmaxf(t0, t1));
    if (hi < fmaxf(lo, 0.0f) || lo > tmax_in) return false;
    tmin_out = fmaxf(lo, 0.0f);
    return true;
}

// 256-bit read-only load (sm_100): eight floats from a 32-byte aligned
// address in one request, where two 128-bit loads would take two.
__device__ __forceinline__ void ldg8(const void* p, float (&v)[8])
{
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
        : "l"(p));
}

// The three float4s of triangle ti's intersection record.
__device__ __forceinline__ void load_tri(const float4* __restrict__ tv, int ti, float4& a, float4& b, float4& c)
{
    const float4* p = tv + (size_t)kTriVec * ti;
    if (kTriVec == 4)
    {
        float v[8];
        ldg8(p, v);
        a = make_float4(v[0], v[1], v[2], v[3]);
        b = make_float4(v[4], v[5], v[6], v[7]);
    }
    else
    {
        a = __ldg(p);
        b = __ldg(p + 1);
    }
    c = __ldg(p + 2);
}

// Moller-Trumbore (pathtracer.cu:82-107) on a precomputed (v0, e1, e2).
__device__ __forceinline__ bool tri_hit(const Ray& r, const float4* __restrict__ tv, int ti, float tmax, float& outT,
                                        float& outU, float& outV)
{
    constexpr float kEps = 1e-6f;
    float4 a, b, c;
    load_tri(tv, ti, a, b, c);
    const vec3 v0 = v3(a.x, a.y, a.z);
    const vec3 e1 = v3(b.x, b.y, b.z);
    const vec3 e2 = v3(c.x, c.y, c.z);
    vec3 p = cross(r.d, e2);
    float det = dot(e1, p);
    if (det > -kEps && det < kEps) return false;
    float invDet = 1.0f / det;
    vec3 s = vsub(r.o, v0);
    float u = dot(s, p) * invDet;
    if (u < 0.0f || u > 1.0f) return false;
    vec3 q = cross(s, e1);
    float v = dot(r.d, q) * invDet;
    if (v < 0.0f || u + v > 1.0f) return false;
    float tt = dot(e2, q) * invDet;
    if (tt <= kEps || tt >= tmax) return false;
    outT = tt;
    outU = u;
    outV = v;
    return true;
}

// Watertight ray/triangle test (Woop, Benthin, Wald, "Watertight
// Ray/Triangle Intersection", JCGT 2013) on (v0, v1, v2): vertices are
// translated to the ray origin and sheared so the ray runs along +z; the
// three 2-D edge functions are products and differences rounded once each
// (no contraction), so an edge shared by two triangles gives opposite-signed
// values in both and a ray through the edge or a shared vertex cannot pass
// between them; exact zeros are re-evaluated in double.  Same outputs as
// tri_hit: u, v are the weights of v1 and v2, and the hit must satisfy
// 1e-6 < t < tmax.  No determinant epsilon: only det == 0 is rejected.
__device__ __forceinline__ float comp(vec3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

__device__ __forceinline__ bool tri_hit_wt(const Ray& r, const float4* __restrict__ tv, int ti, float tmax,
                                           float& outT, float& outU, float& outV)
{
    constexpr float kEps = 1e-6f;
    const float ax = fabsf(r.d.x), ay = fabsf(r.d.y), az = fabsf(r.d.z);
    const int kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    const float dz = comp(r.d, kz);
    if (dz < 0.0f) { const int t = kx; kx = ky; ky = t; }
    const float Sz = __frcp_rn(dz);
    const float Sx = __fmul_rn(comp(r.d, kx), Sz), Sy = __fmul_rn(comp(r.d, ky), Sz);
    float4 a4, b4, c4;
    load_tri(tv, ti, a4, b4, c4);
    const vec3 A = v3(__fsub_rn(a4.x, r.o.x), __fsub_rn(a4.y, r.o.y), __fsub_rn(a4.z, r.o.z));
    const vec3 B = v3(__fsub_rn(b4.x, r.o.x), __fsub_rn(b4.y, r.o.y), __fsub_rn(b4.z, r.o.z));
    const vec3 C = v3(__fsub_rn(c4.x, r.o.x), __fsub_rn(c4.y, r.o.y), __fsub_rn(c4.z, r.o.z));
    const float Az = comp(A, kz), Bz = comp(B, kz), Cz = comp(C, kz);
    const float Ax = __fsub_rn(comp(A, kx), __fmul_rn(Sx, Az)), Ay = __fsub_rn(comp(A, ky), __fmul_rn(Sy, Az));
    const float Bx = __fsub_rn(comp(B, kx), __fmul_rn(Sx, Bz)), By = __fsub_rn(comp(B, ky), __fmul_rn(Sy, Bz));
    const float Cx = __fsub_rn(comp(C, kx), __fmul_rn(Sx, Cz)), Cy = __fsub_rn(comp(C, ky), __fmul_rn(Sy, Cz));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f)
    {
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = U + V + W;
    if (det == 0.0f) return false;
    const float T = U * __fmul_rn(Sz, Az) + V * __fmul_rn(Sz, Bz) + W * __fmul_rn(Sz, Cz);
    const float invDet = 1.0f / det;
    const float tt = T * invDet;
    if (tt <= kEps || tt >= tmax) return false;
    outT = tt;
    outU = V * invDet;
    outV = W * invDet;
    return true;
}

template <bool kWT>
__device__ __forceinline__ bool tri_test(const Ray& r, const float4* __restrict__ tv, int ti, float tmax, float& outT,
                                         float& outU, float& outV)
{
    return kWT ? tri_hit_wt(r, tv, ti, tmax, outT, outU, outV) : tri_hit(r, tv, ti, tmax, outT, outU, outV);
}

struct Counters
{
    unsigned long long closest, shadow, overflow, nodes, tris, leaves;
};

__device__ __forceinline__ void cswap(float& ta, int& la, float& tb, int& lb)
{
    if (tb < ta)
    {
        const float t = ta; ta = tb; tb = t;
        const int l = la; la = lb; lb = l;
    }
}

// Traversal state of one ray: the record or leaf link to visit next (kDone
// once the stack is empty), a leaf postponed for testing (0 = none; leaf
// links are negative), the stack depth, and the closest hit so far (t starts
// at the ray's tmax).
constexpr int kDone = (int)0x80000000;  // no leaf or record link takes this value
struct Trav
{
    int cur, pend, sp, tri;
    float t, u, v;
};

template <bool kCount>
__device__ __forceinline__ void trav_begin(Trav& q, int root, float tmax, bool anyhit, Counters& cnt)
{
    q.cur = root;
    q.pend = 0;
    q.sp = 0;
    q.tri = -1;
    q.t = tmax;
    q.u = 0.0f;
    q.v = 0.0f;
    if (kCount) { if (anyhit) cnt.shadow++; else cnt.closest++; }
}

__device__ __forceinline__ int pop(Trav& q, const int* stack) { return q.sp == 0 ? kDone : stack[--q.sp]; }

// Stacks `link`; a push past kStack entries is dropped and flags the scene's
// fault word (the host turns it into LG_ERR_DEVICE), so a tree too deep for
// the stack never yields a silently incomplete image.  kChecked = false is
// for trees whose stack bound (computed when their records are built) fits
// in kStack: no traversal over them can overflow, so the test is left out.
template <bool kCount, bool kChecked = true>
__device__ __forceinline__ void push(Trav& q, int* stack, int link, const DevScene& s, Counters& cnt)
{
    if (!kChecked)
    {
        stack[q.sp++] = link;
        return;
    }
    if (q.sp < kStack)
    {
        stack[q.sp++] = link;
        return;
    }
    if (kCount) cnt.overflow++;
    *s.fault = 1u;
}

// The four boxes of a quantized 4-wide record against one ray.  Per axis,
// t(q) = q * (step / d) + (origin - o) / d: the step is a power of two, so
// the first product is exact, and each plane costs a byte-to-float
// conversion (exact) and one fused multiply-add.  The near
// plane is the min plane when 1/d >= 0 and the max plane otherwise; the signs
// of 1/d pick the byte words.  Hit rule and entry distance are the
// reference's (pathtracer.cu:61-80): hit unless hi < max(lo, 0) or lo > tmax
// (tested as max(lo, 0) > tmax, the same for tmax >= 0), entry max(lo, 0).
// The quantized boxes enclose the exact ones with a step to spare, which
// covers the rounding of these products.  Children that miss get t = +inf.
__device__ __forceinline__ float qplane(uint32_t w, int k)
{
    // byte k as a float (exact); the plain conversion measured 6% faster over
    // the whole kernel than building 2^23 + q with a byte permute and
    // subtracting 2^23
    return (float)((w >> (8 * k)) & 0xffu);
}
// The two 32-byte halves of 4-wide record i: a = o[3], step[3], qlo[0..1];
// b = qlo[2], qhi[3], link[4].  Records below top_n come from the block's
// shared-memory copy of the top of the tree (the first records in BFS
// order), the others through the read-only path.
__device__ __forceinline__ void load_rec4(const DevScene& s, const Wide4Node* s_top, int top_n, int i, float (&a)[8],
                                          float (&b)[8])
{
    if ((unsigned)i < (unsigned)top_n)  // never true when top_n is the constant 0
    {
        const float4* p = reinterpret_cast<const float4*>(s_top + i);
        const float4 x = p[0], y = p[1], z = p[2], w = p[3];
        a[0] = x.x; a[1] = x.y; a[2] = x.z; a[3] = x.w; a[4] = y.x; a[5] = y.y; a[6] = y.z; a[7] = y.w;
        b[0] = z.x; b[1] = z.y; b[2] = z.z; b[3] = z.w; b[4] = w.x; b[5] = w.y; b[6] = w.z; b[7] = w.w;
        return;
    }
    ldg8(&s.nodes4[i], a);
    ldg8(reinterpret_cast<const char*>(&s.nodes4[i]) + 32, b);
}

__device__ __forceinline__ int4 box4(const float (&a)[8], const float (&b)[8], const Ray& r, float tmax, float& t0,
                                     float& t1, float& t2, float& t3)
{
    const int4 ln = make_int4(__float_as_int(b[4]), __float_as_int(b[5]), __float_as_int(b[6]), __float_as_int(b[7]));
    const float ix = a[3] * r.inv_d.x, iy = a[4] * r.inv_d.y, iz = a[5] * r.inv_d.z;
    const float bx = (a[0] - r.o.x) * r.inv_d.x, by = (a[1] - r.o.y) * r.inv_d.y, bz = (a[2] - r.o.z) * r.inv_d.z;
    const bool sx = __float_as_int(r.inv_d.x) < 0, sy = __float_as_int(r.inv_d.y) < 0,
               sz = __float_as_int(r.inv_d.z) < 0;
    const uint32_t qlx = __float_as_uint(a[6]), qly = __float_as_uint(a[7]), qlz = __float_as_uint(b[0]);
    const uint32_t qhx = __float_as_uint(b[1]), qhy = __float_as_uint(b[2]), qhz = __float_as_uint(b[3]);
    const uint32_t nx = sx ? qhx : qlx, fx = sx ? qlx : qhx;
    const uint32_t ny = sy ? qhy : qly, fy = sy ? qly : qhy;
    const uint32_t nz = sz ? qhz : qlz, fz = sz ? qlz : qhz;
    const float inf = __int_as_float(0x7f800000);
    auto one = [&](int k) {
        const float l0 = fmaxf(fmaxf(fmaf(qplane(nx, k), ix, bx), fmaf(qplane(ny, k), iy, by)),
                               fmaxf(fmaf(qplane(nz, k), iz, bz), 0.0f));
        const float hi = fminf(fminf(fmaf(qplane(fx, k), ix, bx), fmaf(qplane(fy, k), iy, by)),
                               fmaf(qplane(fz, k), iz, bz));
        return (hi < l0 || l0 > tmax) ? inf : l0;
    };
    t0 = one(0);
    t1 = one(1);
    t2 = one(2);
    t3 = one(3);
    return ln;
}

// Visits record q.cur (>= 0).  4-wide: up to four child boxes; the hit
// children are ordered by entry distance, the nearest becomes q.cur and the
// rest are stacked nearest-on-top.  2-wide (traverse_closest, :109-160, for
// one record): both children's boxes with the reference's slab arithmetic,
// the nearer hit child first and the farther one stacked.  With no child hit
// the next entry is popped (kDone when the stack is empty).
// Measured alternatives on the 64-spp engine frame (633 ms with whole-ray
// traversal and records from the even-depth collapse): a "while-while" loop
// without speculation (internal records until every lane holds a leaf, then
// the leaves) ran 745 ms, and a 24-entry shared-memory stack 675 ms (its
// 96 KB per SM comes out of the L1 that caches the BVH records).
template <int kWidth, bool kCount, bool kChecked = true>
__device__ __forceinline__ void node_step(const DevScene& s, const Ray& r, Trav& q, int* stack, Counters& cnt,
                                          const Wide4Node* s_top = nullptr, int top_n = 0)
{
    if (kCount) cnt.nodes++;
    const float inf = __int_as_float(0x7f800000);
    if (kWidth == 4)
    {
        float t0, t1, t2, t3;
        float a[8], b[8];
        load_rec4(s, s_top, top_n, q.cur, a, b);
        const int4 ln = box4(a, b, r, q.t, t0, t1, t2, t3);
        int l0 = ln.x, l1 = ln.y, l2 = ln.z, l3 = ln.w;
        cswap(t0, l0, t1, l1);
        cswap(t2, l2, t3, l3);
        cswap(t0, l0, t2, l2);
        cswap(t1, l1, t3, l3);
        cswap(t1, l1, t2, l2);
        if (t0 != inf)
        {
            // push farthest first so the nearest remaining is on top
            if (t3 != inf) push<kCount, kChecked>(q, stack, l3, s, cnt);
            if (t2 != inf) push<kCount, kChecked>(q, stack, l2, s, cnt);
            if (t1 != inf) push<kCount, kChecked>(q, stack, l1, s, cnt);
            q.cur = l0;
            return;
        }
    }
    else
    {
        const float4 xy0 = __ldg(&s.nodes[q.cur].xy0);
        const float4 xy1 = __ldg(&s.nodes[q.cur].xy1);
        const float4 z01 = __ldg(&s.nodes[q.cur].z01);
        const int4 ln = __ldg(&s.nodes[q.cur].link);
        float t0, t1;
        const bool h0 = slab(r, xy0.x, xy0.y, xy0.z, xy0.w, z01.x, z01.y, q.t, t0);
        const bool h1 = slab(r, xy1.x, xy1.y, xy1.z, xy1.w, z01.z, z01.w, q.t, t1);
        if (h0 && h1)
        {
            const bool swap = t1 < t0;
            push<kCount, kChecked>(q, stack, swap ? ln.x : ln.y, s, cnt);
            q.cur = swap ? ln.y : ln.x;
            return;
        }
        if (h0 || h1)
        {
            q.cur = h0 ? ln.x : ln.y;
            return;
        }
    }
    q.cur = pop(q, stack);
}

// Tests every triangle of leaf `link` in order (strict < on t, as
// traverse_closest's leaf loop).  4-wide leaf links carry (first, count) for
// 1..15 triangles; larger leaves and 2-wide links index the leaf table.
// Returns true when a shadow ray found an occluder.
template <int kWidth, bool kCount, bool kWT>
__device__ __forceinline__ bool leaf_step(const DevScene& s, const Ray& r, bool anyhit, int link, Trav& q,
                                          Counters& cnt)
{
    int2 lf;
    if (kWidth == 4 && s.leaf_inline)
    {
        const int v = ~link;
        lf = make_int2(v >> 4, v & 15);
        if (lf.y == 0)
        {
            lf = __ldg(&s.leaves[lf.x]);
            if (kCount) { cnt.leaves++; }
        }
    }
    else
    {
        lf = __ldg(&s.leaves[~link]);
        if (kCount) { cnt.leaves++; }
    }
    for (int i = 0; i < lf.y; ++i)
    {
        const int ti = lf.x + i;
        float tt, uu, vv;
        if (kCount) cnt.tris++;
        if (tri_test<kWT>(r, s.tv, ti, q.t, tt, uu, vv))
        {
            q.t = tt;
            q.tri = ti;
            q.u = uu;
            q.v = vv;
            if (anyhit) return true;
        }
    }
    return false;
}

// A whole traversal of one ray, one record or leaf at a time: the closest
// hit (triangle or -1) and its t, u, v, as traverse_closest returns them; a
// shadow ray stops at its first hit.
template <int kWidth, bool kCount, bool kWT>
__device__ __forceinline__ int traverse_ray(const DevScene& s, const Ray& r, float tmax, bool anyhit, float& bestT,
                                            float& bestU, float& bestV, Counters& cnt)
{
    int stack[kStack];
    Trav q;
    trav_begin<kCount>(q, kWidth == 4 ? s.root4 : s.root, tmax, anyhit, cnt);
    while (q.cur != kDone)
    {
        if (q.cur >= 0) node_step<kWidth, kCount>(s, r, q, stack, cnt);
        else
        {
            if (leaf_step<kWidth, kCount, kWT>(s, r, anyhit, q.cur, q, cnt)) break;
            q.cur = pop(q, stack);
        }
    }
    bestT = q.t;
    bestU = q.u;
    bestV = q.v;
    return q.tri;
}

// One warp-wide step of the persistent kernel's traversals, with leaves
// postponed (Aila and Laine, "Understanding the Efficiency of Ray Traversal
// on GPUs", HPG 2009): a lane that reaches a leaf sets it aside and keeps
// visiting records from its stack while other lanes still look for a leaf.
// The warp visits records while more than `quorum` lanes are still looking
// (or no lane holds a leaf), and otherwise tests the held leaves together;
// quorum 0 waits for every lane, as in the paper.  Every step makes
// progress: a record step has at least one searching lane, a leaf step at
// least one held leaf.  The records visited past a postponed leaf would be
// culled by a nearer hit in it only for closest-hit rays, and then only cost
// time: the closest hit is the same (up to exact ties in t).  `busy` is this
// lane's ray in flight; returns true when its traversal has finished.
template <int kWidth, bool kCount, bool kWT, bool kChecked = true>
__device__ __forceinline__ bool warp_step(const DevScene& s, const Ray& r, bool anyhit, bool busy, int quorum,
                                          Trav& q, int* stack, Counters& cnt, const Wide4Node* s_top, int top_n)
{
    if (busy && q.pend == 0 && q.cur < 0 && q.cur != kDone)
    {
        q.pend = q.cur;
        q.cur = pop(q, stack);
    }
    const bool fin = busy && q.pend == 0 && q.cur == kDone;
    // every lane takes part in the votes, finished or idle ones included
    const bool searching = busy && !fin && q.pend == 0;  // then q.cur >= 0
    const unsigned n_searching = __popc(__ballot_sync(0xffffffffu, searching));
    const bool holding = __any_sync(0xffffffffu, busy && !fin && q.pend != 0);
    if (n_searching > (unsigned)quorum || !holding)
    {
        if (busy && q.cur >= 0) node_step<kWidth, kCount, kChecked>(s, r, q, stack, cnt, s_top, top_n);
        return fin;
    }
    if (!busy || fin || q.pend == 0) return fin;
    const int link = q.pend;
    q.pend = 0;
    return leaf_step<kWidth, kCount, kWT>(s, r, anyhit, link, q, cnt) || q.cur == kDone;
}

// xorshift32 / randf (pathtracer.cu:193-204).
__device__ __forceinline__ uint32_t xorshift32(uint32_t& st)
{
    st ^= st << 13;
    st ^= st >> 17;
    st ^= st << 5;
    return st;
}
__device__ __forceinline__ float randf(uint32_t& st) { return (xorshift32(st) >> 8) * (1.0f / 16777216.0f); }

// Frisvad frame (:206-214) and cosine-weighted direction (:216-228).
__device__ __forceinline__ void onb(vec3 N, vec3& T, vec3& B)
{
    if (N.z < -0.99999f)
    {
        T = v3(0, -1, 0);
        B = v3(-1, 0, 0);
        return;
    }
    float a = 1.0f / (1.0f + N.z);
    float b = -N.x * N.y * a;
    T = v3(1.0f - N.x * N.x * a, b, -N.x);
    B = v3(b, 1.0f - N.y * N.y * a, -N.y);
}
__device__ __forceinline__ vec3 sample_cos_hemi(vec3 N, uint32_t& rng)
{
    float u1 = randf(rng);
    float u2 = randf(rng);
    float r = sqrtf(u1);
    float phi = 2.0f * 3.14159265358979f * u2;
    float x = r * cosf(phi);
    float y = r * sinf(phi);
    float z = sqrtf(fmaxf(0.0f, 1.0f - u1));
    vec3 T, B;
    onb(N, T, B);
    return normalize(vadd(vadd(vmul(T, x), vmul(B, y)), vmul(N, z)));
}

__device__ __forceinline__ Ray primary_ray(const DevCam& cam, int px, int py, float jx, float jy)
{
    float ndcx = (2.0f * (px + jx) / cam.width) - 1.0f;
    float ndcy = 1.0f - (2.0f * (py + jy) / cam.height);
    float rx = ndcx * cam.aspect * cam.tanHalfFov;
    float ry = ndcy * cam.tanHalfFov;
    vec3 dirCam = v3(1.0f, -rx, ry);
    vec3 dirWorld = vadd(vadd(vmul(cam.fwd, dirCam.x), vmul(cam.left, dirCam.y)), vmul(cam.up, dirCam.z));
    return make_ray(cam.pos, dirWorld);
}

// Light `li` as seen from a hit (shade_direct, :230-272): li == 0 is the
// sun, li >= 1 the point light li-1.  Returns false when the light is
// skipped without a shadow ray (facing away, or beyond 3 radii); otherwise
// sets the shadow ray and its tmax and, in *contrib, the radiance it adds
// when unoccluded.
__device__ __forceinline__ bool light_query(const DevScene& s, int li, vec3 P, vec3 N, vec3 albedo, Ray& shadow,
                                            float& tmax, vec3& contrib)
{
    constexpr float kShadowBias = 1e-3f;
    if (li == 0)
    {
        vec3 toLight = normalize(vmul(vfrom(s.sun.dir), -1.0f));
        float ndotl = fmaxf(0.0f, dot(N, toLight));
        if (!(ndotl > 0.0f)) return false;
        shadow = make_ray(vadd(P, vmul(N, kShadowBias)), toLight);
        tmax = 1e30f;
        float I = s.sun.intensity * ndotl;
        contrib = vhad(albedo, vmul(vfrom(s.sun.color), I));
        return true;
    }
    const lg_point_light& L = s.points[li - 1];
    vec3 toLightVec = vsub(vfrom(L.pos), P);
    float dist = len(toLightVec);
    vec3 toLight = vmul(toLightVec, 1.0f / dist);
    float ndotl = fmaxf(0.0f, dot(N, toLight));
    if (ndotl <= 0.0f || dist >= L.radius * 3.0f) return false;
    shadow = make_ray(vadd(P, vmul(N, kShadowBias)), toLight);
    tmax = dist - kShadowBias;
    float rr = L.radius;
    float atten = fmaxf(0.0f, 1.0f - dist / rr);
    atten = atten * atten;
    float I = L.intensity * ndotl * atten;
    contrib = vhad(albedo, vmul(vfrom(L.color), I));
    return true;
}

// sample_albedo (:274-282) at a hit: the material's diffuse texture at the
// interpolated uv (traverse_closest's expressions, :156-157) with v flipped,
// else the material's constant albedo.  The texture objects are created
// as the reference creates them (uchar4 array, sRGB, bilinear, wrap,
// normalised coordinates), so the texture unit filters identically.
__device__ __forceinline__ vec3 hit_albedo(const DevScene& s, const lg_triangle& t, int mat, float w, float hitU,
                                           float hitV)
{
    if (s.texs)
    {
        const unsigned long long tx = __ldg(&s.texs[mat]);
        if (tx)
        {
            const float u = w * t.uv[0][0] + hitU * t.uv[1][0] + hitV * t.uv[2][0];
            const float v = w * t.uv[0][1] + hitU * t.uv[1][1] + hitV * t.uv[2][1];
            const float4 c = tex2D<float4>((cudaTextureObject_t)tx, u, 1.0f - v);
            return v3(c.x, c.y, c.z);
        }
    }
    const float4 alb = __ldg(&s.mats[mat]);
    return v3(alb.x, alb.y, alb.z);
}

