// Device data layout of the 8-wide BVH and the reference-compatible triangle
// test shared by the build and the traversal kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ilg {

// ---------------------------------------------------------------------------
// Node record: 80 bytes = 5 x uint4, 16-byte aligned, read with 128-bit loads.
//   q0: origin.xyz (float bits), w = ex | ey << 8 | ez << 16 | imask << 24
//       (e* are biased power-of-two exponents of the quantisation step,
//        imask bit s = slot s holds an internal child)
//   q1: x = first child node, y = first triangle record,
//       z = meta[0..3], w = meta[4..7]
//   q2: x/y = qlo.x[0..7], z/w = qhi.x[0..7]   (one byte per slot)
//   q3: same for y, q4: same for z
// meta byte: 0 = empty slot; 0x80 = internal child; otherwise a leaf with
// count (1..3) in bits 5-6 and the offset of its first triangle from the
// node's first triangle record (0..23) in bits 0-4.
// Internal children of a node are stored contiguously in slot order, so the
// child in slot s is node first_child + popc(imask & ((1 << s) - 1)).
// Slots are assigned so that a ray in octant o visits children in
// descending order of (slot ^ (7 - o)), which approximates front to back.
// ---------------------------------------------------------------------------
struct __align__(16) Node8 {
    uint4 q[5];
};
static_assert(sizeof(Node8) == 80, "node record must be 80 bytes");

// Triangle record: 48 bytes = 3 x float4.
//   a = (v0.x, v0.y, v0.z, n.x), b = (e1.xyz, n.y), c = (e2.xyz, n.z)
// with e1 = v1 - v0, e2 = v2 - v0, n = e1 x e2 evaluated exactly as the
// reference does (IndexedTriangle.cpp:44-45, :103), one rounding per op.
struct __align__(16) Tri {
    float4 a, b, c;
};
static_assert(sizeof(Tri) == 48, "triangle record must be 48 bytes");

constexpr int kMaxStack = 64;      // traversal stack entries (node groups)
// triangles per leaf child; measured on a B200 with the treelet-restructured
// tree (1 M-triangle heightfield, coherent / incoherent Mrays/s; 21 M-triangle
// field, 960x540x16 ms): 1: 6790 / 2254, 25.6; 2: 7100 / 2357, 26.0;
// 3: 6920 / 2316, 26.7
constexpr int kLeafMax = 2;
constexpr uint32_t kMetaInternal = 0x80u;

// Lower bound of the reference's triangle window, `t < 1e-5` evaluated in
// double (IndexedTriangle.cpp:115): for a float t this is t < the smallest
// float >= 1e-5, i.e. 0x3727C5AD.
__device__ __forceinline__ float window_lo() { return __int_as_float(0x3727C5AD); }

// Upper bound: `t > Max - 1e-5` in double holds for a float t exactly when
// t > (Max - 1e-5) rounded down to float.
__device__ __forceinline__ float window_hi(float tmax)
{
    return __double2float_rd(__dsub_rn((double)tmax, 1e-5));
}

// Shirley-form test of IndexedTriangle::Intersects (IndexedTriangle.cpp:92-128)
// with every product and sum rounded separately (no contraction), so that t,
// beta and gamma are bit-identical to the reference compiled without FMA.
// `hi` is window_hi(current Max).
__device__ __forceinline__ bool shirley(const Tri &tr, float ox, float oy, float oz, float dx, float dy,
                                        float dz, float hi, float &t_out, float &b_out, float &g_out)
{
    const float nx = tr.a.w, ny = tr.b.w, nz = tr.c.w;
    const float den = __fadd_rn(__fadd_rn(__fmul_rn(nx, dx), __fmul_rn(ny, dy)), __fmul_rn(nz, dz));
    const float rcp = __fdiv_rn(1.0f, den);
    const float ex = __fsub_rn(tr.a.x, ox), ey = __fsub_rn(tr.a.y, oy), ez = __fsub_rn(tr.a.z, oz);
    const float num = __fadd_rn(__fadd_rn(__fmul_rn(nx, ex), __fmul_rn(ny, ey)), __fmul_rn(nz, ez));
    const float t = __fmul_rn(num, rcp);
    if (t > hi || t < window_lo()) return false;
    // interm = d x edge2
    const float ix = __fsub_rn(__fmul_rn(dy, ez), __fmul_rn(dz, ey));
    const float iy = __fsub_rn(__fmul_rn(dz, ex), __fmul_rn(dx, ez));
    const float iz = __fsub_rn(__fmul_rn(dx, ey), __fmul_rn(dy, ex));
    const float beta =
        __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(ix, tr.c.x), __fmul_rn(iy, tr.c.y)), __fmul_rn(iz, tr.c.z)), -rcp);
    if (beta < 0.0f) return false;
    const float gamma =
        __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(ix, tr.b.x), __fmul_rn(iy, tr.b.y)), __fmul_rn(iz, tr.b.z)), rcp);
    if (__fadd_rn(beta, gamma) > 1.0f || gamma < 0.0f) return false;
    // A NaN t (origin in the triangle's plane, direction parallel to it)
    // passes the reference's comparisons and poisons its ray.Max; it is
    // rejected here instead.
    if (!(t <= hi)) return false;
    t_out = t;
    b_out = beta;
    g_out = gamma;
    return true;
}

// ---------------------------------------------------------------------------
// Watertight test (Woop, Benthin and Wald 2013, "Watertight Ray/Triangle
// Intersection", JCGT 2(1)): the triangle is sheared into the ray's frame
// (the ray's largest direction component becomes z) and the three 2D edge
// functions U, V, W are evaluated from the vertices themselves, so two
// triangles that share an edge evaluate it with the same numbers and a ray
// through it cannot slip between them. Edge functions that come out exactly
// zero are recomputed in double. Every operation is rounded separately. The
// rejection window is the reference's (t < 1e-5 or t > Max - 1e-5); beta
// and gamma are the weights of v1 and v2, as in the reference.
// ---------------------------------------------------------------------------
struct Shear {
    uint32_t kx, ky, kz;
    float sx, sy, sz;
};

__device__ __forceinline__ float pick(float x, float y, float z, uint32_t k) { return k == 0u ? x : (k == 1u ? y : z); }

__device__ __forceinline__ Shear shear_of(float dx, float dy, float dz)
{
    const float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
    Shear s;
    s.kz = ax >= ay ? (ax >= az ? 0u : 2u) : (ay >= az ? 1u : 2u);
    s.kx = s.kz == 2u ? 0u : s.kz + 1u;
    s.ky = s.kx == 2u ? 0u : s.kx + 1u;
    const float dkz = pick(dx, dy, dz, s.kz);
    if (dkz < 0.f) {
        const uint32_t k = s.kx;
        s.kx = s.ky;
        s.ky = k;
    }
    s.sx = __fdiv_rn(pick(dx, dy, dz, s.kx), dkz);
    s.sy = __fdiv_rn(pick(dx, dy, dz, s.ky), dkz);
    s.sz = __fdiv_rn(1.0f, dkz);
    return s;
}

// v0, v1, v2: the triangle's own vertices (w unused).
__device__ __forceinline__ bool watertight(float4 v0, float4 v1, float4 v2, float ox, float oy, float oz,
                                           const Shear &sh, float hi, float &t_out, float &b_out, float &g_out)
{
    const float a0 = __fsub_rn(v0.x, ox), a1 = __fsub_rn(v0.y, oy), a2 = __fsub_rn(v0.z, oz);
    const float b0 = __fsub_rn(v1.x, ox), b1 = __fsub_rn(v1.y, oy), b2 = __fsub_rn(v1.z, oz);
    const float c0 = __fsub_rn(v2.x, ox), c1 = __fsub_rn(v2.y, oy), c2 = __fsub_rn(v2.z, oz);
    const float akz = pick(a0, a1, a2, sh.kz), bkz = pick(b0, b1, b2, sh.kz), ckz = pick(c0, c1, c2, sh.kz);
    const float Ax = __fsub_rn(pick(a0, a1, a2, sh.kx), __fmul_rn(sh.sx, akz));
    const float Ay = __fsub_rn(pick(a0, a1, a2, sh.ky), __fmul_rn(sh.sy, akz));
    const float Bx = __fsub_rn(pick(b0, b1, b2, sh.kx), __fmul_rn(sh.sx, bkz));
    const float By = __fsub_rn(pick(b0, b1, b2, sh.ky), __fmul_rn(sh.sy, bkz));
    const float Cx = __fsub_rn(pick(c0, c1, c2, sh.kx), __fmul_rn(sh.sx, ckz));
    const float Cy = __fsub_rn(pick(c0, c1, c2, sh.ky), __fmul_rn(sh.sy, ckz));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.f || V == 0.f || W == 0.f) {
        U = __double2float_rn(__dsub_rn(__dmul_rn(Cx, By), __dmul_rn(Cy, Bx)));
        V = __double2float_rn(__dsub_rn(__dmul_rn(Ax, Cy), __dmul_rn(Ay, Cx)));
        W = __double2float_rn(__dsub_rn(__dmul_rn(Bx, Ay), __dmul_rn(By, Ax)));
    }
    if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return false;
    const float det = __fadd_rn(__fadd_rn(U, V), W);
    if (det == 0.f) return false;
    const float Az = __fmul_rn(sh.sz, akz), Bz = __fmul_rn(sh.sz, bkz), Cz = __fmul_rn(sh.sz, ckz);
    const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
    const float rcp = __fdiv_rn(1.0f, det);
    const float t = __fmul_rn(T, rcp);
    if (!(t <= hi) || t < window_lo()) return false;
    t_out = t;
    b_out = __fmul_rn(V, rcp);
    g_out = __fmul_rn(W, rcp);
    return true;
}

}  // namespace ilg
