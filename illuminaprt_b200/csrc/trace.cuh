// Closest-hit and any-hit traversal of the 8-wide BVH (replaces the reference's
// per-ray CPU walks: BasicSpace::Intersects -> KDTreeMesh::Intersect_New /
// BVHMesh::Intersect -> IndexedTriangle::Intersects; BasicSpace.cpp:58-115,
// KDTreeMesh.cpp:313-577, BVHMesh.cpp:143-198, IndexedTriangle.cpp:92-290).
//
// One ray per thread. The stack holds node groups (first child node index,
// remaining-children bits | imask), one entry per level at most; the
// children of a node are intersected together from one 80-byte record and
// visited in octant order. A hit shrinks the ray's Max exactly as the
// reference does, so the triangle window `t > Max - 1e-5` and the result are
// the reference's, up to which of two hits less than 1e-5 apart is visited
// first.
#pragma once

#include "bvh8.cuh"

namespace ilg {

struct TraceOut {
    int32_t *prim;   // closest hit: triangle index or -1
    float *t, *u, *v;
    uint8_t *occ;    // any hit: 0/1
};

struct TraceStats {
    unsigned long long nodes, tris;
};

// Input triangles [lo, lo + n) that a query ignores (the reference's
// `p_pExclude` primitive after its triangles were flattened into one range);
// prim_of maps a triangle record to its input index.
struct Skip {
    const uint32_t *prim_of;
    uint32_t lo, n;
};

// ---------------------------------------------------------------------------
// Traversal state machine shared by every kernel
// ---------------------------------------------------------------------------

// The traversal stack: a plain uint2 array (local memory), or split in two,
// its first kShortStack entries in shared memory (one column per thread of a
// kStackColumns-thread block: entry i of a thread at s[i * kStackColumns]) and
// the rest in local memory. The BVH8 of a few million triangles is 7 to 9
// levels deep, so the local part is rarely touched; shared memory keeps the
// entries out of the L1 lines that node and triangle loads stream through
// (measured on a B200: 3 % more incoherent rays per second on the 1 M
// triangle heightfield).
constexpr int kShortStack = 8;
constexpr int kStackColumns = 128;
struct SplitStack {
    uint2 *s;  // this thread's column of the block's shared array
    uint2 *l;  // entries kShortStack .. kMaxStack - 1
};
__device__ __forceinline__ void stack_put(uint2 *a, int i, uint2 e) { a[i] = e; }
__device__ __forceinline__ uint2 stack_get(uint2 *a, int i) { return a[i]; }
__device__ __forceinline__ void stack_put(const SplitStack &t, int i, uint2 e)
{
    if (i < kShortStack) t.s[i * kStackColumns] = e;
    else t.l[i - kShortStack] = e;
}
__device__ __forceinline__ uint2 stack_get(const SplitStack &t, int i)
{
    return i < kShortStack ? t.s[i * kStackColumns] : t.l[i - kShortStack];
}

struct RayState {
    float ox, oy, oz, dx, dy, dz;
    float ix, iy, iz;
    float tmin, tcur, whi;
    uint32_t octinv;
    uint32_t ng_base, ng_hits, tg_base, tg_hits;
    uint32_t budget;
    int sp;
    int best;
    float bu, bv;
    Shear sh;  // watertight test only
    bool any;  // kMixed traversals: this ray is an any-hit (shadow) ray
};

template <bool kWT = false>
__device__ __forceinline__ void ray_init(RayState &r, float4 o, float4 d, uint32_t n_nodes_total)
{
    if (kWT) r.sh = shear_of(d.x, d.y, d.z);
    const float kTiny = 1e-20f;
    r.ox = o.x; r.oy = o.y; r.oz = o.z; r.dx = d.x; r.dy = d.y; r.dz = d.z;
    r.ix = __frcp_rn(fabsf(d.x) > kTiny ? d.x : copysignf(kTiny, d.x));
    r.iy = __frcp_rn(fabsf(d.y) > kTiny ? d.y : copysignf(kTiny, d.y));
    r.iz = __frcp_rn(fabsf(d.z) > kTiny ? d.z : copysignf(kTiny, d.z));
    const uint32_t oct = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
    r.octinv = 7u - oct;
    r.tmin = o.w;
    r.tcur = d.w;
    r.whi = window_hi(r.tcur);
    r.ng_base = 0;
    r.ng_hits = (1u << (24 + r.octinv)) | 1u;
    r.tg_base = 0;
    r.tg_hits = 0;
    r.budget = n_nodes_total + 1u;
    r.sp = 0;
    r.best = -1;
    r.bu = r.bv = 0.f;
}

// Triangle tests per traversal step in the persistent kernels. A step visits
// a node group only when no triangles of earlier groups are pending, and
// tests at most this many of the pending ones, so the lanes of a warp take
// turns of similar length instead of waiting out the longest leaf (a lane
// that finishes early takes a new ray). Each ray still visits its nodes and
// triangles in the same order, so results do not depend on it. Measured on
// a B200 (1 M-triangle heightfield, 21 M-triangle path-traced field): 2
// gains 11 % on incoherent rays and on the path tracer and 3 % on camera
// rays over testing a whole leaf per step; 1 loses 35 %, 3 and 4 gain less.
// One-ray-per-thread kernels (no refill) test a whole leaf group per step.
constexpr int kTrisPerStep = 2;
constexpr int kTrisWholeGroup = 32;

// One traversal step. Returns true when the ray is finished (r.best is the
// hit record, -1 for a miss, -2 for a reported error).
// kWT selects the watertight triangle test over `raw` (three float4
// vertices per triangle record) instead of the reference's Shirley test.
// kMixed: closest- and any-hit rays share one instance (r.any chooses per ray).
template <bool kAnyHit, bool kStats = false, bool kSkip = false, bool kWT = false, int kTris = kTrisPerStep,
          bool kMixed = false, class Stack = uint2 *>
__device__ __forceinline__ bool ray_step(RayState &r, Stack stack, const Node8 *__restrict__ nodes,
                                         const Tri *__restrict__ tris, uint32_t n_nodes_total, uint32_t n_tris_total,
                                         uint32_t *__restrict__ err, unsigned long long *n_nodes = nullptr,
                                         unsigned long long *n_tris = nullptr, Skip skip = Skip{nullptr, 0u, 0u},
                                         const float4 *__restrict__ raw = nullptr)
{
    if (r.tg_hits == 0u && (r.ng_hits & 0xff000000u)) {
        if (r.budget-- == 0u) {
            atomicOr(err, 4u);
            r.best = -2;
            return true;
        }
        const uint32_t bit = 31u - __clz(r.ng_hits & 0xff000000u);
        r.ng_hits &= ~(1u << bit);
        const uint32_t slot = (bit - 24u) ^ r.octinv;
        const uint32_t node_idx = r.ng_base + __popc(r.ng_hits & 0xffu & ((1u << slot) - 1u));
        if (r.ng_hits & 0xff000000u) {
            if (r.sp >= kMaxStack) {
                atomicOr(err, 1u);
                r.best = -2;
                return true;
            }
            stack_put(stack, r.sp++, make_uint2(r.ng_base, r.ng_hits));
        }
        if (node_idx >= n_nodes_total) {
            atomicOr(err, 2u);
            r.best = -2;
            return true;
        }
        const uint4 *q = reinterpret_cast<const uint4 *>(nodes + node_idx);
        const uint4 q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2), q3 = __ldg(q + 3), q4 = __ldg(q + 4);
        if (kStats) (*n_nodes)++;
        const float sx = __uint_as_float((q0.w & 0xffu) << 23);
        const float sy = __uint_as_float(((q0.w >> 8) & 0xffu) << 23);
        const float sz = __uint_as_float(((q0.w >> 16) & 0xffu) << 23);
        const float ax = (__uint_as_float(q0.x) - r.ox) * r.ix, ay = (__uint_as_float(q0.y) - r.oy) * r.iy,
                    az = (__uint_as_float(q0.z) - r.oz) * r.iz;
        const float bx = sx * r.ix, by = sy * r.iy, bz = sz * r.iz;
        const uint32_t nxl = r.ix >= 0.f ? q2.x : q2.z, nxh = r.ix >= 0.f ? q2.y : q2.w;
        const uint32_t fxl = r.ix >= 0.f ? q2.z : q2.x, fxh = r.ix >= 0.f ? q2.w : q2.y;
        const uint32_t nyl = r.iy >= 0.f ? q3.x : q3.z, nyh = r.iy >= 0.f ? q3.y : q3.w;
        const uint32_t fyl = r.iy >= 0.f ? q3.z : q3.x, fyh = r.iy >= 0.f ? q3.w : q3.y;
        const uint32_t nzl = r.iz >= 0.f ? q4.x : q4.z, nzh = r.iz >= 0.f ? q4.y : q4.w;
        const uint32_t fzl = r.iz >= 0.f ? q4.z : q4.x, fzh = r.iz >= 0.f ? q4.w : q4.y;
        uint32_t hits_int = 0, hits_tri = 0;
#pragma unroll
        for (int s = 0; s < 8; s++) {
            const uint32_t sh = (s & 3) * 8;
            const uint32_t meta = ((s < 4 ? q1.z : q1.w) >> sh) & 0xffu;
            const float tnx = fmaf((float)(((s < 4 ? nxl : nxh) >> sh) & 0xffu), bx, ax);
            const float tfx = fmaf((float)(((s < 4 ? fxl : fxh) >> sh) & 0xffu), bx, ax);
            const float tny = fmaf((float)(((s < 4 ? nyl : nyh) >> sh) & 0xffu), by, ay);
            const float tfy = fmaf((float)(((s < 4 ? fyl : fyh) >> sh) & 0xffu), by, ay);
            const float tnz = fmaf((float)(((s < 4 ? nzl : nzh) >> sh) & 0xffu), bz, az);
            const float tfz = fmaf((float)(((s < 4 ? fzl : fzh) >> sh) & 0xffu), bz, az);
            const float tn = fmaxf(fmaxf(fmaxf(tnx, tny), tnz) * 0.9999990f, r.tmin);
            const float tf = fminf(fminf(fminf(tfx, tfy), tfz) * 1.0000010f, r.tcur);
            if (meta != 0u && tn <= tf) {
                if (meta == kMetaInternal) hits_int |= 1u << (24u + ((uint32_t)s ^ r.octinv));
                else hits_tri |= ((1u << (meta >> 5)) - 1u) << (meta & 31u);
            }
        }
        r.ng_base = q1.x;
        r.ng_hits = hits_int | (q0.w >> 24);
        r.tg_base = q1.y;
        r.tg_hits = hits_tri;
    }
    for (int tested = 0; r.tg_hits && tested < kTris; tested++) {
        const uint32_t b = __ffs(r.tg_hits) - 1u;
        r.tg_hits &= r.tg_hits - 1u;
        const uint32_t ti = r.tg_base + b;
        if (ti >= n_tris_total) {
            atomicOr(err, 2u);
            r.best = -2;
            return true;
        }
        if (kSkip && __ldg(skip.prim_of + ti) - skip.lo < skip.n) continue;
        if (kStats) (*n_tris)++;
        float th, bh, gh;
        bool hit;
        if (kWT) {
            const float4 *vp = raw + 3ull * ti;
            hit = watertight(__ldg(vp), __ldg(vp + 1), __ldg(vp + 2), r.ox, r.oy, r.oz, r.sh, r.whi, th, bh, gh);
        } else {
            const float4 *tp = reinterpret_cast<const float4 *>(tris + ti);
            Tri tr;
            tr.a = __ldg(tp);
            tr.b = __ldg(tp + 1);
            tr.c = __ldg(tp + 2);
            hit = shirley(tr, r.ox, r.oy, r.oz, r.dx, r.dy, r.dz, r.whi, th, bh, gh);
        }
        if (hit) {
            r.best = (int)ti;
            if (kAnyHit || (kMixed && r.any)) return true;
            r.bu = bh;
            r.bv = gh;
            r.tcur = th;
            r.whi = window_hi(r.tcur);
        }
    }
    if (r.tg_hits == 0u && !(r.ng_hits & 0xff000000u)) {
        if (r.sp == 0) return true;
        const uint2 e = stack_get(stack, --r.sp);
        r.ng_base = e.x;
        r.ng_hits = e.y;
    }
    return false;
}

// Whole traversal of one ray (one ray per thread).
template <bool kAnyHit, bool kStats, bool kSkip = false>
__device__ __forceinline__ void trace_one(const Node8 *__restrict__ nodes, const Tri *__restrict__ tris,
                                          uint32_t n_nodes_total, uint32_t n_tris_total,
                                          float4 o, float4 d, int &best, float &bt, float &bu, float &bv,
                                          uint32_t *__restrict__ err, unsigned long long &n_nodes,
                                          unsigned long long &n_tris, Skip skip = Skip{nullptr, 0u, 0u})
{
    uint2 stack[kMaxStack];
    RayState r;
    ray_init(r, o, d, n_nodes_total);
    while (!ray_step<kAnyHit, kStats, kSkip, false, kTrisWholeGroup>(r, stack, nodes, tris, n_nodes_total,
                                                                      n_tris_total, err, &n_nodes, &n_tris, skip)) {
    }
    best = r.best;
    bt = r.best >= 0 ? r.tcur : __int_as_float(0x7f800000);
    bu = r.best >= 0 ? r.bu : 0.f;
    bv = r.best >= 0 ? r.bv : 0.f;
}

// ---------------------------------------------------------------------------
// Persistent traversal with dynamic ray fetch: each warp keeps its lanes busy
// by handing a finished lane a new ray from a global counter whenever at least
// kRefillLanes lanes are idle (Aila & Laine 2009, "Understanding the
// efficiency of ray traversal on GPUs"). One loop iteration = one ray_step
// (a node visit or up to kTrisPerStep triangle tests), so lanes stay in step
// on the same code. Measured on a B200: batched queries (k_trace_dyn) run
// best refilling at 4 idle lanes, the path tracer's bounce and shadow
// kernels at 8.
// ---------------------------------------------------------------------------
constexpr uint32_t kRefillLanesQuery = 4;
constexpr uint32_t kRefillLanes = 8;

}  // namespace ilg
