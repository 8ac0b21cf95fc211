// Device build of the 8-wide BVH (replaces the reference's per-mesh CPU tree
// builders, KDTreeMesh::Compile / BVHMesh::Compile, KDTreeMesh.cpp:114-275 and
// BVHMesh.cpp:78-107, which take ~6-20 s per million triangles on one core).
//
// Pipeline, all on the context's stream:
//   1. k_tri_bounds   per-triangle AABB + centroid, scene centroid bounds
//   2. k_morton       30-bit Morton code of each centroid
//   3. radix sort     (code, triangle) pairs (CUB)
//   4. k_karras       binary radix tree over the sorted codes (Karras 2012),
//                     duplicate codes split by index
//   5. k_refit        bottom-up AABBs, one atomic arrival counter per node
//   5b. k_treelet     bottom-up treelet restructuring for least SAH cost
//                     (Karras & Aila 2013); subtree triangle counts
//   5c. k_collapse_cost  bottom-up SAH costs of the binary subtrees as 1..8
//                     roots of an 8-wide node (Ylitie et al. 2017)
//   6. k_collapse     level by level: each work item turns one binary node
//                     into one 8-wide node (its children: the roots the
//                     step 5c costs chose; a root is a leaf or a node),
//                     orders the slots by octant, quantises the child boxes
//                     to 8 bits against the node origin, and writes the
//                     triangle records of its leaf children.
#include "bvh8.cuh"
#include "build.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <cfloat>
#include <cmath>
#include <utility>

namespace ilg {

namespace {

__device__ __forceinline__ uint32_t float_flip(float f)
{
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float float_unflip(uint32_t u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ __forceinline__ uint32_t expand_bits10(uint32_t v)
{
    v &= 0x3ffu;
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

struct Box {
    float3 lo, hi;
};

__device__ __forceinline__ float area(const float3 &lo, const float3 &hi)
{
    float dx = fmaxf(hi.x - lo.x, 0.f), dy = fmaxf(hi.y - lo.y, 0.f), dz = fmaxf(hi.z - lo.z, 0.f);
    return dx * dy + dy * dz + dz * dx;
}

// ---------------------------------------------------------------- step 1 ----
__global__ void k_tri_bounds(const float *__restrict__ pos, uint32_t n_verts, const uint32_t *__restrict__ idx,
                             uint32_t n, float4 *__restrict__ tlo, float4 *__restrict__ thi,
                             uint32_t *__restrict__ cbounds /* 6 flipped floats: min xyz, max xyz */,
                             uint32_t *__restrict__ err)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float3 clo = make_float3(FLT_MAX, FLT_MAX, FLT_MAX), chi = make_float3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    if (i < n) {
        uint32_t a = idx[3 * i], b = idx[3 * i + 1], c = idx[3 * i + 2];
        if (a >= n_verts || b >= n_verts || c >= n_verts) {
            atomicOr(err, 1u);
            a = b = c = 0;
        }
        float3 p0 = make_float3(pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]);
        float3 p1 = make_float3(pos[3 * b], pos[3 * b + 1], pos[3 * b + 2]);
        float3 p2 = make_float3(pos[3 * c], pos[3 * c + 1], pos[3 * c + 2]);
        float3 lo = make_float3(fminf(p0.x, fminf(p1.x, p2.x)), fminf(p0.y, fminf(p1.y, p2.y)),
                                fminf(p0.z, fminf(p1.z, p2.z)));
        float3 hi = make_float3(fmaxf(p0.x, fmaxf(p1.x, p2.x)), fmaxf(p0.y, fmaxf(p1.y, p2.y)),
                                fmaxf(p0.z, fmaxf(p1.z, p2.z)));
        tlo[i] = make_float4(lo.x, lo.y, lo.z, 0.f);
        thi[i] = make_float4(hi.x, hi.y, hi.z, 0.f);
        clo = make_float3(0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z));
        chi = clo;
    }
    // warp reduce, then one atomic per warp
    for (int o = 16; o > 0; o >>= 1) {
        clo.x = fminf(clo.x, __shfl_xor_sync(0xffffffffu, clo.x, o));
        clo.y = fminf(clo.y, __shfl_xor_sync(0xffffffffu, clo.y, o));
        clo.z = fminf(clo.z, __shfl_xor_sync(0xffffffffu, clo.z, o));
        chi.x = fmaxf(chi.x, __shfl_xor_sync(0xffffffffu, chi.x, o));
        chi.y = fmaxf(chi.y, __shfl_xor_sync(0xffffffffu, chi.y, o));
        chi.z = fmaxf(chi.z, __shfl_xor_sync(0xffffffffu, chi.z, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&cbounds[0], float_flip(clo.x));
        atomicMin(&cbounds[1], float_flip(clo.y));
        atomicMin(&cbounds[2], float_flip(clo.z));
        atomicMax(&cbounds[3], float_flip(chi.x));
        atomicMax(&cbounds[4], float_flip(chi.y));
        atomicMax(&cbounds[5], float_flip(chi.z));
    }
}

// ---------------------------------------------------------------- step 2 ----
__global__ void k_morton(const float4 *__restrict__ tlo, const float4 *__restrict__ thi, uint32_t n,
                         const uint32_t *__restrict__ cbounds, uint32_t *__restrict__ keys,
                         uint32_t *__restrict__ vals)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 lo = make_float3(float_unflip(cbounds[0]), float_unflip(cbounds[1]), float_unflip(cbounds[2]));
    float3 hi = make_float3(float_unflip(cbounds[3]), float_unflip(cbounds[4]), float_unflip(cbounds[5]));
    float4 a = tlo[i], b = thi[i];
    float cx = 0.5f * (a.x + b.x), cy = 0.5f * (a.y + b.y), cz = 0.5f * (a.z + b.z);
    float ex = hi.x - lo.x, ey = hi.y - lo.y, ez = hi.z - lo.z;
    float nx = ex > 0.f ? (cx - lo.x) / ex : 0.f;
    float ny = ey > 0.f ? (cy - lo.y) / ey : 0.f;
    float nz = ez > 0.f ? (cz - lo.z) / ez : 0.f;
    uint32_t ix = (uint32_t)fminf(fmaxf(nx * 1024.f, 0.f), 1023.f);
    uint32_t iy = (uint32_t)fminf(fmaxf(ny * 1024.f, 0.f), 1023.f);
    uint32_t iz = (uint32_t)fminf(fmaxf(nz * 1024.f, 0.f), 1023.f);
    keys[i] = (expand_bits10(ix) << 2) | (expand_bits10(iy) << 1) | expand_bits10(iz);
    vals[i] = i;
}

// ---------------------------------------------------------------- step 4 ----
// Internal node i of n-1; children encoded >= 0 internal, < 0 leaf ~sorted_pos.
__device__ __forceinline__ int delta(const uint32_t *keys, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    uint32_t a = keys[i], b = keys[j];
    if (a == b) return 32 + __clz((uint32_t)i ^ (uint32_t)j);
    return __clz(a ^ b);
}

__global__ void k_karras(const uint32_t *__restrict__ keys, int n, int2 *__restrict__ child,
                         int *__restrict__ parent_int, int *__restrict__ parent_leaf, int2 *__restrict__ range)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int dl = delta(keys, n, i, i - 1), dr = delta(keys, n, i, i + 1);
    int d = dr > dl ? 1 : -1;
    int dmin = d > 0 ? dl : dr;
    int lmax = 2;
    while (lmax < (1 << 30) && delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta(keys, n, i, j);
    int s = 0;
    int len = l;
    int t = (len + 1) >> 1;
    for (int it = 0; it < 64 && t >= 1; it++) {  // t halves (rounding up) to 1; the cap is only a guard
        if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
        if (t == 1) break;
        t = (t + 1) >> 1;
    }
    int gamma = i + s * d + min(d, 0);
    int first = min(i, j), last = max(i, j);
    int left = (first == gamma) ? ~gamma : gamma;
    int right = (last == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    child[i] = make_int2(left, right);
    range[i] = make_int2(first, last);
    if (i == 0) parent_int[0] = -1;  // the root ends every bottom-up walk
    if (left >= 0) parent_int[left] = i; else parent_leaf[~left] = i;
    if (right >= 0) parent_int[right] = i; else parent_leaf[~right] = i;
}

// ---------------------------------------------------------------- step 5 ----
__global__ void k_refit(int n, const uint32_t *__restrict__ sorted_tri, const float4 *__restrict__ tlo,
                        const float4 *__restrict__ thi, const int2 *__restrict__ child,
                        const int *__restrict__ parent_int, const int *__restrict__ parent_leaf,
                        uint32_t *__restrict__ arrivals, float4 *__restrict__ nlo, float4 *__restrict__ nhi)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int p = parent_leaf[i];
    // bounded by the tree height (< n); each node's second arrival proceeds
    for (int guard = 0; p >= 0 && p < n - 1 && guard < n; guard++) {
        __threadfence();
        if (atomicAdd(&arrivals[p], 1u) == 0) return;
        __threadfence();
        int2 c = child[p];
        float4 alo, ahi, blo, bhi;
        if (c.x >= 0) { alo = __ldcg(&nlo[c.x]); ahi = __ldcg(&nhi[c.x]); }
        else { uint32_t t = sorted_tri[~c.x]; alo = tlo[t]; ahi = thi[t]; }
        if (c.y >= 0) { blo = __ldcg(&nlo[c.y]); bhi = __ldcg(&nhi[c.y]); }
        else { uint32_t t = sorted_tri[~c.y]; blo = tlo[t]; bhi = thi[t]; }
        __stcg(&nlo[p], make_float4(fminf(alo.x, blo.x), fminf(alo.y, blo.y), fminf(alo.z, blo.z), 0.f));
        __stcg(&nhi[p], make_float4(fmaxf(ahi.x, bhi.x), fmaxf(ahi.y, bhi.y), fmaxf(ahi.z, bhi.z), 0.f));
        p = parent_int[p];
    }
}

// ------------------------------------------------------------- step 5b ----
// Treelet restructuring (Karras & Aila 2013, "Fast parallel construction of
// high-quality bounding volume hierarchies"): a second bottom-up pass over
// the binary tree. At each internal node p, once both of its subtrees are
// final, the treelet of p (p and the internal nodes below it found by
// repeatedly opening the treelet leaf of largest surface area, until
// kTreeletLeaves leaves) is rebuilt with the topology of least SAH cost over
// those leaves, found by dynamic programming over the leaves' subsets. The
// treelet keeps its node indices and its root's box; only the topology
// below the root changes. The pass also leaves every internal node's
// triangle count in cnt (the collapse reads it).
// SAH cost model: internal node kSahCi x its area, triangle kSahCt x its area.
constexpr int kTreeletLeaves = 7;
// passes of the restructuring; measured on a B200 (1 M-triangle heightfield,
// coherent / incoherent Mrays/s): none 5835 / 2043, 1 pass 6686 / 2250,
// 2 passes 6928 / 2319, 3 passes 6988 / 2331
constexpr int kTreeletPasses = 2;
constexpr float kSahCi = 1.2f, kSahCt = 1.0f;

__device__ __forceinline__ void handle_box(int c, const uint32_t *sorted_tri, const float4 *tlo, const float4 *thi,
                                           const float4 *nlo, const float4 *nhi, float3 &lo, float3 &hi)
{
    float4 a, b;
    if (c >= 0) { a = __ldcg(&nlo[c]); b = __ldcg(&nhi[c]); }
    else { const uint32_t t = sorted_tri[~c]; a = tlo[t]; b = thi[t]; }
    lo = make_float3(a.x, a.y, a.z);
    hi = make_float3(b.x, b.y, b.z);
}

// The 127 non-empty subsets of the 7 treelet leaves ordered by size (7 of
// size 1, 21 of size 2, 35, 35, 21, 7, 1), and where each size starts.
struct SubsetTable {
    uint8_t s[127];
    uint8_t start[8];
};
__constant__ SubsetTable c_subsets;

SubsetTable make_subset_table()
{
    SubsetTable t{};
    int k = 0;
    for (int size = 1; size <= kTreeletLeaves; size++) {
        t.start[size - 1] = (uint8_t)k;
        for (int S = 1; S < (1 << kTreeletLeaves); S++)
            if (__builtin_popcount(S) == size) t.s[k++] = (uint8_t)S;
    }
    t.start[kTreeletLeaves] = (uint8_t)k;
    return t;
}

constexpr int kTreeletThreads = 128;
constexpr int kTreeletWarps = kTreeletThreads / 32;

// One warp rebuilds the treelet of root p: every lane forms the same treelet
// (the reads are the same), the lanes fill the subsets of one size per round
// (each its own subsets' splits, against the smaller subsets of the rounds
// before), then lane 0 writes the new topology below p if it is cheaper.
// p's count and cost are final. All 32 lanes call this together.
__device__ void treelet_warp(int p, float costp, const uint32_t *sorted_tri, const float4 *tlo, const float4 *thi,
                             int2 *child, int *parent_int, int *parent_leaf, float4 *nlo, float4 *nhi, int *cnt,
                             float *cost, float *s_copt, uint8_t *s_split, float *s_box)
{
    const int lane = threadIdx.x & 31;
    __syncwarp();
    __threadfence();  // the subtree below p is final: written before its nodes' arrivals
    auto sub_cost = [&](int h) {
        if (h >= 0) return __ldcg(&cost[h]);
        float3 lo, hi;
        handle_box(h, sorted_tri, tlo, thi, nlo, nhi, lo, hi);
        return kSahCt * area(lo, hi);
    };
    int tl[kTreeletLeaves], tin[kTreeletLeaves - 1];
    const int2 c = __ldcg(&child[p]);
    float3 plo, phi;
    handle_box(p, sorted_tri, tlo, thi, nlo, nhi, plo, phi);
    int n_l = 2, n_in = 1;
    tl[0] = c.x;
    tl[1] = c.y;
    tin[0] = p;
    float cur = kSahCi * area(plo, phi);
    while (n_l < kTreeletLeaves) {
        int best = -1;
        float best_a = -1.f;
        for (int k = 0; k < n_l; k++) {
            if (tl[k] < 0) continue;
            float3 lo, hi;
            handle_box(tl[k], sorted_tri, tlo, thi, nlo, nhi, lo, hi);
            const float a = area(lo, hi);
            if (a > best_a) { best_a = a; best = k; }
        }
        if (best < 0) break;
        const int2 cc = __ldcg(&child[tl[best]]);
        tin[n_in++] = tl[best];
        cur += kSahCi * best_a;
        tl[best] = cc.x;
        tl[n_l++] = cc.y;
    }
    if (n_l < kTreeletLeaves) return;  // (not reached: p has >= 7 triangles)
    // leaf boxes and costs, one lane each
    if (lane < kTreeletLeaves) {
        float3 lo, hi;
        handle_box(tl[lane], sorted_tri, tlo, thi, nlo, nhi, lo, hi);
        float *bx = s_box + 6 * lane;
        bx[0] = lo.x; bx[1] = lo.y; bx[2] = lo.z; bx[3] = hi.x; bx[4] = hi.y; bx[5] = hi.z;
        s_copt[1 << lane] = sub_cost(tl[lane]);
    }
    __syncwarp();
    for (int k = 0; k < kTreeletLeaves; k++) cur += s_copt[1 << k];
    for (int size = 2; size <= kTreeletLeaves; size++) {
        for (int j = c_subsets.start[size - 1] + lane; j < c_subsets.start[size]; j += 32) {
            const int S = c_subsets.s[j];
            float3 lo = make_float3(FLT_MAX, FLT_MAX, FLT_MAX), hi = make_float3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
            for (int k = 0; k < kTreeletLeaves; k++) {
                if (!(S & (1 << k))) continue;
                const float *bx = s_box + 6 * k;
                lo = make_float3(fminf(lo.x, bx[0]), fminf(lo.y, bx[1]), fminf(lo.z, bx[2]));
                hi = make_float3(fmaxf(hi.x, bx[3]), fmaxf(hi.y, bx[4]), fmaxf(hi.z, bx[5]));
            }
            // splits P | S ^ P with P holding S's lowest leaf (each split once)
            const int low = S & -S;
            float best = FLT_MAX;
            int bp = low;
            for (int P = (S - 1) & S; P > 0; P = (P - 1) & S) {
                if (!(P & low)) continue;
                const float cc = s_copt[P] + s_copt[S ^ P];
                if (cc < best) { best = cc; bp = P; }
            }
            s_copt[S] = kSahCi * area(lo, hi) + best;
            s_split[S] = (uint8_t)bp;
        }
        __syncwarp();
    }
    constexpr int kAll = (1 << kTreeletLeaves) - 1;
    if (lane == 0 && s_copt[kAll] < cur * 0.9999f) {
        // rebuild below p with the treelet's own internal nodes
        int st_s[kTreeletLeaves], st_node[kTreeletLeaves];
        int sp = 0, pool = 1;
        st_s[sp] = kAll;
        st_node[sp++] = p;
        for (int it = 0; it < kTreeletLeaves && sp > 0; it++) {
            const int S = st_s[--sp], node = st_node[sp];
            const int parts[2] = {s_split[S], S ^ s_split[S]};
            int h[2];
            for (int q = 0; q < 2; q++) {
                const int P = parts[q];
                if ((P & (P - 1)) == 0) {
                    h[q] = tl[__ffs(P) - 1];
                } else {
                    h[q] = tin[pool++];
                    st_s[sp] = P;
                    st_node[sp++] = h[q];
                }
                if (h[q] >= 0) __stcg(&parent_int[h[q]], node);
                else __stcg(&parent_leaf[~h[q]], node);
            }
            __stcg(&child[node], make_int2(h[0], h[1]));
            if (node != p) {
                float3 lo = make_float3(FLT_MAX, FLT_MAX, FLT_MAX), hi = make_float3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
                int cn = 0;
                for (int k = 0; k < kTreeletLeaves; k++) {
                    if (!(S & (1 << k))) continue;
                    const float *bx = s_box + 6 * k;
                    lo = make_float3(fminf(lo.x, bx[0]), fminf(lo.y, bx[1]), fminf(lo.z, bx[2]));
                    hi = make_float3(fmaxf(hi.x, bx[3]), fmaxf(hi.y, bx[4]), fmaxf(hi.z, bx[5]));
                    cn += tl[k] >= 0 ? __ldcg(&cnt[tl[k]]) : 1;
                }
                __stcg(&nlo[node], make_float4(lo.x, lo.y, lo.z, 0.f));
                __stcg(&nhi[node], make_float4(hi.x, hi.y, hi.z, 0.f));
                __stcg(&cnt[node], cn);
            }
            __stcg(&cost[node], s_copt[S]);
        }
    }
    (void)costp;
    __syncwarp();
}

// The bottom-up pass: every lane walks up from its leaf; a lane whose node
// has both subtrees final (second arrival) sets the node's count and cost,
// and the warp then rebuilds, one after another, the treelets of the nodes
// its lanes hold that have >= kTreeletLeaves triangles. Lanes stay in the
// loop until the whole warp is done (the treelet work uses all 32).
__global__ void __launch_bounds__(kTreeletThreads) k_treelet(int n, const uint32_t *__restrict__ sorted_tri,
                                                             const float4 *__restrict__ tlo,
                                                             const float4 *__restrict__ thi, int2 *child,
                                                             int *parent_int, int *parent_leaf,
                                                             uint32_t *__restrict__ arrivals, float4 *nlo,
                                                             float4 *nhi, int *cnt, float *cost, int restructure)
{
    __shared__ float s_copt[kTreeletWarps][1 << kTreeletLeaves];
    __shared__ uint8_t s_split[kTreeletWarps][1 << kTreeletLeaves];
    __shared__ float s_box[kTreeletWarps][6 * kTreeletLeaves];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int w = threadIdx.x >> 5;
    int p = i < n ? parent_leaf[i] : -1;
    bool alive = i < n;
    for (int guard = 0; guard <= n; guard++) {
        bool ready = false;
        float costp = 0.f;
        if (alive && (p < 0 || p >= n - 1)) alive = false;
        if (alive) {
            __threadfence();
            if (atomicAdd(&arrivals[p], 1u) == 0) {
                alive = false;
            } else {
                __threadfence();
                ready = true;
                const int2 c = __ldcg(&child[p]);
                float3 plo, phi;
                handle_box(p, sorted_tri, tlo, thi, nlo, nhi, plo, phi);
                int cp = 0;
                float cc = kSahCi * area(plo, phi);
                for (int q = 0; q < 2; q++) {
                    const int h = q ? c.y : c.x;
                    if (h >= 0) {
                        cp += __ldcg(&cnt[h]);
                        cc += __ldcg(&cost[h]);
                    } else {
                        float3 lo, hi;
                        handle_box(h, sorted_tri, tlo, thi, nlo, nhi, lo, hi);
                        cp += 1;
                        cc += kSahCt * area(lo, hi);
                    }
                }
                __stcg(&cnt[p], cp);
                __stcg(&cost[p], cc);
                costp = cc;
                ready = restructure && cp >= kTreeletLeaves;
            }
        }
        unsigned todo = __ballot_sync(0xffffffffu, ready);
        while (todo) {
            const int leader = __ffs(todo) - 1;
            todo &= todo - 1;
            const int q = __shfl_sync(0xffffffffu, p, leader);
            const float qc = __shfl_sync(0xffffffffu, costp, leader);
            treelet_warp(q, qc, sorted_tri, tlo, thi, child, parent_int, parent_leaf, nlo, nhi, cnt, cost, s_copt[w],
                         s_split[w], s_box[w]);
        }
        if (alive) p = __ldcg(&parent_int[p]);
        if (!__any_sync(0xffffffffu, alive)) break;
    }
}

// ------------------------------------------------------------- step 5c ----
// Which binary nodes become 8-wide nodes, and which leaves, for least SAH
// cost (the dynamic program of Ylitie, Karras & Laine 2017, "Efficient
// incoherent ray traversal on GPUs through compressed wide BVHs", without its
// leaf reordering): bottom-up, for each binary node n and i = 1..8, the least
// cost of the subtree of n as at most i roots under an 8-wide parent. One
// root is n itself, as a leaf (<= kLeafMax triangles: its area x kColTri x
// its triangles) or as an 8-wide node (its area x kColNode + the least cost
// of its subtree below as at most 8 roots); more roots split the subtree
// between n's two children. Decisions per node (dpd, 16 bytes): [0] n as one
// root is a leaf (1) or an 8-wide node (0); [j - 1], j = 2..8: the left
// child's share of a j-root split; [8 + i - 1]: the roots (1 = n itself, or
// the split j) that give the least cost with at most i roots.
constexpr float kColNode = 1.0f, kColTri = 0.3f;

__device__ __forceinline__ void root_costs(int h, const uint32_t *sorted_tri, const float4 *tlo, const float4 *thi,
                                           const float *dpc, float (&c)[8])
{
    if (h < 0) {
        const uint32_t t = sorted_tri[~h];
        const float4 lo = tlo[t], hi = thi[t];
        const float a = kColTri * area(make_float3(lo.x, lo.y, lo.z), make_float3(hi.x, hi.y, hi.z));
#pragma unroll
        for (int i = 0; i < 8; i++) c[i] = a;
    } else {
        const float4 *src = reinterpret_cast<const float4 *>(dpc + 8 * (size_t)h);
        const float4 x = __ldcg(src), y = __ldcg(src + 1);
        c[0] = x.x; c[1] = x.y; c[2] = x.z; c[3] = x.w; c[4] = y.x; c[5] = y.y; c[6] = y.z; c[7] = y.w;
    }
}

__global__ void __launch_bounds__(128) k_collapse_cost(int n, const uint32_t *__restrict__ sorted_tri,
                                                       const float4 *__restrict__ tlo, const float4 *__restrict__ thi,
                                                       const int2 *__restrict__ child, const int *__restrict__ parent_int,
                                                       const int *__restrict__ parent_leaf,
                                                       uint32_t *__restrict__ arrivals, const float4 *__restrict__ nlo,
                                                       const float4 *__restrict__ nhi, const int *__restrict__ cnt,
                                                       float *dpc, uint8_t *__restrict__ dpd)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int p = parent_leaf[i];
    for (int guard = 0; p >= 0 && p < n - 1 && guard < n; guard++) {
        __threadfence();
        if (atomicAdd(&arrivals[p], 1u) == 0) return;
        __threadfence();
        const int2 c = child[p];
        float ca[8], cb[8];
        root_costs(c.x, sorted_tri, tlo, thi, dpc, ca);
        root_costs(c.y, sorted_tri, tlo, thi, dpc, cb);
        uint8_t dec[16];
        float split[8];  // [j - 1]: least cost of j roots split between the children
#pragma unroll
        for (int j = 2; j <= 8; j++) {
            float best = FLT_MAX;
            int bk = 1;
#pragma unroll
            for (int k = 1; k < j; k++) {
                const float v = ca[k - 1] + cb[j - k - 1];
                if (v < best) { best = v; bk = k; }
            }
            split[j - 1] = best;
            dec[j - 1] = (uint8_t)bk;
        }
        const float4 lo = nlo[p], hi = nhi[p];
        const float a = area(make_float3(lo.x, lo.y, lo.z), make_float3(hi.x, hi.y, hi.z));
        const int np = cnt[p];
        const float as_leaf = np <= kLeafMax ? kColTri * a * (float)np : FLT_MAX;
        const float as_node = kColNode * a + split[7];
        float cost[8];
        cost[0] = fminf(as_leaf, as_node);
        dec[0] = as_leaf <= as_node ? 1u : 0u;
        dec[8] = 1;
#pragma unroll
        for (int k = 2; k <= 8; k++) {
            cost[k - 1] = cost[k - 2];
            dec[8 + k - 1] = dec[8 + k - 2];
            if (split[k - 1] < cost[k - 1]) {
                cost[k - 1] = split[k - 1];
                dec[8 + k - 1] = (uint8_t)k;
            }
        }
        float4 *dst = reinterpret_cast<float4 *>(dpc + 8 * (size_t)p);
        __stcg(dst, make_float4(cost[0], cost[1], cost[2], cost[3]));
        __stcg(dst + 1, make_float4(cost[4], cost[5], cost[6], cost[7]));
        uint4 d;
        memcpy(&d, dec, 16);
        *reinterpret_cast<uint4 *>(dpd + 16 * (size_t)p) = d;
        p = parent_int[p];
    }
}

// ---------------------------------------------------------------- step 6 ----
struct Work {
    int bin;       // binary node: >= 0 internal, < 0 leaf ~sorted_pos (only for n == 1)
    uint32_t node; // 8-wide node index to fill
};

static_assert(sizeof(Work) == 8, "work item is 8 bytes");

__device__ __forceinline__ void child_box(int c, const uint32_t *sorted_tri, const float4 *tlo, const float4 *thi,
                                          const float4 *nlo, const float4 *nhi, float3 &lo, float3 &hi)
{
    float4 a, b;
    if (c >= 0) { a = nlo[c]; b = nhi[c]; }
    else { uint32_t t = sorted_tri[~c]; a = tlo[t]; b = thi[t]; }
    lo = make_float3(a.x, a.y, a.z);
    hi = make_float3(b.x, b.y, b.z);
}

// triangles below handle c (an internal node's count from k_treelet)
__device__ __forceinline__ int child_count(int c, const int *cnt) { return c >= 0 ? cnt[c] : 1; }

// whether root handle c becomes an 8-wide node (else a leaf child)
__device__ __forceinline__ bool is_node_root(int c, const uint8_t *dpd) { return c >= 0 && dpd[16 * (size_t)c] == 0; }

// The sorted positions of the triangles below handle c, which holds at most
// kLeafMax of them, left to right. Returns how many.
__device__ __forceinline__ int leaf_tris(int c, const int2 *child, int (&out)[kLeafMax])
{
    int st[2 * kLeafMax], sp = 0, m = 0;
    st[sp++] = c;
    for (int it = 0; it < 4 * kLeafMax && sp > 0; it++) {
        const int x = st[--sp];
        if (x < 0) {
            if (m < kLeafMax) out[m++] = ~x;
        } else if (sp + 2 <= 2 * kLeafMax) {
            const int2 cc = child[x];
            st[sp++] = cc.y;
            st[sp++] = cc.x;
        }
    }
    return m;
}

// Quantisation step for one axis: the smallest power of two 2^e with
// extent / 2^e <= 255 - 2 (one step of slack each side), and never below
// `min_step` so that a step stays many float ulps wide.
__device__ __forceinline__ int quant_exp(float extent, float min_step)
{
    float target = fmaxf(extent / 253.0f, min_step);
    int e;
    frexpf(target, &e);  // target = m * 2^e, m in [0.5, 1)  ->  2^e >= target
    e = max(e, -120);
    e = min(e, 127);
    return e;
}

__device__ __forceinline__ float exp2i(int e) { return ldexpf(1.0f, e); }

__global__ void k_collapse(const Work *__restrict__ in, const uint32_t *__restrict__ in_count, Work *__restrict__ out,
                           uint32_t *__restrict__ out_count, uint32_t out_cap, const int2 *__restrict__ child,
                           const int *__restrict__ cnt, const uint8_t *__restrict__ dpd, const float4 *__restrict__ nlo,
                           const float4 *__restrict__ nhi, const uint32_t *__restrict__ sorted_tri,
                           const float4 *__restrict__ tlo, const float4 *__restrict__ thi,
                           const float *__restrict__ pos, const uint32_t *__restrict__ idx, Node8 *__restrict__ nodes,
                           uint32_t *__restrict__ node_count, uint32_t node_cap, Tri *__restrict__ tris,
                           uint32_t *__restrict__ prim_of, uint32_t *__restrict__ tri_count, uint32_t tri_cap,
                           float min_step, uint32_t *__restrict__ err)
{
    uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= *in_count) return;
    const Work job = in[w];

    int ch[8];
    int m = 0;
    if (job.bin >= 0) {
        // the roots the collapse costs chose for this node's subtree below
        // it: its children's split of 8 roots, each side followed down to the
        // handles that stand as one root
        const int2 c = child[job.bin];
        const int k8 = dpd[16 * (size_t)job.bin + 7];
        int st_h[16], st_i[16], sp = 0;
        st_h[sp] = c.y;
        st_i[sp++] = 8 - k8;
        st_h[sp] = c.x;
        st_i[sp++] = k8;
        for (int it = 0; it < 32 && sp > 0 && m < 8; it++) {
            const int h = st_h[--sp], r = st_i[sp];
            const int j = h >= 0 ? dpd[16 * (size_t)h + 8 + r - 1] : 1;
            if (j <= 1 || sp + 2 > 16) {
                ch[m++] = h;
                continue;
            }
            const int k = dpd[16 * (size_t)h + j - 1];
            const int2 cc = child[h];
            st_h[sp] = cc.y;
            st_i[sp++] = j - k;
            st_h[sp] = cc.x;
            st_i[sp++] = k;
        }
        if (sp > 0) { atomicOr(err, 16u); return; }
    } else {
        ch[m++] = job.bin;  // single-triangle scene
    }

    // child boxes, centroids, classification
    float3 clo[8], chi[8];
    float3 plo = make_float3(FLT_MAX, FLT_MAX, FLT_MAX), phi = make_float3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    int n_int = 0, n_leaf_tris = 0;
    for (int k = 0; k < m; k++) {
        child_box(ch[k], sorted_tri, tlo, thi, nlo, nhi, clo[k], chi[k]);
        plo = make_float3(fminf(plo.x, clo[k].x), fminf(plo.y, clo[k].y), fminf(plo.z, clo[k].z));
        phi = make_float3(fmaxf(phi.x, chi[k].x), fmaxf(phi.y, chi[k].y), fmaxf(phi.z, chi[k].z));
        if (is_node_root(ch[k], dpd)) n_int++;
        else n_leaf_tris += child_count(ch[k], cnt);
    }

    // slot assignment: slot s is the corner with bit k set = positive along axis k
    int slot_of[8];
    {
        float3 pc = make_float3(0.5f * (plo.x + phi.x), 0.5f * (plo.y + phi.y), 0.5f * (plo.z + phi.z));
        float score[8][8];
        for (int k = 0; k < m; k++) {
            float3 c = make_float3(0.5f * (clo[k].x + chi[k].x) - pc.x, 0.5f * (clo[k].y + chi[k].y) - pc.y,
                                   0.5f * (clo[k].z + chi[k].z) - pc.z);
            for (int s = 0; s < 8; s++)
                score[k][s] = ((s & 1) ? c.x : -c.x) + ((s & 2) ? c.y : -c.y) + ((s & 4) ? c.z : -c.z);
        }
        uint32_t used_slots = 0, used_kids = 0;
        for (int it = 0; it < m; it++) {
            float best = -FLT_MAX;
            int bk = -1, bs = -1;
            for (int k = 0; k < m; k++) {
                if (used_kids & (1u << k)) continue;
                for (int s = 0; s < 8; s++) {
                    if (used_slots & (1u << s)) continue;
                    if (score[k][s] > best || bk < 0) { best = score[k][s]; bk = k; bs = s; }
                }
            }
            used_kids |= 1u << bk;
            used_slots |= 1u << bs;
            slot_of[bk] = bs;
        }
    }

    // allocate children and triangle records
    uint32_t child_base = 0, tri_base = 0;
    if (n_int) {
        child_base = atomicAdd(node_count, (uint32_t)n_int);
        if (child_base + n_int > node_cap) { atomicOr(err, 2u); return; }
    }
    if (n_leaf_tris) {
        tri_base = atomicAdd(tri_count, (uint32_t)n_leaf_tris);
        if (tri_base + n_leaf_tris > tri_cap) { atomicOr(err, 4u); return; }
    }

    // quantisation frame
    int ex = quant_exp(phi.x - plo.x, min_step), ey = quant_exp(phi.y - plo.y, min_step),
        ez = quant_exp(phi.z - plo.z, min_step);
    float sx = exp2i(ex), sy = exp2i(ey), sz = exp2i(ez);
    // origin one step below the union so that floor() never goes negative
    float3 org = make_float3(plo.x - sx, plo.y - sy, plo.z - sz);

    uint8_t meta[8], qlx[8], qly[8], qlz[8], qhx[8], qhy[8], qhz[8];
    for (int s = 0; s < 8; s++) meta[s] = qlx[s] = qly[s] = qlz[s] = qhx[s] = qhy[s] = qhz[s] = 0;

    // internal children in slot order -> contiguous child nodes
    uint32_t imask = 0;
    for (int k = 0; k < m; k++)
        if (is_node_root(ch[k], dpd)) imask |= 1u << slot_of[k];
    int tri_off = 0;
    for (int s = 0; s < 8; s++) {
        int k = -1;
        for (int q = 0; q < m; q++)
            if (slot_of[q] == s) k = q;
        if (k < 0) continue;
        // conservative 8-bit box: floor/ceil in double (exact for float inputs),
        // one extra step of slack each side
        double lx = floor(((double)clo[k].x - org.x) / sx) - 1, ly = floor(((double)clo[k].y - org.y) / sy) - 1,
               lz = floor(((double)clo[k].z - org.z) / sz) - 1;
        double hx = ceil(((double)chi[k].x - org.x) / sx) + 1, hy = ceil(((double)chi[k].y - org.y) / sy) + 1,
               hz = ceil(((double)chi[k].z - org.z) / sz) + 1;
        qlx[s] = (uint8_t)fmin(fmax(lx, 0.0), 255.0);
        qly[s] = (uint8_t)fmin(fmax(ly, 0.0), 255.0);
        qlz[s] = (uint8_t)fmin(fmax(lz, 0.0), 255.0);
        qhx[s] = (uint8_t)fmin(fmax(hx, 0.0), 255.0);
        qhy[s] = (uint8_t)fmin(fmax(hy, 0.0), 255.0);
        qhz[s] = (uint8_t)fmin(fmax(hz, 0.0), 255.0);
        if (imask & (1u << s)) {
            meta[s] = (uint8_t)kMetaInternal;
            uint32_t ci = child_base + __popc(imask & ((1u << s) - 1u));
            uint32_t slot = atomicAdd(out_count, 1u);
            if (slot >= out_cap) { atomicOr(err, 8u); continue; }
            out[slot] = Work{ch[k], ci};
        } else {
            int pos_of[kLeafMax];
            const int nt = leaf_tris(ch[k], child, pos_of);
            meta[s] = (uint8_t)((nt << 5) | tri_off);
            for (int q = 0; q < nt; q++) {
                uint32_t t = sorted_tri[pos_of[q]];
                uint32_t a = idx[3 * t], b = idx[3 * t + 1], c = idx[3 * t + 2];
                float v0x = pos[3 * a], v0y = pos[3 * a + 1], v0z = pos[3 * a + 2];
                float e1x = __fsub_rn(pos[3 * b], v0x), e1y = __fsub_rn(pos[3 * b + 1], v0y),
                      e1z = __fsub_rn(pos[3 * b + 2], v0z);
                float e2x = __fsub_rn(pos[3 * c], v0x), e2y = __fsub_rn(pos[3 * c + 1], v0y),
                      e2z = __fsub_rn(pos[3 * c + 2], v0z);
                float nx = __fsub_rn(__fmul_rn(e1y, e2z), __fmul_rn(e1z, e2y));
                float ny = __fsub_rn(__fmul_rn(e1z, e2x), __fmul_rn(e1x, e2z));
                float nz = __fsub_rn(__fmul_rn(e1x, e2y), __fmul_rn(e1y, e2x));
                Tri tr;
                tr.a = make_float4(v0x, v0y, v0z, nx);
                tr.b = make_float4(e1x, e1y, e1z, ny);
                tr.c = make_float4(e2x, e2y, e2z, nz);
                tris[tri_base + tri_off + q] = tr;
                prim_of[tri_base + tri_off + q] = t;
            }
            tri_off += nt;
        }
    }

    auto pack4 = [](const uint8_t *b) {
        return (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
    };
    Node8 nd;
    nd.q[0] = make_uint4(__float_as_uint(org.x), __float_as_uint(org.y), __float_as_uint(org.z),
                         (uint32_t)(ex + 127) | ((uint32_t)(ey + 127) << 8) | ((uint32_t)(ez + 127) << 16) |
                             (imask << 24));
    nd.q[1] = make_uint4(child_base, tri_base, pack4(meta), pack4(meta + 4));
    nd.q[2] = make_uint4(pack4(qlx), pack4(qlx + 4), pack4(qhx), pack4(qhx + 4));
    nd.q[3] = make_uint4(pack4(qly), pack4(qly + 4), pack4(qhy), pack4(qhy + 4));
    nd.q[4] = make_uint4(pack4(qlz), pack4(qlz + 4), pack4(qhz), pack4(qhz + 4));
    nodes[job.node] = nd;
}

__global__ void k_root(Work *q, uint32_t *count, int n, uint32_t *node_count)
{
    q[0] = Work{n > 1 ? 0 : ~0, 0u};
    *count = 1;
    *node_count = 1;
}

inline uint32_t div_up(uint64_t a, uint32_t b) { return (uint32_t)((a + b - 1) / b); }

}  // namespace

// ---------------------------------------------------------------------------
#define ILG_CK(call)                                                                       \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            snprintf(err, err_len, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return 3;                                                                      \
        }                                                                                  \
    } while (0)

int bvh_build(BuildBuffers &B, const float *d_pos, uint32_t n_verts, const uint32_t *d_idx, uint32_t n,
              cudaStream_t st, BuildResult &res, char *err, size_t err_len)
{
    if (n == 0) {
        snprintf(err, err_len, "ilg_build: empty mesh");
        return 1;
    }
    // scratch sizing
    size_t sort_tmp = 0;
    ILG_CK(cub::DeviceRadixSort::SortPairs(nullptr, sort_tmp, (uint32_t *)nullptr, (uint32_t *)nullptr,
                                           (uint32_t *)nullptr, (uint32_t *)nullptr, (int)n, 0, 30, st));
    const uint32_t node_cap = n;           // 8-wide nodes never exceed the triangle count
    const uint32_t tri_cap = n;
    const uint32_t queue_cap = n + 1;
    ILG_CK(B.reserve(n, sort_tmp, node_cap, queue_cap, st));

    ILG_CK(cudaMemsetAsync(B.err, 0, sizeof(uint32_t), st));
    uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    ILG_CK(cudaMemcpyAsync(B.cbounds, init, sizeof(init), cudaMemcpyHostToDevice, st));
    const uint32_t T = 256;
    k_tri_bounds<<<div_up(n, T), T, 0, st>>>(d_pos, n_verts, d_idx, n, B.tlo, B.thi, B.cbounds, B.err);
    k_morton<<<div_up(n, T), T, 0, st>>>(B.tlo, B.thi, n, B.cbounds, B.keys, B.vals);
    ILG_CK(cudaGetLastError());
    ILG_CK(cub::DeviceRadixSort::SortPairs(B.sort_tmp, sort_tmp, B.keys, B.keys_alt, B.vals, B.vals_alt, (int)n, 0,
                                           30, st));
    if (n > 1) {
        k_karras<<<div_up(n - 1, T), T, 0, st>>>(B.keys_alt, (int)n, B.child, B.parent_int, B.parent_leaf, B.range);
        ILG_CK(cudaMemsetAsync(B.arrivals, 0, sizeof(uint32_t) * (n - 1), st));
        k_refit<<<div_up(n, T), T, 0, st>>>((int)n, B.vals_alt, B.tlo, B.thi, B.child, B.parent_int, B.parent_leaf,
                                             B.arrivals, B.nlo, B.nhi);
        ILG_CK(cudaGetLastError());
        if (res.treelets) {
            static const SubsetTable table = make_subset_table();
            ILG_CK(cudaMemcpyToSymbolAsync(c_subsets, &table, sizeof(table), 0, cudaMemcpyHostToDevice, st));
        }
        for (int pass = 0; pass < (res.treelets ? kTreeletPasses : 1); pass++) {
            ILG_CK(cudaMemsetAsync(B.arrivals, 0, sizeof(uint32_t) * (n - 1), st));
            k_treelet<<<div_up(n, kTreeletThreads), kTreeletThreads, 0, st>>>((int)n, B.vals_alt, B.tlo, B.thi, B.child, B.parent_int,
                                                      B.parent_leaf, B.arrivals, B.nlo, B.nhi, B.cnt, B.cost,
                                                      res.treelets ? 1 : 0);
            ILG_CK(cudaGetLastError());
        }
        ILG_CK(cudaMemsetAsync(B.arrivals, 0, sizeof(uint32_t) * (n - 1), st));
        k_collapse_cost<<<div_up(n, 128), 128, 0, st>>>((int)n, B.vals_alt, B.tlo, B.thi, B.child, B.parent_int,
                                                        B.parent_leaf, B.arrivals, B.nlo, B.nhi, B.cnt, B.dpc, B.dpd);
        ILG_CK(cudaGetLastError());
    }
    ILG_CK(cudaMemsetAsync(B.counters, 0, 4 * sizeof(uint32_t), st));
    // counters: [0] node_count, [1] tri_count, [2] queue A count, [3] queue B count
    k_root<<<1, 1, 0, st>>>((Work *)B.qa_raw, B.counters + 2, (int)n, B.counters + 0);
    ILG_CK(cudaGetLastError());

    const float min_step = res.min_step;
    Work *qin = (Work *)B.qa_raw, *qout = (Work *)B.qb_raw;
    uint32_t *cin = B.counters + 2, *cout = B.counters + 3;
    uint32_t host_in = 1;
    uint32_t depth = 0;
    while (host_in > 0) {
        ILG_CK(cudaMemsetAsync(cout, 0, sizeof(uint32_t), st));
        k_collapse<<<div_up(host_in, 64), 64, 0, st>>>(qin, cin, qout, cout, queue_cap, B.child, B.cnt, B.dpd, B.nlo,
                                                        B.nhi, B.vals_alt, B.tlo, B.thi, d_pos, d_idx, B.nodes,
                                                        B.counters + 0, node_cap, B.tris, B.prim_of, B.counters + 1,
                                                        tri_cap, min_step, B.err);
        ILG_CK(cudaGetLastError());
        ILG_CK(cudaMemcpyAsync(&host_in, cout, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        ILG_CK(cudaStreamSynchronize(st));
        depth++;
        if (depth > 200) {
            snprintf(err, err_len, "ilg_build: collapse did not converge");
            return 5;
        }
        std::swap(qin, qout);
        std::swap(cin, cout);
    }
    uint32_t h[4], herr = 0;
    ILG_CK(cudaMemcpyAsync(h, B.counters, sizeof(h), cudaMemcpyDeviceToHost, st));
    ILG_CK(cudaMemcpyAsync(&herr, B.err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    ILG_CK(cudaStreamSynchronize(st));
    if (herr & 1u) {
        snprintf(err, err_len, "ilg_build: triangle index out of range of the vertex array");
        return 1;
    }
    if (herr) {
        snprintf(err, err_len, "ilg_build: capacity exceeded (flags 0x%x)", herr);
        return 5;
    }
    if (h[1] != n) {
        snprintf(err, err_len, "ilg_build: %u triangle records written for %u triangles", h[1], n);
        return 5;
    }
    res.n_nodes = h[0];
    res.n_tris = h[1];
    res.depth = depth;
    return 0;
}

}  // namespace ilg
