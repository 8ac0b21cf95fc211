// Batched closest-hit / any-hit kernels over the 8-wide BVH.
#include "trace.cuh"
#include "trace_api.cuh"
#include "devinfo.cuh"

#include <algorithm>

namespace ilg {

namespace {

template <bool kStats, bool kSkip = false>
__global__ void __launch_bounds__(128) k_closest(const Node8 *__restrict__ nodes, const Tri *__restrict__ tris,
                                                 const uint32_t *__restrict__ prim_of, uint32_t n_nodes_total,
                                                 uint32_t n_tris_total,
                                                 const float4 *__restrict__ ro, const float4 *__restrict__ rd,
                                                 uint32_t n, int32_t *__restrict__ prim, float *__restrict__ tout,
                                                 float *__restrict__ uout, float *__restrict__ vout,
                                                 uint32_t *__restrict__ err, unsigned long long *__restrict__ stats,
                                                 uint32_t skip_lo = 0, uint32_t skip_n = 0)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 o = __ldcs(ro + i), d = __ldcs(rd + i);
    int best;
    float bt, bu, bv;
    unsigned long long nn = 0, nt = 0;
    trace_one<false, kStats, kSkip>(nodes, tris, n_nodes_total, n_tris_total, o, d, best, bt, bu, bv, err, nn, nt,
                                    Skip{prim_of, skip_lo, skip_n});
    __stcs(prim + i, best >= 0 ? (int32_t)__ldg(prim_of + best) : (best == -2 ? -2 : -1));
    __stcs(tout + i, bt);
    __stcs(uout + i, bu);
    __stcs(vout + i, bv);
    if (kStats) {
        atomicAdd(&stats[0], nn);
        atomicAdd(&stats[1], nt);
    }
}

template <bool kSkip = false>
__global__ void __launch_bounds__(128) k_any(const Node8 *__restrict__ nodes, const Tri *__restrict__ tris,
                                             uint32_t n_nodes_total, uint32_t n_tris_total,
                                             const float4 *__restrict__ ro, const float4 *__restrict__ rd,
                                             uint32_t n, uint8_t *__restrict__ occ, uint32_t *__restrict__ err,
                                             const uint32_t *__restrict__ prim_of = nullptr, uint32_t skip_lo = 0,
                                             uint32_t skip_n = 0)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 o = __ldcs(ro + i), d = __ldcs(rd + i);
    int best;
    float bt, bu, bv;
    unsigned long long nn = 0, nt = 0;
    trace_one<true, false, kSkip>(nodes, tris, n_nodes_total, n_tris_total, o, d, best, bt, bu, bv, err, nn, nt,
                                  Skip{prim_of, skip_lo, skip_n});
    occ[i] = best >= 0 ? 1 : 0;
}

// Persistent closest / any hit with dynamic ray fetch (see trace.cuh);
// kWT: the watertight triangle test over `raw`.
template <bool kAnyHit, bool kWT = false>
__global__ void __launch_bounds__(128) k_trace_dyn(const Node8 *__restrict__ nodes, const Tri *__restrict__ tris,
                                                   const uint32_t *__restrict__ prim_of, uint32_t n_nodes_total,
                                                   uint32_t n_tris_total, const float4 *__restrict__ ro,
                                                   const float4 *__restrict__ rd, uint32_t n,
                                                   int32_t *__restrict__ prim, float *__restrict__ tout,
                                                   float *__restrict__ uout, float *__restrict__ vout,
                                                   uint8_t *__restrict__ occ, uint32_t *__restrict__ next,
                                                   uint32_t *__restrict__ err, const float4 *__restrict__ raw = nullptr)
{
    const uint32_t lane = threadIdx.x & 31u;
    static_assert(kStackColumns == 128, "k_trace_dyn runs 128 threads a block");
    __shared__ uint2 sstack[kShortStack * kStackColumns];
    uint2 lstack[kMaxStack - kShortStack];
    const SplitStack stack{sstack + threadIdx.x, lstack};
    RayState r;
    bool active = false, exhausted = false;  // exhausted is warp-uniform
    uint32_t id = 0;
    while (true) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !active);
        if (!exhausted && (__popc(idle) >= kRefillLanesQuery || idle == 0xffffffffu)) {
            const uint32_t leader = __ffs(idle) - 1u;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(next, (uint32_t)__popc(idle));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base >= n) exhausted = true;
            if (!active) {
                const uint32_t k = base + __popc(idle & ((1u << lane) - 1u));
                if (k < n) {
                    id = k;
                    ray_init<kWT>(r, __ldcs(ro + id), __ldcs(rd + id), n_nodes_total);
                    active = true;
                }
            }
        }
        if (__ballot_sync(0xffffffffu, active) == 0u) break;
        if (active && ray_step<kAnyHit, false, false, kWT, kTrisPerStep, false, SplitStack>(r, stack, nodes, tris, n_nodes_total, n_tris_total, err,
                                                            nullptr, nullptr, Skip{nullptr, 0u, 0u}, raw)) {
            if (kAnyHit) {
                occ[id] = r.best >= 0 ? 1 : 0;
            } else {
                __stcs(prim + id, r.best >= 0 ? (int32_t)__ldg(prim_of + r.best) : (r.best == -2 ? -2 : -1));
                __stcs(tout + id, r.best >= 0 ? r.tcur : __int_as_float(0x7f800000));
                __stcs(uout + id, r.best >= 0 ? r.bu : 0.f);
                __stcs(vout + id, r.best >= 0 ? r.bv : 0.f);
            }
            active = false;
        }
    }
}

int sm_count() { return current_sm_count(); }

}  // namespace

cudaError_t preload_closest_dyn()
{
    cudaFuncAttributes a;
    return cudaFuncGetAttributes(&a, (const void *)k_trace_dyn<false>);
}

cudaError_t launch_closest_dyn(const SceneView &s, const float4 *ro, const float4 *rd, uint32_t n, int32_t *prim,
                               float *t, float *u, float *v, uint32_t *next, uint32_t *err, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(next, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const uint32_t blocks = std::min<uint32_t>((n + 127) / 128, (uint32_t)sm_count() * 16u);
    k_trace_dyn<false><<<blocks, 128, 0, st>>>(s.nodes, s.tris, s.prim_of, s.n_nodes, s.n_tris, ro, rd, n, prim, t,
                                               u, v, nullptr, next, err);
    return cudaGetLastError();
}

cudaError_t launch_any_dyn(const SceneView &s, const float4 *ro, const float4 *rd, uint32_t n, uint8_t *occ,
                           uint32_t *next, uint32_t *err, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(next, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const uint32_t blocks = std::min<uint32_t>((n + 127) / 128, (uint32_t)sm_count() * 16u);
    k_trace_dyn<true><<<blocks, 128, 0, st>>>(s.nodes, s.tris, nullptr, s.n_nodes, s.n_tris, ro, rd, n, nullptr,
                                              nullptr, nullptr, nullptr, occ, next, err);
    return cudaGetLastError();
}

cudaError_t launch_closest_wt(const SceneView &s, const float4 *raw, const float4 *ro, const float4 *rd, uint32_t n,
                              int32_t *prim, float *t, float *u, float *v, uint32_t *next, uint32_t *err,
                              cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(next, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const uint32_t blocks = std::min<uint32_t>((n + 127) / 128, (uint32_t)sm_count() * 16u);
    k_trace_dyn<false, true><<<blocks, 128, 0, st>>>(s.nodes, s.tris, s.prim_of, s.n_nodes, s.n_tris, ro, rd, n,
                                                     prim, t, u, v, nullptr, next, err, raw);
    return cudaGetLastError();
}

cudaError_t launch_any_wt(const SceneView &s, const float4 *raw, const float4 *ro, const float4 *rd, uint32_t n,
                          uint8_t *occ, uint32_t *next, uint32_t *err, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(next, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const uint32_t blocks = std::min<uint32_t>((n + 127) / 128, (uint32_t)sm_count() * 16u);
    k_trace_dyn<true, true><<<blocks, 128, 0, st>>>(s.nodes, s.tris, nullptr, s.n_nodes, s.n_tris, ro, rd, n,
                                                    nullptr, nullptr, nullptr, nullptr, occ, next, err, raw);
    return cudaGetLastError();
}

// Three float4 vertices per triangle record, in record order: the input
// vertices of the record's triangle, copied bit for bit.
__global__ void k_raw_tris(const uint32_t *__restrict__ prim_of, const uint32_t *__restrict__ idx,
                           const float *__restrict__ pos, uint32_t n, float4 *__restrict__ raw)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t p = prim_of[i];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const uint32_t v = idx[3ull * p + c];
        raw[3ull * i + c] = make_float4(pos[3ull * v], pos[3ull * v + 1], pos[3ull * v + 2], 0.f);
    }
}

cudaError_t build_raw_tris(const uint32_t *prim_of, const uint32_t *idx, const float *pos, uint32_t n, float4 *raw,
                           cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    k_raw_tris<<<(n + 255) / 256, 256, 0, st>>>(prim_of, idx, pos, n, raw);
    return cudaGetLastError();
}

cudaError_t launch_closest(const SceneView &s, const float4 *ro, const float4 *rd, uint32_t n, int32_t *prim,
                           float *t, float *u, float *v, uint32_t *err, unsigned long long *stats, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    const uint32_t T = 128;
    const uint32_t blocks = (n + T - 1) / T;
    if (stats)
        k_closest<true><<<blocks, T, 0, st>>>(s.nodes, s.tris, s.prim_of, s.n_nodes, s.n_tris, ro, rd, n, prim, t, u, v, err, stats);
    else
        k_closest<false><<<blocks, T, 0, st>>>(s.nodes, s.tris, s.prim_of, s.n_nodes, s.n_tris, ro, rd, n, prim, t, u, v, err, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_any(const SceneView &s, const float4 *ro, const float4 *rd, uint32_t n, uint8_t *occ,
                       uint32_t *err, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    const uint32_t T = 128;
    k_any<false><<<(n + T - 1) / T, T, 0, st>>>(s.nodes, s.tris, s.n_nodes, s.n_tris, ro, rd, n, occ, err);
    return cudaGetLastError();
}

cudaError_t launch_closest_skip(const SceneView &s, const float4 *ro, const float4 *rd, uint32_t n,
                                uint32_t skip_lo, uint32_t skip_n, int32_t *prim, float *t, float *u, float *v,
                                uint32_t *err, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    const uint32_t T = 128;
    k_closest<false, true><<<(n + T - 1) / T, T, 0, st>>>(s.nodes, s.tris, s.prim_of, s.n_nodes, s.n_tris, ro, rd, n,
                                                          prim, t, u, v, err, nullptr, skip_lo, skip_n);
    return cudaGetLastError();
}

cudaError_t launch_any_skip(const SceneView &s, const float4 *ro, const float4 *rd, uint32_t n, uint32_t skip_lo,
                            uint32_t skip_n, uint8_t *occ, uint32_t *err, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    const uint32_t T = 128;
    k_any<true><<<(n + T - 1) / T, T, 0, st>>>(s.nodes, s.tris, s.n_nodes, s.n_tris, ro, rd, n, occ, err, s.prim_of,
                                               skip_lo, skip_n);
    return cudaGetLastError();
}

}  // namespace ilg
