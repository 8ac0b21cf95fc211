// Batched closest-hit / any-hit kernels over the 8-wide BVH.
#include "trace.cuh"
#include "trace_api.cuh"

namespace ilg {

namespace {

template <bool kStats>
__global__ void __launch_bounds__(128) k_closest(const Node8 *__restrict__ nodes, const Tri *__restrict__ tris,
                                                 const uint32_t *__restrict__ prim_of, uint32_t n_nodes_total,
                                                 uint32_t n_tris_total,
                                                 const float4 *__restrict__ ro, const float4 *__restrict__ rd,
                                                 uint32_t n, int32_t *__restrict__ prim, float *__restrict__ tout,
                                                 float *__restrict__ uout, float *__restrict__ vout,
                                                 uint32_t *__restrict__ err, unsigned long long *__restrict__ stats)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 o = __ldcs(ro + i), d = __ldcs(rd + i);
    int best;
    float bt, bu, bv;
    unsigned long long nn = 0, nt = 0;
    trace_one<false, kStats>(nodes, tris, n_nodes_total, n_tris_total, o, d, best, bt, bu, bv, err, nn, nt);
    __stcs(prim + i, best >= 0 ? (int32_t)__ldg(prim_of + best) : (best == -2 ? -2 : -1));
    __stcs(tout + i, bt);
    __stcs(uout + i, bu);
    __stcs(vout + i, bv);
    if (kStats) {
        atomicAdd(&stats[0], nn);
        atomicAdd(&stats[1], nt);
    }
}

__global__ void __launch_bounds__(128) k_any(const Node8 *__restrict__ nodes, const Tri *__restrict__ tris,
                                             uint32_t n_nodes_total, uint32_t n_tris_total,
                                             const float4 *__restrict__ ro, const float4 *__restrict__ rd,
                                             uint32_t n, uint8_t *__restrict__ occ, uint32_t *__restrict__ err)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 o = __ldcs(ro + i), d = __ldcs(rd + i);
    int best;
    float bt, bu, bv;
    unsigned long long nn = 0, nt = 0;
    trace_one<true, false>(nodes, tris, n_nodes_total, n_tris_total, o, d, best, bt, bu, bv, err, nn, nt);
    occ[i] = best >= 0 ? 1 : 0;
}

}  // namespace

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
    k_any<<<(n + T - 1) / T, T, 0, st>>>(s.nodes, s.tris, s.n_nodes, s.n_tris, ro, rd, n, occ, err);
    return cudaGetLastError();
}

}  // namespace ilg
