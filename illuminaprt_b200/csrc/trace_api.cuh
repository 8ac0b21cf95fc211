// Host-side launch interface of the traversal kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "bvh8.cuh"

namespace ilg {

struct SceneView {
    const Node8 *nodes;
    const Tri *tris;
    const uint32_t *prim_of;
    uint32_t n_nodes, n_tris;
};

cudaError_t launch_closest(const SceneView &s, const float4 *ro, const float4 *rd, uint32_t n, int32_t *prim,
                           float *t, float *u, float *v, uint32_t *err, unsigned long long *stats, cudaStream_t st);
cudaError_t launch_any(const SceneView &s, const float4 *ro, const float4 *rd, uint32_t n, uint8_t *occ,
                       uint32_t *err, cudaStream_t st);

// Queries that ignore the input triangles [skip_lo, skip_lo + skip_n).
cudaError_t launch_closest_skip(const SceneView &s, const float4 *ro, const float4 *rd, uint32_t n,
                                uint32_t skip_lo, uint32_t skip_n, int32_t *prim, float *t, float *u, float *v,
                                uint32_t *err, cudaStream_t st);
cudaError_t launch_any_skip(const SceneView &s, const float4 *ro, const float4 *rd, uint32_t n, uint32_t skip_lo,
                            uint32_t skip_n, uint8_t *occ, uint32_t *err, cudaStream_t st);

// Watertight test (persistent kernels); raw = three float4 vertices per
// triangle record, made by build_raw_tris from the input mesh.
cudaError_t launch_closest_wt(const SceneView &s, const float4 *raw, const float4 *ro, const float4 *rd, uint32_t n,
                              int32_t *prim, float *t, float *u, float *v, uint32_t *next, uint32_t *err,
                              cudaStream_t st);
cudaError_t launch_any_wt(const SceneView &s, const float4 *raw, const float4 *ro, const float4 *rd, uint32_t n,
                          uint8_t *occ, uint32_t *next, uint32_t *err, cudaStream_t st);
cudaError_t build_raw_tris(const uint32_t *prim_of, const uint32_t *idx, const float *pos, uint32_t n, float4 *raw,
                           cudaStream_t st);

// Loads the code of the closest-hit persistent kernel on the current device
// (kernels load lazily on first launch otherwise, which may allocate).
cudaError_t preload_closest_dyn();

// Persistent variants with dynamic ray fetch; `next` is a device counter word.
cudaError_t launch_closest_dyn(const SceneView &s, const float4 *ro, const float4 *rd, uint32_t n, int32_t *prim,
                               float *t, float *u, float *v, uint32_t *next, uint32_t *err, cudaStream_t st);
cudaError_t launch_any_dyn(const SceneView &s, const float4 *ro, const float4 *rd, uint32_t n, uint8_t *occ,
                           uint32_t *next, uint32_t *err, cudaStream_t st);

}  // namespace ilg
