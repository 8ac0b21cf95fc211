/*
 * ilg.h - C ABI of the B200 ray/scene query and path-tracing library.
 *
 * Plain pointers and sizes only. Every call returns an ilg_status; the text
 * of the last failure is available from ilg_last_error(). A context owns one
 * CUDA stream and its device buffers and must be used from one host thread
 * at a time; distinct contexts are independent.
 *
 * Host input pointers are borrowed for the duration of a call. With
 * ILG_DEVICE_PTRS the ray and hit arrays are device pointers instead (the call
 * then enqueues on the context's stream and returns without a host copy).
 *
 * What each entry point replaces in the reference (keithbugeja/illuminaPRT):
 *   ilg_set_mesh + ilg_build   ISpace::Initialise/Build over the PrimitiveList
 *                              (Core/Space/Space.h:33-36, BasicSpace.cpp:16-48)
 *                              and the per-mesh tree build it hands to shapes,
 *                              ITriangleMesh::Compile (KDTreeMesh.cpp:114-275,
 *                              BVHMesh.cpp:78-107)
 *   ilg_intersect              ISpace::Intersects(const Ray&, Intersection&)
 *                              (Core/Space/Space.h:40, BasicSpace.cpp:58-73),
 *                              batched over N rays
 *   ilg_occluded               ISpace::Intersects(const Ray&)
 *                              (Core/Space/Space.h:42, BasicSpace.cpp:94-103),
 *                              batched over N rays
 */
#ifndef ILG_H
#define ILG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ilg_status {
    ILG_OK = 0,
    ILG_EINVAL = 1,    /* bad argument (null pointer, size out of range, bad flag) */
    ILG_ENOMEM = 2,    /* device or host allocation failed */
    ILG_ECUDA = 3,     /* a CUDA runtime call failed */
    ILG_ETIMEOUT = 4,  /* a bounded device wait ran out */
    ILG_EOVERFLOW = 5, /* a device queue or traversal stack bound was exceeded */
    ILG_ESTATE = 6     /* call out of order (e.g. intersect before build) */
} ilg_status;

/* ilg_intersect / ilg_occluded flags */
#define ILG_DEVICE_PTRS 0x1u /* ray and hit arrays are device pointers */

typedef struct ilg_ctx ilg_ctx;

typedef struct ilg_opts {
    int32_t device;      /* CUDA device ordinal */
    uint32_t reserved[7];
} ilg_opts;

typedef struct ilg_stats {
    uint32_t n_tris;        /* triangles in the built scene */
    uint32_t n_nodes;       /* 8-wide BVH nodes */
    uint32_t n_leaf_tris;   /* triangle records (== n_tris) */
    uint32_t max_depth;     /* deepest 8-wide level */
    float build_ms;         /* device time of the last ilg_build */
    uint64_t node_bytes;    /* bytes of node records */
    uint64_t tri_bytes;     /* bytes of triangle records */
} ilg_stats;

int ilg_create(ilg_ctx **out, const ilg_opts *opts);
int ilg_destroy(ilg_ctx *ctx);
const char *ilg_last_error(const ilg_ctx *ctx);

/* Positions are n_verts x 3 floats (world space), indices n_tris x 3.
 * mat_ids (optional, n_tris) tags each triangle with a material slot. */
int ilg_set_mesh(ilg_ctx *ctx, const float *pos_xyz, uint32_t n_verts,
                 const uint32_t *idx, uint32_t n_tris, const uint32_t *mat_ids);
int ilg_build(ilg_ctx *ctx);
int ilg_get_stats(const ilg_ctx *ctx, ilg_stats *out);

/* Closest hit. Rays: ray_o_tmin = N x (ox, oy, oz, tmin), ray_d_tmax =
 * N x (dx, dy, dz, tmax), both float4-aligned. Hits: prim[i] = triangle index
 * (-1 on a miss), t[i] (+inf on a miss), u[i] = beta, v[i] = gamma, in the
 * reference's Shirley arithmetic and rejection window. */
int ilg_intersect(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n,
                  int32_t *prim, float *t, float *u, float *v, uint32_t flags);

/* ilg_intersect plus work counters: counts[0] = node records read,
 * counts[1] = triangle records tested, summed over the batch (the per-query
 * work behind the reference's tree statistics, TreeMeshStatistics,
 * Core/Shape/TreeMesh.cpp:11-29). Synchronous; used to state algorithmic
 * bytes per ray. */
int ilg_intersect_counted(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n,
                          int32_t *prim, float *t, float *u, float *v, uint64_t counts[2], uint32_t flags);

/* Any hit: occ[i] = 1 when some triangle is hit inside the ray's window. */
int ilg_occluded(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n,
                 uint8_t *occ, uint32_t flags);

/* Blocks until the context's stream is idle (for ILG_DEVICE_PTRS callers). */
int ilg_sync(ilg_ctx *ctx);

/* The context's CUDA stream (a cudaStream_t), for callers that time or order
 * their own work against it. */
void *ilg_stream(ilg_ctx *ctx);

#ifdef __cplusplus
}
#endif

#endif /* ILG_H */
