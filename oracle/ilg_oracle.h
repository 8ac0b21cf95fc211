/* CPU oracle for the closest-hit / any-hit path - TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's ray/mesh query. Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the
 * product path never does.
 *
 * Follows, operation for operation:
 *   IndexedTriangle::Intersects (Shirley form)  Core/Shape/IndexedTriangle.cpp:92-128
 *     edges precomputed as v1-v0, v2-v0          Core/Shape/IndexedTriangle.cpp:44-45
 *     reject t > Max - 1e-5 || t < 1e-5 (double) Core/Shape/IndexedTriangle.cpp:115
 *   closest hit shrinks ray.Max to the hit t     Core/Shape/BVHMesh.cpp:186-190
 *   any hit returns on the first accepted test   Core/Shape/BVHMesh.cpp:143-165
 *   slab test rejects tmin > Max, tmax < Min     Core/Geometry/BoundingBox.cpp:215-238
 * The binary BVH here is our own (median split); like the reference's
 * KD-tree and BVH it changes only which of two hits closer than 1e-5 wins.
 */
#ifndef ILG_ORACLE_H
#define ILG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One Shirley test with ray.Max = tmax; returns 1 on accept. */
int orc_shirley(const float *pos, const uint32_t *idx, uint32_t tri,
                const float o[3], const float d[3], float tmax,
                float *t, float *beta, float *gamma);

/* Closest hit over all triangles in index order (the reference's linear
 * BasicSpace loop over a mesh of one-triangle primitives). */
void orc_intersect_brute(const float *pos, const uint32_t *idx, uint32_t ntris,
                         const float *o4, const float *d4, int64_t n,
                         int32_t *prim, float *t, float *u, float *v);

/* Closest hit (and any hit into occ, when not NULL) with the watertight test
 * of Woop, Benthin and Wald 2013 - the restatement behind the device's
 * ILG_WATERTIGHT mode, not a reference function. */
void orc_watertight_brute(const float *pos, const uint32_t *idx, uint32_t ntris, const float *o4, const float *d4,
                          int64_t n, int32_t *prim, float *t, float *u, float *v, uint8_t *occ);

void *orc_bvh_create(const float *pos, uint32_t nverts, const uint32_t *idx, uint32_t ntris);
void orc_bvh_destroy(void *h);
/* stats (optional, 2 x uint64): total node visits, total triangle tests. */
void orc_bvh_intersect(void *h, const float *o4, const float *d4, int64_t n,
                       int32_t *prim, float *t, float *u, float *v,
                       int nthreads, uint64_t *stats);
void orc_bvh_occluded(void *h, const float *o4, const float *d4, int64_t n,
                      uint8_t *occ, int nthreads);

/* Single-ray queries on an oracle BVH (triangle index or -1; t on a hit). */
int32_t orc_bvh_closest1(void *h, const float o[3], const float d[3], float rmin, float rmax, float *t);
int orc_bvh_any1(void *h, const float o[3], const float d[3], float rmin, float rmax);

/* Path tracing restatement (pt_oracle.c). Layouts match the device's
 * ilg_material / ilg_quad_light. cam = eye[3], target[3], up[3], fov, aspect.
 * out: H x W x 3 floats. */
typedef struct { float albedo[3]; uint32_t kind; float f0[3]; float alpha; } orc_material;
typedef struct { float v[4][3]; float emit[3]; uint32_t first_tri; } orc_quad_light;
int orc_render(const float *pos, uint32_t nverts, const uint32_t *idx, uint32_t ntris, const uint32_t *mat_ids,
               const orc_material *mats, uint32_t nmats, const orc_quad_light *lights, uint32_t nlights,
               const float cam[11], uint32_t W, uint32_t H, uint32_t spp, uint32_t max_depth, float eps,
               uint32_t seed, const float sky[3], int nthreads, float *out);

#ifdef __cplusplus
}
#endif
#endif
