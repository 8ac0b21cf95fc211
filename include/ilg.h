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

/* Only the ilg_* entry points are exported from libilg.so. */
#if defined(__GNUC__)
#define ILG_API __attribute__((visibility("default")))
#else
#define ILG_API
#endif

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
/* ilg_intersect / ilg_occluded: the watertight triangle test (Woop, Benthin
 * and Wald 2013) instead of the reference's Shirley test. A ray through an
 * edge or vertex shared by two triangles hits one of them, where the
 * reference's test can let it through ("edge cracks"); elsewhere the hit is
 * the reference's up to float rounding of t, beta and gamma. Same rejection
 * window (t < 1e-5 or t > Max - 1e-5). */
#define ILG_WATERTIGHT 0x2u

typedef struct ilg_ctx ilg_ctx;

typedef struct ilg_opts {
    int32_t device;      /* CUDA device ordinal */
    uint32_t build_flags; /* ILG_BUILD_* for every ilg_build of the context (0: the default build) */
    uint32_t reserved[6];
} ilg_opts;

/* ilg_opts.build_flags. By default ilg_build restructures the Morton tree by
 * treelets for least SAH cost (two passes; about 12 ms at 1 M triangles and
 * 0.1-0.4 s at 21 M on a B200, for 15-25 % faster traversal); ILG_BUILD_FAST
 * skips that step (about 9 / 19 ms), for scenes rebuilt often. Both trees
 * give the same hits, up to which of two hits less than 1e-5 apart wins. */
#define ILG_BUILD_FAST 0x1u

typedef struct ilg_stats {
    uint32_t n_tris;        /* triangles in the built scene */
    uint32_t n_nodes;       /* 8-wide BVH nodes */
    uint32_t n_leaf_tris;   /* triangle records (== n_tris) */
    uint32_t max_depth;     /* deepest 8-wide level */
    float build_ms;         /* device time of the last ilg_build */
    uint64_t node_bytes;    /* bytes of node records */
    uint64_t tri_bytes;     /* bytes of triangle records */
} ilg_stats;

ILG_API int ilg_create(ilg_ctx **out, const ilg_opts *opts);
ILG_API int ilg_destroy(ilg_ctx *ctx);
ILG_API const char *ilg_last_error(const ilg_ctx *ctx);

/* Positions are n_verts x 3 floats (world space), indices n_tris x 3.
 * mat_ids (optional, n_tris) tags each triangle with a material slot. */
ILG_API int ilg_set_mesh(ilg_ctx *ctx, const float *pos_xyz, uint32_t n_verts,
                 const uint32_t *idx, uint32_t n_tris, const uint32_t *mat_ids);
ILG_API int ilg_build(ilg_ctx *ctx);
ILG_API int ilg_get_stats(const ilg_ctx *ctx, ilg_stats *out);

/* Persistent scenes (this project's format; the reference's counterpart is
 * its memory-mapped PersistentMesh, Core/Shape/PersistentMesh.h:22-35): the
 * uploaded mesh and the built BVH written to / read from one checksummed
 * file. ilg_load leaves the context as ilg_set_mesh + ilg_build would, with
 * the same records, without building; malformed or corrupted files are
 * ILG_EINVAL. */
ILG_API int ilg_save(ilg_ctx *ctx, const char *path);
ILG_API int ilg_load(ilg_ctx *ctx, const char *path);

/* Closest hit. Rays: ray_o_tmin = N x (ox, oy, oz, tmin), ray_d_tmax =
 * N x (dx, dy, dz, tmax), both float4-aligned. Hits: prim[i] = triangle index
 * (-1 on a miss), t[i] (+inf on a miss), u[i] = beta, v[i] = gamma, in the
 * reference's Shirley arithmetic and rejection window. */
ILG_API int ilg_intersect(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n,
                  int32_t *prim, float *t, float *u, float *v, uint32_t flags);

/* ilg_intersect plus work counters: counts[0] = node records read,
 * counts[1] = triangle records tested, summed over the batch (the per-query
 * work behind the reference's tree statistics, TreeMeshStatistics,
 * Core/Shape/TreeMesh.cpp:11-29). Synchronous; used to state algorithmic
 * bytes per ray. */
ILG_API int ilg_intersect_counted(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n,
                          int32_t *prim, float *t, float *u, float *v, uint64_t counts[2], uint32_t flags);

/* Closest hit from host buffers that allocates no device memory. This entry
 * point has no counterpart in the reference. It is for callers that must not
 * trigger a cudaMalloc at query time (a fixed per-frame device budget, or
 * device memory owned by another allocator): it stages rays and hits through
 * one fixed device array per GPU (12 MiB, resident until exit) instead of the
 * context's growable buffers. At most ILG_NOALLOC_MAX_RAYS rays per call
 * (more is ILG_EINVAL). All calls on a device share that array, so calls whose
 * device work overlaps race; serialise them. The array becomes resident, and
 * its device address is looked up (cudaGetSymbolAddress), when a context is
 * created on the device (ilg_create), so a call itself only copies, clears
 * two words of the array and launches one kernel. The status covers this call
 * only: its device error flags are kept in the array, not in the context.
 * Results equal ilg_intersect's. */
#define ILG_NOALLOC_MAX_RAYS 262144u
ILG_API int ilg_intersect_noalloc(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n,
                          int32_t *prim, float *t, float *u, float *v);

/* Any hit: occ[i] = 1 when some triangle is hit inside the ray's window. */
ILG_API int ilg_occluded(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n,
                 uint8_t *occ, uint32_t flags);

/* Closest hit / any hit that ignore the input triangles [skip_first,
 * skip_first + skip_count): the reference's `p_pExclude` overloads,
 * ISpace::Intersects(const Ray&, Intersection&, IPrimitive*) and
 * ISpace::Intersects(const Ray&, IPrimitive*) (Core/Space/Space.h:39,41,
 * BasicSpace.cpp:75-91,104-115), once a primitive's triangles occupy one
 * contiguous range of the mesh given to ilg_set_mesh. Same arguments and
 * results as ilg_intersect / ilg_occluded otherwise. */
ILG_API int ilg_intersect_excluding(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n,
                            uint32_t skip_first, uint32_t skip_count, int32_t *prim, float *t, float *u,
                            float *v, uint32_t flags);
ILG_API int ilg_occluded_excluding(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n,
                           uint32_t skip_first, uint32_t skip_count, uint8_t *occ, uint32_t flags);

/* ------------------------------------------------------------------------
 * Path tracing (the reference's PathIntegrator::Radiance bounce loop,
 * Core/Integrator/PathIntegrator.cpp:44-367, driven per pixel as
 * BaseRenderer::RenderRegion does, Core/Renderer/BaseRenderer.cpp:62-169).
 * ---------------------------------------------------------------------- */

#define ILG_MAT_LAMBERT 0u /* MatteMaterial: Lambertian BxDF (Core/Material/Matte.h) */
#define ILG_MAT_GGX 1u     /* GGX conductor (no reference counterpart) */
#define ILG_MAT_MIRROR 2u  /* MirrorMaterial: SpecularReflection (Core/Material/Mirror.h) */
#define ILG_MAT_GLASS 3u   /* GlassMaterial: SpecularTransmission + SpecularReflection, picked with
                            * equal probability, no Fresnel weight (Core/Material/Glass.h) */

typedef struct ilg_material {
    float albedo[3];  /* Lambertian reflectance; mirror and glass: reflectivity */
    uint32_t kind;    /* ILG_MAT_* */
    float f0[3];      /* GGX: Schlick reflectance at normal incidence; glass: transmittance */
    float alpha;      /* GGX: roughness (alpha); glass: eta_i / eta_t (1 / 1.52 by default) */
} ilg_material;

/* A one-sided area light on a Quad (DiffuseAreaLight over Core/Shape/Quad.cpp).
 * v holds the reference's Quad vertices in its order; the quad's two
 * triangles must be in the mesh at first_tri and first_tri + 1 as
 * (v[0], v[2], v[1]) and (v[0], v[3], v[2]), which is how the reference
 * tessellates a Quad. */
typedef struct ilg_quad_light {
    float v[4][3];
    float emit[3];
    uint32_t first_tri;
} ilg_quad_light;

/* Lights of every kind the device path tracer samples (ilg_set_lights):
 *   ILG_LIGHT_QUAD      DiffuseAreaLight on a Quad, as ilg_quad_light
 *                       (Core/Light/DiffuseAreaLight.cpp, Core/Shape/Quad.cpp)
 *   ILG_LIGHT_MESH      DiffuseAreaLight on a triangle mesh whose triangles
 *                       are [first_tri, first_tri + tri_count) of the mesh
 *                       given to ilg_set_mesh: one-sided emission seen by the
 *                       path, light samples as the reference takes them
 *                       (ITriangleMesh::SamplePoint, TriangleMesh.cpp:142-161:
 *                       a triangle uniform by index, a uniform point on it,
 *                       its normal turned toward the shaded point, pdf 1 / the
 *                       mesh's area)
 *   ILG_LIGHT_INFINITE  InfiniteAreaLight without a texture, with the
 *                       reference's semantics (InfiniteAreaLight.cpp:39-90):
 *                       a camera ray that escapes, or a path escaping right
 *                       after a specular bounce, sees radiance 1 whatever the
 *                       intensity; its light samples take a direction in the
 *                       cone cos(theta) >= 1e-4 about the normal and add
 *                       intensity * cos * BSDF, not divided by their pdf.
 * Set the lights after the mesh: a mesh light's area is computed from the
 * mesh uploaded at the time. */
#define ILG_LIGHT_QUAD 0u
#define ILG_LIGHT_MESH 1u
#define ILG_LIGHT_INFINITE 2u
typedef struct ilg_light {
    uint32_t kind;       /* ILG_LIGHT_* */
    float emit[3];       /* quad, mesh: emitted radiance; infinite: intensity */
    float v[4][3];       /* quad: its vertices, as ilg_quad_light::v */
    uint32_t first_tri;  /* quad, mesh: first of its triangles in the mesh */
    uint32_t tri_count;  /* mesh: its number of triangles (quad: 2; infinite: unused) */
} ilg_light;

/* Pinhole camera as the reference's camera factory builds it
 * (Core/Camera/CameraFactories.h:40-80): frame from (target - eye, up),
 * image plane at distance 1, SetFieldOfView(fov_deg, aspect). */
typedef struct ilg_camera {
    float eye[3];
    float target[3];
    float up[3];
    float fov_deg;
    float aspect;
} ilg_camera;

typedef struct ilg_render_opts {
    uint32_t width, height;
    uint32_t spp;            /* samples per pixel */
    uint32_t max_depth;      /* RayDepth (factory default 6) */
    float epsilon;           /* reflect epsilon (factory default 1e-4) */
    uint32_t seed;           /* sample-sequence seed */
    uint32_t paths_per_wave; /* wavefront size; 0 = automatic */
    float sky[3];            /* constant environment radiance; 0 = none */
    /* radiance cache (needs ilg_mlp_init): 0 = plain path tracing; k >= 1 =
     * rendering paths stop into the cache at their k-th bounce vertex, one
     * path in train_every is traced to full depth and its vertices train the
     * cache after the call (train_steps Adam steps of train_batch records) */
    uint32_t cache_depth;
    uint32_t train_every;    /* 0 = 16 */
    uint32_t train_steps;    /* Adam steps after the call; 0 = none (the cache stays frozen) */
    uint32_t train_batch;    /* 0 = 16384 */
    /* 0 = training paths are traced to max_depth; k >= 1 = they stop into
     * the cache at vertex cache_depth + k, and the cache's answer there
     * completes their targets (self-training; the frame then ends at that
     * depth) */
    uint32_t train_tail;
    /* passes over the call's training records (0 = 1): each pass runs the
     * same train_steps Adam steps on the same records again */
    uint32_t train_epochs;
} ilg_render_opts;

/* Materials indexed by the mat_ids given to ilg_set_mesh. */
ILG_API int ilg_set_materials(ilg_ctx *ctx, const ilg_material *mats, uint32_t n);
ILG_API int ilg_set_quad_lights(ilg_ctx *ctx, const ilg_quad_light *lights, uint32_t n);
/* At most 8 lights of any kinds (replaces the lights set before); the
 * scene's LightList (Core/Scene/Scene.h) in the order the reference samples it. */
ILG_API int ilg_set_lights(ilg_ctx *ctx, const ilg_light *lights, uint32_t n);

/* Renders width x height pixels at spp samples each into out_rgb
 * (height x width x 3 floats, row y = image-plane 'up' coordinate y, as the
 * reference's RenderRegion indexes its buffer). Host pointer unless
 * ILG_DEVICE_PTRS. Needs ilg_build, ilg_set_mesh with mat_ids, and
 * ilg_set_materials. */
ILG_API int ilg_render(ilg_ctx *ctx, const ilg_camera *cam, const ilg_render_opts *opts, float *out_rgb,
               uint32_t flags);

/* ilg_render flag: count the traversal work of the render (slower kernels)
 * for ilg_render_counts: counts = {closest-hit rays, node records they read,
 * triangle records they tested, shadow rays, node records, triangle records}.
 * These are the per-sample bytes of the path tracer's memory roofline. */
#define ILG_RENDER_COUNT 0x4u
/* ilg_render / ilg_render_batch flag: the whole render as one persistent
 * kernel launch instead of the wavefront's launches per bounce. Each GPU
 * thread carries one path through all its bounces (closest hit, shading, a
 * shadow ray per light, the next ray) and takes a new path, of any scene of
 * a batch, when its path ends. Same paths as the wavefront (same sample
 * sequence and arithmetic): the images agree up to float summation order.
 * Plain renders only (no cache options, ILG_RENDER_COUNT, or Direct /
 * Albedo outputs). */
#define ILG_RENDER_PERSISTENT 0x20u
ILG_API int ilg_render_counts(ilg_ctx *ctx, uint64_t counts[6]);

/* ilg_render / ilg_render_region flag: with cache_depth set, a hash-grid
 * radiance cache answers the cache queries instead of the network: a cell
 * per voxel of the scene's box (256 per axis) x normal direction (6) x
 * octant of the outgoing direction (8) holds the running mean of the
 * training records that fell in it (4 M cells, 80 MB, open addressing); a
 * query that finds no filled cell answers 0. It is the non-learned baseline
 * the network is measured against (the reference's own cache, the
 * irradiance cache of Core/Integrator/ICIntegrator.*, inserts its records
 * one query at a time). train_steps / train_batch / train_epochs do not
 * apply; call ilg_hash_cache_reset first. */
#define ILG_RENDER_HASH_CACHE 0x8u
ILG_API int ilg_hash_cache_reset(ilg_ctx *ctx);

/* Training records of the last cached render (ILG_RENDER_* with
 * cache_depth): *records = records its training paths produced; *dropped =
 * those the hash-grid cache could not store because all 8 cells of their
 * probe window held other keys (0 unless the render used
 * ILG_RENDER_HASH_CACHE). Synchronises the context's stream. This project's
 * own statistics; no counterpart in the reference. */
ILG_API int ilg_last_train_stats(ilg_ctx *ctx, uint32_t *records, uint32_t *dropped);

/* A camera as the reference's ICamera holds it after construction
 * (Core/Camera/Camera.h:23-28: m_centre, m_corner, m_across, m_up): the ray
 * through normalised image point (px, py) is normalize(corner + across * px
 * + up * py - centre) (PerspectiveCamera::GetRay, PerspectiveCamera.cpp:44-60). */
typedef struct ilg_camera_frame {
    float centre[3];
    float corner[3];
    float across[3];
    float up[3];
} ilg_camera_frame;

/* The frame PerspectiveCamera(eye, normalize(target - eye), up, -1, 1, -1, 1, 1)
 * + SetFieldOfView(fov_deg, aspect) builds (Core/Camera/Camera.cpp:30-44). */
ILG_API int ilg_camera_frame_of(const ilg_camera *cam, ilg_camera_frame *out);

/* Pixels [x, x + width) x [y, y + height) of the opts->width x opts->height image. */
typedef struct ilg_region {
    uint32_t x, y, width, height;
} ilg_region;

/* IRenderer::RenderRegion(buffer, x, y, w, h) with a PathIntegrator
 * (BaseRenderer.cpp:62-169): renders one region of the image, each pixel
 * with exactly the paths a whole-image render gives it (same seed), so
 * regions tile the image seamlessly. Outputs are region-sized (region height
 * x width x 3): final_rgb = RadianceContext::Final; direct_rgb (optional) =
 * RadianceContext::Direct, what the first vertex adds (emission seen
 * directly and its light samples; Indirect = Final - Direct); albedo_rgb
 * (optional) = RadianceContext::Albedo, the first hit's reflectance. All are
 * per-sample averages. Host pointers unless ILG_DEVICE_PTRS. The radiance
 * cache options of opts work as in ilg_render: the region's paths query the
 * cache, its training paths train it after the call (with train_steps 0 a
 * frozen cache, and regions still tile the image exactly); Direct and Albedo
 * come from the first vertex, before any cache query. */
ILG_API int ilg_render_region(ilg_ctx *ctx, const ilg_camera_frame *frame, const ilg_render_opts *opts,
                      const ilg_region *region, float *final_rgb, float *direct_rgb, float *albedo_rgb,
                      uint32_t flags);

/* IIntegrator::Radiance(context, scene, ray, intersection, radiance_context)
 * of the reference's PathIntegrator (Core/Integrator/Integrator.h:53-54,
 * PathIntegrator.cpp:44-367), batched over n caller-given rays: ray i
 * (float4 (o, Min) and (d, Max), 16-byte aligned; its first intersection
 * uses its own [Min, Max]) starts opts->spp paths through the device bounce
 * loop, and final_rgb / direct_rgb / albedo_rgb (n x 3 each; the last two
 * optional) receive their averages of Direct + Indirect, Direct and Albedo,
 * as the reference's RadianceContext holds them. opts->width and
 * opts->height are ignored; max_depth, epsilon, seed, sky and the cache
 * options mean what they mean for ilg_render. Host pointers unless
 * ILG_DEVICE_PTRS (then the ray and output arrays are device pointers and
 * the call only enqueues). */
ILG_API int ilg_radiance(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n,
                 const ilg_render_opts *opts, float *final_rgb, float *direct_rgb, float *albedo_rgb,
                 uint32_t flags);

/* ------------------------------------------------------------------------
 * Radiance-cache network (no counterpart in the reference, whose closest
 * analogue is the irradiance cache of Core/Integrator/ICIntegrator.*): a
 * 96 -> 64 x 5 (ReLU) -> 3 MLP, BF16 weights and activations, FP32
 * accumulation on the tensor cores, trained with Adam on a relative L2 loss.
 * Queries are ILG_MLP_RAW floats per row: position normalised to [0,1]^3,
 * outgoing direction, normal, roughness, albedo, 3 unused. The position is
 * encoded on the device by a trainable multiresolution hash grid (16 levels
 * of 2 features, 2^15 entries a level, resolutions floor(16 * 2^(7 l / 15))
 * per unit; Mueller et al. 2022) and by 4 sine/cosine frequency bands per
 * axis.
 * ---------------------------------------------------------------------- */
#define ILG_MLP_RAW 16u
#define ILG_MLP_PARAMS 23040u /* FP32 weights, per layer row-major [in][out] */
#define ILG_MLP_GRID_PARAMS 1048576u /* FP32 grid features [level][entry][feature] */

ILG_API int ilg_mlp_init(ilg_ctx *ctx, uint32_t seed, float learning_rate);
/* ilg_mlp_init with a choice of input encoding: ILG_MLP_ENC_HASHGRID (the
 * encoding above, ilg_mlp_init's) or ILG_MLP_ENC_FREQ12: 12 sine/cosine
 * frequency bands per position axis (sin and cos of 2^b pi x, b < 12) next
 * to the raw outgoing direction, normal, roughness and albedo and a
 * constant 1 (84 of the 96 input columns; no grid is read or trained). */
#define ILG_MLP_ENC_HASHGRID 0u
#define ILG_MLP_ENC_FREQ12 1u
ILG_API int ilg_mlp_init_encoding(ilg_ctx *ctx, uint32_t seed, float learning_rate, uint32_t encoding);
ILG_API int ilg_mlp_get_params(ilg_ctx *ctx, float *params /* ILG_MLP_PARAMS */);
ILG_API int ilg_mlp_set_params(ilg_ctx *ctx, const float *params);
ILG_API int ilg_mlp_get_grid(ilg_ctx *ctx, float *grid /* ILG_MLP_GRID_PARAMS */);
ILG_API int ilg_mlp_set_grid(ilg_ctx *ctx, const float *grid);
/* The grid part of the gradient the last ilg_mlp_grads computed. */
ILG_API int ilg_mlp_get_grid_grads(ilg_ctx *ctx, float *grad /* ILG_MLP_GRID_PARAMS */);
/* out: n x 3 radiance. Host pointers unless ILG_DEVICE_PTRS (device query
 * rows must start 16-byte aligned). Runs on the
 * tcgen05 tensor cores (accumulators in TMEM); ILG_MLP_WARP_MMA selects the
 * warp-level mma.sync kernel that training's forward pass uses instead. */
#define ILG_MLP_WARP_MMA 0x10u
ILG_API int ilg_mlp_infer(ilg_ctx *ctx, const float *raw, uint32_t n, float *out, uint32_t flags);
/* Gradient of the mean relative L2 loss over the batch (no update). Runs on
 * the tcgen05 tensor cores (forward, loss and backward in one kernel, the
 * weight gradients in another, accumulators in TMEM; device rows 16-byte
 * aligned); with ILG_MLP_WARP_MMA on the warp-level mma.sync kernels. */
ILG_API int ilg_mlp_grads(ilg_ctx *ctx, const float *raw, const float *target, uint32_t n, float *grad /* ILG_MLP_PARAMS */,
                  float *loss, uint32_t flags);
/* One Adam step on the batch; *loss (optional) receives the loss before the step. */
ILG_API int ilg_mlp_train_step(ilg_ctx *ctx, const float *raw, const float *target, uint32_t n, float *loss, uint32_t flags);

/* Many independent scenes rendered together: one wavefront over the paths of
 * every item (a scene context with its built mesh, materials and lights, a
 * camera, image size, spp and depth), so scenes of very different sizes and
 * path lengths share the queues. The runner context supplies the wavefront
 * buffers and the stream; all contexts must be on its device.
 * paths_per_wave: 0 = automatic; block: threads per block of the extend,
 * shade and shadow kernels (64, 128 or 256; 0 = 128). flags: ILG_DEVICE_PTRS,
 * ILG_RENDER_COUNT (the batch's traversal work for ilg_render_counts on the
 * runner). */
typedef struct ilg_batch_item {
    ilg_ctx *scene;
    ilg_camera camera;
    uint32_t width, height, spp, max_depth;
    float epsilon;
    uint32_t seed;
    float sky[3];
    float *out_rgb; /* height x width x 3 */
} ilg_batch_item;

ILG_API int ilg_render_batch(ilg_ctx *runner, const ilg_batch_item *items, uint32_t n, uint32_t paths_per_wave,
                     uint32_t block, uint32_t flags);

/* ------------------------------------------------------------------------
 * Post-processing on the device, so a progressive renderer copies only the
 * displayed image back. Images are n_pixels x 3 floats; host pointers unless
 * ILG_DEVICE_PTRS (then both are device pointers and the call only enqueues).
 * ---------------------------------------------------------------------- */
/* AccumulationBuffer::Apply (Core/Postproc/AccumulationBuffer.h:59-87): the
 * context's running sum gets frame_rgb added (sum = frame + sum) and out_rgb
 * = sum * (1 / frames so far), bit for bit the reference's arithmetic. A new
 * image size, or ilg_accumulate_reset (AccumulationBuffer::Reset), starts
 * over. */
ILG_API int ilg_accumulate(ilg_ctx *ctx, const float *frame_rgb, uint32_t n_pixels, float *out_rgb, uint32_t flags);
ILG_API int ilg_accumulate_reset(ilg_ctx *ctx);

#define ILG_TONE_GLOBAL 0u /* GlobalTone (Core/Postproc/GlobalTone.h): c / (c + 1) */
#define ILG_TONE_AUTO 1u   /* AutoTone (AutoTone.h): (c - min) / (max - min), clamped to [0, 1] */
#define ILG_TONE_DRAGO 2u  /* DragoTone (DragoTone.h): Drago et al. 2003, bias 0.8, scale 0.95 */
/* Tone mapping of a whole image. GLOBAL and AUTO are bit for bit the
 * reference's; DRAGO evaluates its logarithms and power in double as the
 * reference does and agrees to within float rounding. */
ILG_API int ilg_tonemap(ilg_ctx *ctx, const float *in_rgb, uint32_t n_pixels, float *out_rgb, uint32_t op, uint32_t flags);

/* Device probe (this project's measurement tool; no counterpart in the
 * reference): *gbs = bytes read per second by a streaming read kernel that
 * passes `reps` times over a device buffer of `bytes` bytes (1 MiB .. 8 GiB),
 * with L2-only loads. A buffer below the device's L2 size gives the L2 read
 * bandwidth, the roofline denominator of traversal over scenes that fit in
 * L2. Allocates and frees its buffer; synchronous. */
ILG_API int ilg_probe_read_gbs(ilg_ctx *ctx, uint64_t bytes, uint32_t reps, float *gbs);

/* Blocks until the context's stream is idle (for ILG_DEVICE_PTRS callers). */
ILG_API int ilg_sync(ilg_ctx *ctx);

/* The context's CUDA stream (a cudaStream_t), for callers that time or order
 * their own work against it. */
ILG_API void *ilg_stream(ilg_ctx *ctx);

#ifdef __cplusplus
}
#endif

#endif /* ILG_H */
