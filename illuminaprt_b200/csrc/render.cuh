// Device state of the wavefront path tracer (render.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "bvh8.cuh"

namespace ilg {

constexpr uint32_t kMaxLights = 8;

struct Mat {  // mirrors ilg_material (32 bytes)
    float3 albedo;
    uint32_t kind;
    float3 f0;
    float alpha;
};
static_assert(sizeof(Mat) == 32, "material record is 32 bytes");

// Light kinds (ilg_light::kind)
constexpr uint32_t kLightQuad = 0, kLightMesh = 1, kLightInfinite = 2;

struct Light {
    float3 p[4];   // quad: the reference's Quad vertices v1..v4
    float3 emit;   // quad, mesh: emitted radiance; infinite: intensity (scales its light samples only)
    float3 n;      // quad: unit normal (v3 - v1) x (v2 - v1), as Quad::SamplePoint returns it, normalised
    float area;    // quad: area of the two tessellation triangles; mesh: summed area of its triangles
    uint32_t kind;
    uint32_t first_tri, tri_count;  // quad, mesh: its triangles in the uploaded mesh
};

// One scene of a (batched) render: its BVH, shading data, camera and where
// its paths and pixels sit in the wave's global index spaces.
struct SceneRec {
    const Node8 *nodes;
    const Tri *tris;
    uint32_t n_nodes, n_tris;
    const uint32_t *tri_attr;  // per triangle record: material (low 16) | light (high 16, 0xffff none)
    const Mat *mats;
    uint32_t n_mats;
    const Light *lights;
    uint32_t n_lights;
    float3 sky;
    // what an escaping path sees of the scene's infinite lights at depth 0 or
    // after a specular bounce: 1 per light (InfiniteAreaLight::Radiance
    // ignores its intensity, Core/Light/InfiniteAreaLight.cpp:39-56)
    float inf_escape;
    // the uploaded mesh (mesh lights sample points on its triangles)
    const float *pos;
    const uint32_t *idx;
    // rays given by the caller (ilg_radiance): pixel i of the region starts
    // its paths with ray i instead of a camera ray; null for camera paths
    const float4 *ray_o, *ray_d;
    // camera (PerspectiveCamera after SetFieldOfView)
    float3 centre, corner, across, up;
    uint32_t width, height;  // the whole image (the camera's normalisation)
    uint32_t wh;             // pixels rendered: the region's
    uint32_t region_x, region_y, region_w;  // the rendered region of the image
    uint32_t full_wh;        // width * height: the sample-sequence stride
    float rcp_w, rcp_h;
    uint32_t max_depth;
    float eps;
    uint32_t spp;
    uint32_t seed;
    uint64_t path_begin;   // first global path index (paths are sample-major: sample * wh + pixel)
    uint32_t pixel_base;   // first pixel of this scene in the accumulation buffer
};

// Everything the kernels of one render need, passed by value.
struct RenderDev {
    const SceneRec *scenes;
    uint32_t n_scenes;
    uint32_t depth_max;    // largest max_depth over the scenes
    uint32_t *path_scene;  // per path of the wave: its scene
    uint32_t *s_sid;       // per shadow segment: its scene
    // wavefront queues (ping-pong) and path state
    float4 *q_o[2], *q_d[2];
    uint32_t *q_path[2];
    uint32_t *count;       // [2]
    uint32_t capacity;
    int *hit_tri;
    float *hit_t;
    float4 *beta;
    float4 *s_o, *s_d, *s_c;  // shadow segments and their contribution (w = pixel bits)
    uint32_t *sh_count;
    uint32_t sh_capacity;
    float4 *accum;         // per pixel rgb sums, plus one discard slot at discard_pixel
    uint32_t discard_pixel;
    float4 *accum_direct;  // per pixel sums of the first vertex's emission and light samples (or null)
    float4 *accum_albedo;  // per pixel sums of the first hit's albedo (or null)
    uint32_t *err;
    unsigned long long *stats;  // counted render: [closest rays, nodes, tris, shadow rays, nodes, tris], or null
    // persistent (dynamic-fetch) extend and shadow kernels; off when every
    // scene is tiny, where rays are too short for refills to pay
    uint32_t persistent;

    // radiance cache (cache_depth == 0: plain path tracing, none of this is used)
    uint32_t cache_depth;      // rendering paths stop into the cache at this vertex
    uint32_t train_every;      // one path in train_every is a training path
    uint32_t train_tail;       // training paths stop into the cache at vertex cache_depth + train_tail
                               // (0: they are traced to the full depth)
    float3 scene_lo, scene_inv_ext;
    uint32_t *train_slot;      // per path of the wave: training slot or ~0
    uint32_t *train_count;     // training slots handed out in this wave
    uint32_t train_cap;
    uint32_t *rec_of;          // train_cap x (max_depth + 1): record of (slot, vertex) or ~0
    float *rec_feat;           // rec_cap x 16 raw features
    float4 *rec_beta;          // throughput at the recorded vertex
    float *rec_tgt;            // rec_cap x 3: radiance leaving the vertex, summed over the path's tail
    uint32_t *rec_count;
    uint32_t rec_cap;
    float *qry_feat;           // cache queries of rendering paths: cap x 16
    float4 *qry_beta;          // throughput (w = pixel bits)
    float *qry_out;            // cap x 3 network outputs
    uint32_t *qry_count;
    uint32_t *qry_meta;        // per query: (slot << 8 | vertex) of a training path's tail, or ~0
    // hash-grid radiance cache (the non-learned baseline; null: the network answers queries)
    unsigned long long *hc_keys;  // hc_mask + 1 cells: key + 1, 0 = empty
    float4 *hc_vals;              // per cell: radiance sum (xyz) and sample count (w)
    uint32_t *hc_dropped;         // records of the call that found no free cell in their probe window
    uint32_t *s_meta;          // per shadow segment: (slot << 8 | vertex) of a training path, or ~0
};

// light_range: per light (first triangle, triangle count) in the uploaded mesh
cudaError_t build_tri_attr(const uint32_t *prim_of, uint32_t n_tris, const uint32_t *mat_ids,
                           const uint2 *light_range, uint32_t n_lights, uint32_t *light_of_prim,
                           uint32_t *attr, cudaStream_t st);
// area[k] = area of uploaded triangle first + k (0.5 |(v1 - v0) x (v2 - v0)|,
// IndexedTriangle::GetArea, Core/Shape/IndexedTriangle.cpp:386-393)
cudaError_t triangle_areas(const float *pos, const uint32_t *idx, uint32_t first, uint32_t count, float *area,
                           cudaStream_t st);
struct MlpDev;
// One wave: global paths [wave_begin, wave_begin + n_paths).
cudaError_t render_wave(const RenderDev &R, uint32_t n_paths, uint64_t wave_begin, cudaStream_t st,
                        uint32_t *launches, const MlpDev *cache, uint32_t block = 128);
cudaError_t render_resolve(const float4 *accum, uint32_t wh, float scale, float *out, cudaStream_t st);
// Every path of the render ([0, total)) in one persistent launch
// (k_render_persistent); `next` is a device counter. Plain renders only.
cudaError_t render_persistent(const RenderDev &R, uint64_t total, unsigned long long *next, uint32_t *launches,
                              cudaStream_t st);

// Hash-grid radiance cache: the n_rec training records of a call (raw
// features + targets) are added to their cells.
constexpr uint32_t kHashCacheCells = 1u << 22;
cudaError_t hash_cache_update(const RenderDev &R, uint32_t n_rec, cudaStream_t st);

}  // namespace ilg
