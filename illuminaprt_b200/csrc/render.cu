// Wavefront path tracer: the reference's PathIntegrator::Radiance bounce loop
// (Core/Integrator/PathIntegrator.cpp:44-367) restated as queue-driven
// kernels over SoA path state:
//
//   k_camera   one camera ray per (pixel, sample) of the wave
//              (BaseRenderer::RenderRegion, Core/Renderer/BaseRenderer.cpp:62-169;
//               PerspectiveCamera::GetRay, Core/Camera/PerspectiveCamera.cpp:44-60)
//   k_extend   closest hit of every queued ray (the traversal of trace.cuh)
//   k_shade    emission at depth 0, NEE toward every quad light but the hit one
//              (IIntegrator::SampleAllLights / EstimateDirectLighting,
//               Core/Integrator/Integrator.cpp:114-185; DiffuseAreaLight,
//               Core/Light/DiffuseAreaLight.cpp:52-69), BSDF sample, throughput,
//              Russian roulette after depth 3, spawn offset along the
//              geometric normal; pushes shadow rays and continuations with
//              warp-aggregated atomics (the queue compaction)
//   k_shadow   any hit of every shadow segment; unoccluded contributions are
//              added to the pixel
//   k_resolve  pixel sums / spp
//
// Random numbers come from a counter-based hash of (seed, pixel, sample,
// depth, dimension) instead of the reference's shared Mersenne twister, so
// images agree with the reference statistically, not bit for bit.
#include "bvh8.cuh"
#include "render.cuh"
#include "trace.cuh"
#include "mlp.cuh"
#include "devinfo.cuh"

#include <algorithm>
#include <cfloat>

namespace ilg {

namespace {

constexpr float kInvPi = 0.318309886183790671538f;
constexpr float kTwoPi = 6.28318530717958647692f;

__device__ __forceinline__ uint64_t mix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// uniform float in [0, 1) for one (path, dimension)
__device__ __forceinline__ float rnd(uint64_t key, uint32_t dim)
{
    return (float)(uint32_t)(mix64(key + (uint64_t)dim * 0xD1B54A32D192ED03ull) >> 40) * 0x1p-24f;
}

__device__ __forceinline__ uint64_t path_key(uint32_t seed, uint64_t path_global)
{
    return mix64(path_global ^ ((uint64_t)seed * 0xA24BAED4963EE407ull));
}

// dimensions: per depth d, base 32*d: lights 2l, 2l+1 (l < 8); bsdf 20, 21, 22; roulette 23
constexpr uint32_t kDimCam = 0xFFFFFF00u;
__device__ __forceinline__ uint32_t dim_of(uint32_t depth, uint32_t k) { return depth * 32u + k; }

__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 normalize3(float3 a) { return a * rsqrtf(dot3(a, a)); }
__device__ __forceinline__ bool is_black(float3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }

// OrthonormalBasis::InitFromW, Core/Geometry/Basis.cpp:85-99
__device__ __forceinline__ void onb_from_w(float3 w, float3 &u, float3 &v)
{
    if (fabsf(w.x) > fabsf(w.y)) {
        float inv = 1.f / sqrtf(w.x * w.x + w.z * w.z);
        v = make_float3(-w.z * inv, 0.f, w.x * inv);
    } else {
        float inv = 1.f / sqrtf(w.y * w.y + w.z * w.z);
        v = make_float3(0.f, w.z * inv, -w.y * inv);
    }
    u = cross3(w, v);
}

// warp-aggregated queue push: returns this lane's slot (or 0xffffffff if !want)
__device__ __forceinline__ uint32_t push_slot(bool want, uint32_t *count)
{
    const uint32_t mask = __ballot_sync(__activemask(), want);
    if (!want) return 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t leader = __ffs(mask) - 1u;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}

__device__ __forceinline__ void add_pixel(float4 *accum, uint32_t pixel, float3 c)
{
    float *a = reinterpret_cast<float *>(accum + pixel);
    atomicAdd(a, c.x);
    atomicAdd(a + 1, c.y);
    atomicAdd(a + 2, c.z);
}

// scene of a global path index (the scenes' path ranges are consecutive)
__device__ __forceinline__ uint32_t scene_of(const RenderDev &R, uint64_t g)
{
    uint32_t lo = 0, hi = R.n_scenes;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (R.scenes[mid].path_begin <= g) lo = mid;
        else hi = mid;
    }
    return lo;
}

// path identity inside its scene: (pixel, sample-sequence key)
// (pixel = index in the rendered region, image coordinates x, y). The key
// depends on the image pixel and the sample only, so a region renders exactly
// the paths the whole image renders there.
__device__ __forceinline__ void path_ident(const SceneRec &S, uint64_t g, uint32_t &pixel, uint64_t &key,
                                           uint32_t &x, uint32_t &y)
{
    const uint64_t local = g - S.path_begin;
    const uint64_t sample = local / S.wh;
    pixel = (uint32_t)(local - sample * S.wh);
    x = S.region_x + pixel % S.region_w;
    y = S.region_y + pixel / S.region_w;
    key = path_key(S.seed, sample * S.full_wh + (uint64_t)y * S.width + x);
}

__global__ void k_camera(RenderDev R, uint32_t n_paths, uint64_t wave_begin)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0) R.count[0] = n_paths;  // the wave's first extend queue is every path
    if (p >= n_paths) return;
    const uint64_t g = wave_begin + p;
    const uint32_t sid = scene_of(R, g);
    const SceneRec &S = R.scenes[sid];
    uint32_t pixel, x, y;
    uint64_t key;
    path_ident(S, g, pixel, key, x, y);
    if (S.ray_o) {
        // a path from the caller's ray (IIntegrator::Radiance(..., ray, ...),
        // whose first intersection uses the ray's own [Min, Max])
        R.q_o[0][p] = S.ray_o[pixel];
        R.q_d[0][p] = S.ray_d[pixel];
    } else {
        // BoxFilter shifts the [0,1) sample by -0.5 (Core/Filter/BoxFilter.cpp:20-28)
        const float xi1 = rnd(key, kDimCam) - 0.5f, xi2 = rnd(key, kDimCam + 1) - 0.5f;
        const float fx = x * S.rcp_w + xi1 * S.rcp_w, fy = y * S.rcp_h + xi2 * S.rcp_h;
        const float3 target = S.corner + S.across * fx + S.up * fy;
        const float3 d = normalize3(target - S.centre);
        R.q_o[0][p] = make_float4(S.centre.x, S.centre.y, S.centre.z, 0.f);
        R.q_d[0][p] = make_float4(d.x, d.y, d.z, FLT_MAX);
    }
    R.q_path[0][p] = p;
    R.path_scene[p] = sid;
    R.beta[p] = make_float4(1.f, 1.f, 1.f, 0.f);
    if (R.cache_depth) {
        uint32_t slot = 0xffffffffu;
        if (mix64(key ^ 0x5851F42D4C957F2Dull) % R.train_every == 0) {
            const uint32_t s = atomicAdd(R.train_count, 1u);
            if (s < R.train_cap) slot = s;
        }
        R.train_slot[p] = slot;
    }
}

// Adds contribution c, found at vertex `vert` of a training path, to the
// targets of that path's recorded vertices 1..vert (each in units of the
// radiance leaving its own vertex: divided by the throughput there).
__device__ __forceinline__ void credit(const RenderDev &R, uint32_t slot, uint32_t vert, float3 c)
{
    const uint32_t stride = R.depth_max + 1;
    for (uint32_t k = 1; k <= vert && k <= R.depth_max; k++) {
        const uint32_t ri = R.rec_of[slot * stride + k];
        if (ri == 0xffffffffu || ri >= R.rec_cap) continue;
        const float4 b = R.rec_beta[ri];
        atomicAdd(&R.rec_tgt[3 * ri], c.x / fmaxf(b.x, 1e-8f));
        atomicAdd(&R.rec_tgt[3 * ri + 1], c.y / fmaxf(b.y, 1e-8f));
        atomicAdd(&R.rec_tgt[3 * ri + 2], c.z / fmaxf(b.z, 1e-8f));
    }
}

__device__ __forceinline__ void write_features(float *f, const RenderDev &R, float3 p, float3 wo, float3 n,
                                               const Mat &m)
{
    f[0] = (p.x - R.scene_lo.x) * R.scene_inv_ext.x;
    f[1] = (p.y - R.scene_lo.y) * R.scene_inv_ext.y;
    f[2] = (p.z - R.scene_lo.z) * R.scene_inv_ext.z;
    f[3] = wo.x; f[4] = wo.y; f[5] = wo.z;
    f[6] = n.x; f[7] = n.y; f[8] = n.z;
    const bool ggx = m.kind == 1u;
    f[9] = ggx ? m.alpha : 1.f;
    const float3 a = ggx ? m.f0 : m.albedo;
    f[10] = a.x; f[11] = a.y; f[12] = a.z;
    f[13] = f[14] = f[15] = 0.f;
}

// Work counters of a counted render: R.stats[k0] += rays, [k0 + 1] += node
// records read, [k0 + 2] += triangle records tested (one atomic per warp).
__device__ __forceinline__ void count_work(const RenderDev &R, int k0, bool ray, unsigned long long nn,
                                           unsigned long long nt)
{
    unsigned long long r = ray ? 1ull : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        r += __shfl_xor_sync(0xffffffffu, r, o);
        nn += __shfl_xor_sync(0xffffffffu, nn, o);
        nt += __shfl_xor_sync(0xffffffffu, nt, o);
    }
    if ((threadIdx.x & 31u) == 0u && r) {
        atomicAdd(R.stats + k0, r);
        atomicAdd(R.stats + k0 + 1, nn);
        atomicAdd(R.stats + k0 + 2, nt);
    }
}

// An unoccluded shadow segment adds its contribution to its pixel (and to
// Direct when tagged), and credits the training record it belongs to.
__device__ __forceinline__ void shadow_unoccluded(const RenderDev &R, uint32_t i)
{
    const float4 c = R.s_c[i];
    const uint32_t bits = __float_as_uint(c.w);
    add_pixel(R.accum, bits & 0x7fffffffu, make_float3(c.x, c.y, c.z));
    if (bits >> 31) add_pixel(R.accum_direct, bits & 0x7fffffffu, make_float3(c.x, c.y, c.z));
    if (R.cache_depth) {
        const uint32_t meta = R.s_meta[i];
        if (meta != 0xffffffffu) credit(R, meta >> 8, meta & 0xffu, make_float3(c.x, c.y, c.z));
    }
}

template <bool kStats>
__global__ void __launch_bounds__(256) k_extend(RenderDev R, int cur)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < R.count[cur];
    if (!kStats && !live) return;
    unsigned long long nn = 0, nt = 0;
    if (live) {
        const float4 o = R.q_o[cur][i], d = R.q_d[cur][i];
        const SceneRec &S = R.scenes[R.path_scene[R.q_path[cur][i]]];
        int best;
        float bt, bu, bv;
        trace_one<false, kStats>(S.nodes, S.tris, S.n_nodes, S.n_tris, o, d, best, bt, bu, bv, R.err, nn, nt);
        R.hit_tri[i] = best;
        R.hit_t[i] = bt;
    }
    if (kStats) count_work(R, 0, live, nn, nt);
}

// GGX conductor (Trowbridge-Reitz D, Smith G1 separable, Schlick F), sampled
// with the visible-normal distribution (Heitz 2018). Local frame: z = normal.
__device__ __forceinline__ float ggx_d(float3 h, float a)
{
    const float a2 = a * a;
    const float t = h.x * h.x / a2 + h.y * h.y / a2 + h.z * h.z;
    return 1.f / (3.14159265358979f * a2 * t * t);
}
__device__ __forceinline__ float ggx_g1(float3 w, float a)
{
    const float z2 = w.z * w.z;
    if (z2 <= 0.f) return 0.f;
    const float t2 = (w.x * w.x + w.y * w.y) * a * a / z2;
    return 2.f / (1.f + sqrtf(1.f + t2));
}
__device__ __forceinline__ float3 schlick(float3 f0, float c)
{
    const float m = 1.f - fminf(fmaxf(c, 0.f), 1.f);
    const float m5 = m * m * m * m * m;
    return f0 + (make_float3(1.f, 1.f, 1.f) - f0) * m5;
}
__device__ __forceinline__ float3 ggx_f(float3 wo, float3 wi, float3 f0, float a)
{
    if (wo.z <= 0.f || wi.z <= 0.f) return make_float3(0.f, 0.f, 0.f);
    const float3 h = normalize3(wo + wi);
    const float g = ggx_g1(wo, a) * ggx_g1(wi, a);
    return schlick(f0, dot3(wi, h)) * (ggx_d(h, a) * g / (4.f * wo.z * wi.z));
}
__device__ __forceinline__ float ggx_pdf(float3 wo, float3 wi, float a)
{
    if (wo.z <= 0.f || wi.z <= 0.f) return 0.f;
    const float3 h = normalize3(wo + wi);
    // pdf of the visible normal h, times the reflection Jacobian 1 / (4 wo.h)
    return ggx_g1(wo, a) * fmaxf(dot3(wo, h), 0.f) * ggx_d(h, a) / wo.z / (4.f * dot3(wo, h));
}
__device__ __forceinline__ float3 ggx_sample_vndf(float3 wo, float a, float u1, float u2)
{
    const float3 vh = normalize3(make_float3(a * wo.x, a * wo.y, wo.z));
    const float lensq = vh.x * vh.x + vh.y * vh.y;
    const float3 t1 = lensq > 0.f ? make_float3(-vh.y, vh.x, 0.f) * rsqrtf(lensq) : make_float3(1.f, 0.f, 0.f);
    const float3 t2 = cross3(vh, t1);
    const float r = sqrtf(u1);
    float s, c;
    sincosf(kTwoPi * u2, &s, &c);
    const float p1 = r * c;
    float p2 = r * s;
    const float sh = 0.5f * (1.f + vh.z);
    p2 = (1.f - sh) * sqrtf(fmaxf(0.f, 1.f - p1 * p1)) + sh * p2;
    const float3 nh = t1 * p1 + t2 * p2 + vh * sqrtf(fmaxf(0.f, 1.f - p1 * p1 - p2 * p2));
    const float3 h = normalize3(make_float3(a * nh.x, a * nh.y, fmaxf(0.f, nh.z)));
    const float3 wi = h * (2.f * dot3(wo, h)) - wo;
    return wi;
}

// BSDF::F for one material in the local frame (Core/Material/BSDF.cpp:214-234:
// reflection lobes only count when wi.z > 0)
// BSDF value for a direction pair; the specular materials (mirror, glass)
// are zero for every pair, as their BxDFs' F is (SpecularReflection::F,
// SpecularTransmission::F).
__device__ __forceinline__ float3 bsdf_f(const Mat &m, float3 wo, float3 wi)
{
    if (m.kind == 1u) return ggx_f(wo, wi, m.f0, m.alpha);
    if (m.kind == 0u && wi.z > 0.f) return m.albedo * kInvPi;
    return make_float3(0.f, 0.f, 0.f);
}

// Specular sampling of the reference's MirrorMaterial and GlassMaterial in
// the local frame (z = normal). Mirror: SpecularReflection::SampleF
// (Core/Material/SpecularReflectionBxDF.cpp:26-33): wi = (-wo.x, -wo.y,
// wo.z), pdf 1, f = reflectivity / |wi.z|. Glass: BSDF::SampleF
// (Core/Material/BSDF.cpp:141-211) picks one of its two BxDFs with the 1D
// sample (index (int)(w * 2) % 2: 0 = SpecularTransmission with the
// transmittance, 1 = SpecularReflection with the reflectivity) and halves
// the pdf; SpecularTransmission::SampleF
// (Core/Material/SpecularTransmissionBxDF.cpp:24-58) refracts by the ratio
// of indices with no Fresnel weight, and total internal reflection gives
// f = 0 (the path ends). `transmit` tells the caller to offset the next ray
// origin below the surface (PathIntegrator.cpp:184-187).
__device__ __forceinline__ void sample_specular(const Mat &m, float3 wo, float w, float3 &wi, float3 &f, float &pdf,
                                                bool &transmit)
{
    transmit = false;
    const float3 zero = make_float3(0.f, 0.f, 0.f);
    if (m.kind == 2u || (int)(w * 2.f) % 2 == 1) {
        wi = make_float3(-wo.x, -wo.y, wo.z);
        f = m.albedo * (1.f / fabsf(wi.z));
        pdf = m.kind == 2u ? 1.f : 0.5f;
        return;
    }
    // glass, transmission: m.alpha holds eta_i / eta_t
    const bool entering = wo.z > 0.f;
    const float eta = entering ? m.alpha : 1.f / m.alpha;
    const float sin_i2 = 1.f - wo.z * wo.z;
    const float sin_t2 = sin_i2 * eta * eta;
    pdf = 0.5f;
    if (sin_t2 > 1.f) {
        wi = zero;
        f = zero;
        return;
    }
    float cos_t = sqrtf(fmaxf(0.f, 1.f - sin_t2));
    if (entering) cos_t = -cos_t;
    wi = make_float3(eta * -wo.x, eta * -wo.y, cos_t);
    f = m.f0 * (1.f / fabsf(cos_t));
    transmit = true;
}

// One light sample of next-event estimation at a shading point
// (IIntegrator::EstimateDirectLighting, Core/Integrator/Integrator.cpp:114-139,
// with the light's SampleRadiance): light l's shadow segment and the
// contribution it adds when unoccluded; false when the sample adds nothing.
// The shading frame is (U, V, W) with W the shading normal; wo_l is the
// outgoing direction in it.
__device__ __forceinline__ bool light_sample(const SceneRec &S, uint32_t l, uint64_t key, uint32_t depth, float3 p,
                                             float3 U, float3 V, float3 W, float3 wo_l, const Mat &m, float3 beta,
                                             float4 &so, float4 &sd, float3 &c)
{
    const Light &L = S.lights[l];
    const float u = rnd(key, dim_of(depth, 2 * l)), v = rnd(key, dim_of(depth, 2 * l + 1));
    if (L.kind == kLightInfinite) {
        // InfiniteAreaLight::SampleRadiance (InfiniteAreaLight.cpp:73-83):
        // a direction in the cone cos(theta) >= 1e-4 about the shading
        // normal (Montecarlo::UniformSampleCone, Montecarlo.h:74-80), the
        // light's intensity with no division by the pdf, a shadow ray
        // over [1e-4, FLT_MAX] from the point itself
        const float ct = (1.f - u) + u * 1e-4f;
        const float st = sqrtf(1.f - ct * ct);
        float sp, cp;
        sincosf(kTwoPi * v, &sp, &cp);
        const float3 wi = U * (cp * st) + V * (sp * st) + W * ct;
        const float3 wi_l = make_float3(dot3(U, wi), dot3(V, wi), dot3(W, wi));
        c = beta * L.emit * fmaxf(0.f, dot3(wi, W)) * bsdf_f(m, wo_l, wi_l);
        if (is_black(c)) return false;
        so = make_float4(p.x, p.y, p.z, 1e-4f);
        sd = make_float4(wi.x, wi.y, wi.z, FLT_MAX);
        return true;
    }
    float3 P, nl;
    if (L.kind == kLightMesh) {
        // ITriangleMesh::SamplePoint (Core/Shape/TriangleMesh.cpp:142-161):
        // a triangle picked uniformly by index (not by area), a uniform
        // point on it (IndexedTriangle::SamplePoint, Montecarlo.h:59-64),
        // its normal (p3 - p1) x (p2 - p1) turned to face the shaded
        // point; the pdf is 1 / the mesh's whole area (DiffuseAreaLight.cpp:36-40)
        const uint32_t k = min((uint32_t)((float)L.tri_count * rnd(key, dim_of(depth, 24 + l))),
                               L.tri_count - 1u);
        const uint32_t *tv = S.idx + 3ull * (L.first_tri + k);
        const float *a = S.pos + 3ull * tv[0], *b = S.pos + 3ull * tv[1], *cc = S.pos + 3ull * tv[2];
        const float3 p1 = make_float3(a[0], a[1], a[2]), p2 = make_float3(b[0], b[1], b[2]),
                     p3 = make_float3(cc[0], cc[1], cc[2]);
        const float su = sqrtf(u);
        const float b1 = 1.f - su, b2 = v * su;
        P = p1 * b1 + p2 * b2 + p3 * (1.f - b1 - b2);
        nl = normalize3(cross3(p3 - p1, p2 - p1));
        if (dot3(P - p, nl) > 0.f) nl = nl * -1.f;
    } else {
        // Quad::SamplePoint (Core/Shape/Quad.cpp:144-153): a bilinear
        // patch over the reference's tessellation vertices
        P = L.p[0] + (L.p[2] - L.p[0]) * u + (L.p[3] - L.p[2]) * v +
            (L.p[0] - L.p[2] + L.p[1] - L.p[3]) * (u * v);
        nl = L.n;
    }
    float3 win = p - P;
    const float dist2 = dot3(win, win);
    win = normalize3(win);
    const float cl = fmaxf(0.f, dot3(win, nl));
    const float3 Ls = L.emit * (cl * L.area / dist2);
    if (is_black(Ls)) return false;
    const float3 wi = win * -1.f;
    const float3 wi_l = make_float3(dot3(U, wi), dot3(V, wi), dot3(W, wi));
    c = beta * Ls * (fmaxf(0.f, dot3(wi, W))) * bsdf_f(m, wo_l, wi_l);
    if (is_black(c)) return false;
    const float3 seg = P - p;
    so = make_float4(p.x, p.y, p.z, S.eps);
    sd = make_float4(seg.x, seg.y, seg.z, 1.f - S.eps);
    return true;
}

// The path's next ray (PathIntegrator.cpp:141-187): a BSDF sample
// (BSDF::SampleF, Core/Material/BSDF.cpp:141-211), the throughput update,
// Russian roulette after depth 3 and the spawn offset along the geometric
// normal (below the surface for a transmitted ray). False when the path
// ends here; beta is updated when it continues.
__device__ __forceinline__ bool continue_path(const SceneRec &S, uint64_t key, uint32_t depth, const Mat &m,
                                              bool specular, float3 p, float3 ng, float3 U, float3 V, float3 W,
                                              float3 wo_l, float3 &beta, float4 &no, float4 &nd)
{
    const float u1 = rnd(key, dim_of(depth, 20)), u2 = rnd(key, dim_of(depth, 21));
    float3 wi_l, f;
    float pdf;
    bool transmit = false;
    if (specular) {
        sample_specular(m, wo_l, rnd(key, dim_of(depth, 22)), wi_l, f, pdf, transmit);
    } else if (m.kind == 1u) {
        wi_l = ggx_sample_vndf(wo_l, m.alpha, u1, u2);
        pdf = ggx_pdf(wo_l, wi_l, m.alpha);
        f = ggx_f(wo_l, wi_l, m.f0, m.alpha);
    } else {
        // Lambertian::SampleF (Core/Material/LambertianBxDF.cpp:27-37)
        const float r = sqrtf(u1);
        float s, c;
        sincosf(kTwoPi * u2, &s, &c);
        wi_l = make_float3(r * c, r * s, sqrtf(1.f - u1));
        if (wo_l.z < 0.f) wi_l.z = -wi_l.z;
        pdf = fabsf(wi_l.z) * kInvPi;
        f = bsdf_f(m, wo_l, wi_l);
    }
    if (is_black(f) || !(pdf > 0.f)) return false;
    const float3 wi = U * wi_l.x + V * wi_l.y + W * wi_l.z;
    float3 b = beta * f * (fabsf(dot3(wi, W)) / pdf);
    if (depth > 3) {
        const float q = fminf(0.5f, 0.212671f * b.x + 0.715160f * b.y + 0.072169f * b.z);
        if (rnd(key, dim_of(depth, 23)) > q) return false;
        b = b * (1.f / q);
    }
    beta = b;
    // a transmitted ray starts below the surface (PathIntegrator.cpp:184-187)
    const float3 org = p + ng * (transmit ? -S.eps : S.eps);
    no = make_float4(org.x, org.y, org.z, S.eps);
    nd = make_float4(wi.x, wi.y, wi.z, FLT_MAX);
    return true;
}

__global__ void __launch_bounds__(256) k_shade(RenderDev R, int cur, uint32_t depth, uint64_t wave_begin)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const int nxt = cur ^ 1;
    bool cont = false;
    float4 no = make_float4(0.f, 0.f, 0.f, 0.f), nd = no;
    uint32_t path = 0;
    uint32_t pixel = 0;
    bool query = false;           // rendering path stopping into the cache here
    float4 qb = make_float4(0.f, 0.f, 0.f, 0.f);
    float qf[kMlpRaw];
    uint32_t tslot = 0xffffffffu;  // training slot of this path
    uint32_t qmeta = 0xffffffffu;  // the query's training tail, if it is one
    uint32_t sid = 0;

    if (i < R.count[cur]) {
        path = R.q_path[cur][i];
        if (R.cache_depth) tslot = R.train_slot[path];
        sid = R.path_scene[path];
        const SceneRec &S = R.scenes[sid];
        const float4 o = R.q_o[cur][i], d = R.q_d[cur][i];
        const int ti = R.hit_tri[i];
        uint64_t key;
        uint32_t px, py;
        path_ident(S, wave_begin + path, pixel, key, px, py);
        pixel += S.pixel_base;
        // A training path's pixel takes the cache's value at the cache vertex,
        // as a rendering path's does; what its tail adds from there on (light
        // samples at that vertex and beyond, escapes after it) only trains the
        // cache and goes to the discard slot past the last pixel.
        const uint32_t image_pixel = pixel;
        if (R.cache_depth && tslot != 0xffffffffu &&
            (ti >= 0 ? depth >= R.cache_depth : depth > R.cache_depth))
            pixel = R.discard_pixel;
        const float4 beta4 = R.beta[path];
        float3 beta = make_float3(beta4.x, beta4.y, beta4.z);
        const bool after_specular = beta4.w != 0.f;  // the previous bounce was a specular one
        float3 add = make_float3(0.f, 0.f, 0.f);

        if (ti < 0) {
            // escape: constant environment (zero for the reference's area-light scenes)
            add = beta * S.sky;
            // the reference's infinite lights, seen by a camera ray or after a
            // specular bounce (PathIntegrator.cpp:84-92 and :194-198)
            if ((depth == 0 || after_specular) && S.inf_escape > 0.f) add = add + beta * S.inf_escape;
            if (tslot != 0xffffffffu && depth >= 2 && !is_black(add)) credit(R, tslot, depth - 1, add);
        } else if (depth <= S.max_depth) {
            const uint32_t attr = S.tri_attr[ti];
            const uint32_t mat_id = attr & 0xffffu, light_id = attr >> 16;
            const Mat m = S.mats[mat_id < S.n_mats ? mat_id : 0];
            const Tri tr = S.tris[ti];
            const float3 ng = normalize3(make_float3(tr.a.w, tr.b.w, tr.c.w));
            const float t = R.hit_t[i];
            const float3 dd = make_float3(d.x, d.y, d.z);
            const float3 p = make_float3(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
            const float3 wo = normalize3(dd) * -1.f;
            // flat shading: the shading normal is the face normal
            const float3 W = ng;
            float3 U, V;
            onb_from_w(W, U, V);
            const float3 wo_l = make_float3(dot3(U, wo), dot3(V, wo), dot3(W, wo));

            // emission at depth 0 or right after a specular bounce
            // (PathIntegrator.cpp:126-128), one-sided (DiffuseAreaLight::Radiance,
            // DiffuseAreaLight.cpp:47-50)
            if ((depth == 0 || after_specular) && light_id != 0xffffu && light_id < S.n_lights &&
                dot3(W, wo) > 0.f) {
                const float3 e = beta * S.lights[light_id].emit;
                add = add + e;
                if (tslot != 0xffffffffu && depth >= 2) credit(R, tslot, depth - 1, e);
            }
            // RadianceContext::Albedo = the first hit's Material::Rho
            // (PathIntegrator.cpp:121): the reflectance; for the GGX conductor
            // its F0; for glass the sum over its two BxDFs (BSDF::Rho,
            // Core/Material/BSDF.cpp:123-139)
            if (depth == 0 && R.accum_albedo)
                add_pixel(R.accum_albedo, pixel,
                          m.kind == 1u ? m.f0 : (m.kind == 3u ? m.albedo + m.f0 : m.albedo));
            const bool specular = m.kind >= 2u;

            const bool at_cache = depth < S.max_depth && R.cache_depth && depth == R.cache_depth;
            // a training path with a short tail stops into the cache too; the
            // cache's answer there completes the targets of its records
            // (self-training), not its pixel
            const bool at_tail = depth < S.max_depth && R.train_tail && tslot != 0xffffffffu &&
                                 depth == R.cache_depth + R.train_tail;
            if (at_cache) {
                // the cache supplies the radiance leaving this vertex to the pixel
                query = true;
                write_features(qf, R, p, wo, W, m);
                qb = make_float4(beta.x, beta.y, beta.z, __uint_as_float(image_pixel));
            }
            if (at_tail) {
                query = true;
                qmeta = (tslot << 8) | depth;
                write_features(qf, R, p, wo, W, m);
                qb = make_float4(beta.x, beta.y, beta.z, __uint_as_float(R.discard_pixel));
            }
            if ((at_cache && tslot == 0xffffffffu) || at_tail) {
                // the path stops here
            } else if (depth < S.max_depth) {
                if (tslot != 0xffffffffu && depth >= 1) {
                    // training record of this vertex; its target fills in as the tail is traced
                    const uint32_t ri = atomicAdd(R.rec_count, 1u);
                    uint32_t stored = 0xffffffffu;
                    if (ri < R.rec_cap) {
                        float f[kMlpRaw];
                        write_features(f, R, p, wo, W, m);
#pragma unroll
                        for (int k = 0; k < kMlpRaw; k++) R.rec_feat[(size_t)ri * kMlpRaw + k] = f[k];
                        R.rec_beta[ri] = make_float4(beta.x, beta.y, beta.z, 0.f);
                        R.rec_tgt[3 * ri] = R.rec_tgt[3 * ri + 1] = R.rec_tgt[3 * ri + 2] = 0.f;
                        stored = ri;
                    }
                    R.rec_of[tslot * (R.depth_max + 1) + depth] = stored;
                }
                // next-event estimation toward every light but the one hit (a
                // specular BSDF's F is zero for every light direction); each
                // sample goes to the shadow queue as it is made
                for (uint32_t l = 0; l < S.n_lights && l < kMaxLights && !specular; l++) {
                    if (l == light_id) continue;
                    float4 so, sd;
                    float3 sc;
                    const bool ok = light_sample(S, l, key, depth, p, U, V, W, wo_l, m, beta, so, sd, sc);
                    const uint32_t s = push_slot(ok, R.sh_count);
                    if (ok) {
                        if (s < R.sh_capacity) {
                            R.s_o[s] = so;
                            R.s_d[s] = sd;
                            // bit 31 marks a light sample of the first vertex (Direct)
                            const uint32_t tag = (depth == 0 && R.accum_direct) ? 0x80000000u : 0u;
                            R.s_c[s] = make_float4(sc.x, sc.y, sc.z, __uint_as_float(pixel | tag));
                            R.s_sid[s] = sid;
                            if (R.cache_depth)
                                R.s_meta[s] = tslot == 0xffffffffu ? 0xffffffffu : ((tslot << 8) | depth);
                        } else {
                            atomicOr(R.err, 16u);
                        }
                    }
                }

                if (continue_path(S, key, depth, m, specular, p, ng, U, V, W, wo_l, beta, no, nd)) {
                    cont = true;
                    R.beta[path] = make_float4(beta.x, beta.y, beta.z, specular ? 1.f : 0.f);
                }
            }
        }
        if (!is_black(add)) {
            add_pixel(R.accum, pixel, add);
            // what the first vertex adds is RadianceContext::Direct (PathIntegrator.cpp:102)
            if (depth == 0 && R.accum_direct) add_pixel(R.accum_direct, pixel, add);
        }
    }

    const uint32_t slot = push_slot(cont, &R.count[nxt]);
    if (cont) {
        if (slot < R.capacity) {
            R.q_o[nxt][slot] = no;
            R.q_d[nxt][slot] = nd;
            R.q_path[nxt][slot] = path;
        } else {
            atomicOr(R.err, 8u);
        }
    }
    if (R.cache_depth) {
        const uint32_t q = push_slot(query, R.qry_count);
        if (query) {
            if (q < R.capacity) {
#pragma unroll
                for (int k = 0; k < kMlpRaw; k++) R.qry_feat[(size_t)q * kMlpRaw + k] = qf[k];
                R.qry_beta[q] = qb;
                R.qry_meta[q] = qmeta;
            } else {
                atomicOr(R.err, 32u);
            }
        }
    }
}

// pixel += throughput * max(cache output, 0) for every cache query of the
// wave; a training tail's answer goes to its path's records instead (its
// pixel is the discard slot)
__global__ void k_cache_apply(RenderDev R)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *R.qry_count || i >= R.capacity) return;
    const float4 b = R.qry_beta[i];
    const float3 y = make_float3(fmaxf(R.qry_out[3 * i], 0.f), fmaxf(R.qry_out[3 * i + 1], 0.f),
                                 fmaxf(R.qry_out[3 * i + 2], 0.f));
    const float3 c = make_float3(b.x * y.x, b.y * y.y, b.z * y.z);
    add_pixel(R.accum, __float_as_uint(b.w), c);
    if (R.train_tail) {
        const uint32_t meta = R.qry_meta[i];
        if (meta != 0xffffffffu) credit(R, meta >> 8, meta & 0xffu, c);
    }
}

template <bool kStats>
__global__ void __launch_bounds__(256) k_shadow(RenderDev R)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < *R.sh_count;
    if (!kStats && !live) return;
    unsigned long long nn = 0, nt = 0;
    int best = -2;
    if (live) {
        const float4 o = R.s_o[i], d = R.s_d[i];
        const SceneRec &S = R.scenes[R.s_sid[i]];
        float bt, bu, bv;
        trace_one<true, kStats>(S.nodes, S.tris, S.n_nodes, S.n_tris, o, d, best, bt, bu, bv, R.err, nn, nt);
    }
    if (kStats) count_work(R, 3, live, nn, nt);
    if (live && best == -1) shadow_unoccluded(R, i);
}

// ---------------------------------------------------------------------------
// Persistent forms of k_extend and k_shadow: each warp keeps its lanes busy by
// fetching a new ray from a device counter whenever kRefillLanes lanes are
// idle (as k_trace_dyn does for batched queries), so the incoherent bounce
// and shadow rays do not leave lanes waiting on the longest ray of a warp.
// Rays of one warp may belong to different scenes of a batch; each lane
// traverses its own scene's tree.
// ---------------------------------------------------------------------------
template <bool kAnyHit>
__device__ __forceinline__ void wave_trace_dyn(const RenderDev &R, uint32_t n, uint32_t *next, int cur)
{
    const uint32_t lane = threadIdx.x & 31u;
    __shared__ uint2 sstack[kShortStack * kStackColumns];  // launched with kStackColumns threads a block
    uint2 lstack[kMaxStack - kShortStack];
    const SplitStack stack{sstack + threadIdx.x, lstack};
    RayState r;
    const Node8 *nodes = nullptr;
    const Tri *tris = nullptr;
    uint32_t n_nodes = 0, n_tris = 0;
    bool active = false, exhausted = false;  // exhausted is warp-uniform
    uint32_t id = 0;
    while (true) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !active);
        if (!exhausted && (__popc(idle) >= kRefillLanes || idle == 0xffffffffu)) {
            const uint32_t leader = __ffs(idle) - 1u;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(next, (uint32_t)__popc(idle));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base >= n) exhausted = true;
            if (!active) {
                const uint32_t k = base + __popc(idle & ((1u << lane) - 1u));
                if (k < n) {
                    id = k;
                    const SceneRec &S = R.scenes[kAnyHit ? R.s_sid[id] : R.path_scene[R.q_path[cur][id]]];
                    nodes = S.nodes;
                    tris = S.tris;
                    n_nodes = S.n_nodes;
                    n_tris = S.n_tris;
                    if (kAnyHit) ray_init(r, R.s_o[id], R.s_d[id], n_nodes);
                    else ray_init(r, R.q_o[cur][id], R.q_d[cur][id], n_nodes);
                    active = true;
                }
            }
        }
        if (__ballot_sync(0xffffffffu, active) == 0u) break;
        if (active && ray_step<kAnyHit, false, false, false, kTrisPerStep, false, SplitStack>(r, stack, nodes, tris,
                                                                                         n_nodes, n_tris, R.err)) {
            if (kAnyHit) {
                if (r.best == -1) shadow_unoccluded(R, id);
            } else {
                R.hit_tri[id] = r.best;
                R.hit_t[id] = r.best >= 0 ? r.tcur : __int_as_float(0x7f800000);
            }
            active = false;
        }
    }
}

// The shadow rays of depth d and the extension rays of depth d + 1 in one
// persistent launch: both come from k_shade at depth d and neither reads
// what the other writes (shadow rays add to the pixel sums and training
// targets, extension rays write hit records), so one traversal loop
// (ray_step<kMixed>) takes the extension rays first, then the shadow rays:
// twice the rays in flight and one launch tail instead of two. `cur` is the
// queue the extension rays are in.
__global__ void __launch_bounds__(kStackColumns) k_trace_mixed(RenderDev R, int cur, uint32_t *next)
{
    const uint32_t lane = threadIdx.x & 31u;
    __shared__ uint2 sstack[kShortStack * kStackColumns];  // launched with kStackColumns threads a block
    uint2 lstack[kMaxStack - kShortStack];
    const SplitStack stack{sstack + threadIdx.x, lstack};
    const uint32_t n_ext = min(R.count[cur], R.capacity), n_sh = min(*R.sh_count, R.sh_capacity);
    const uint32_t n = n_ext + n_sh;
    RayState r;
    const Node8 *nodes = nullptr;
    const Tri *tris = nullptr;
    uint32_t n_nodes = 0, n_tris = 0;
    bool active = false, exhausted = false;  // exhausted is warp-uniform
    uint32_t id = 0;
    while (true) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !active);
        if (!exhausted && (__popc(idle) >= kRefillLanes || idle == 0xffffffffu)) {
            const uint32_t leader = __ffs(idle) - 1u;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(next, (uint32_t)__popc(idle));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base >= n) exhausted = true;
            if (!active) {
                const uint32_t k = base + __popc(idle & ((1u << lane) - 1u));
                if (k < n) {
                    const bool shadow = k >= n_ext;
                    id = shadow ? k - n_ext : k;
                    const SceneRec &S = R.scenes[shadow ? R.s_sid[id] : R.path_scene[R.q_path[cur][id]]];
                    nodes = S.nodes;
                    tris = S.tris;
                    n_nodes = S.n_nodes;
                    n_tris = S.n_tris;
                    if (shadow) ray_init(r, R.s_o[id], R.s_d[id], n_nodes);
                    else ray_init(r, R.q_o[cur][id], R.q_d[cur][id], n_nodes);
                    r.any = shadow;
                    active = true;
                }
            }
        }
        if (__ballot_sync(0xffffffffu, active) == 0u) break;
        if (active && ray_step<false, false, false, false, kTrisPerStep, true, SplitStack>(r, stack, nodes, tris,
                                                                                             n_nodes, n_tris, R.err)) {
            if (r.any) {
                if (r.best == -1) shadow_unoccluded(R, id);
            } else {
                R.hit_tri[id] = r.best;
                R.hit_t[id] = r.best >= 0 ? r.tcur : __int_as_float(0x7f800000);
            }
            active = false;
        }
    }
}

__global__ void __launch_bounds__(kStackColumns) k_extend_dyn(RenderDev R, int cur, uint32_t *next)
{
    wave_trace_dyn<false>(R, min(R.count[cur], R.capacity), next, cur);
}

__global__ void __launch_bounds__(kStackColumns) k_shadow_dyn(RenderDev R, uint32_t *next)
{
    wave_trace_dyn<true>(R, min(*R.sh_count, R.sh_capacity), next, 0);
}

// ---------------------------------------------------------------------------
// The whole render as one persistent launch: each lane carries one path from
// its camera ray through every bounce (closest hit, shading, one shadow ray
// per light, the next ray) and takes a new path from a device counter when
// its path ends; a warp refills once kRefillLanesPersistent of its lanes are
// idle. The paths of every scene of a batch, of any length, flow through the
// same kernel with no host round trip and no queue in memory. Closest-hit
// and shadow rays share one traversal loop (ray_step<kMixed>), so lanes
// tracing either kind stay on the same code; lanes whose ray finished wait
// and shade together. The sample sequence, the shading code (light_sample,
// continue_path) and the traversal are the wavefront's, so every path is the
// wavefront path of the same index and the images agree up to the order of
// the float additions into each pixel. Plain renders only: no radiance
// cache, no Direct / Albedo outputs, no work counters.
// ---------------------------------------------------------------------------
struct PathLane {
    uint32_t sid, pixel, depth;
    uint64_t key;
    float3 beta;           // throughput at the current vertex
    bool after_specular;   // the previous bounce was specular
    // the vertex being lit: light samples still to trace, then the next ray
    float3 p, W, wo_l, nee_beta, next_beta;
    uint32_t mat_id, light_id, next_light;
    bool specular, cont;
    float4 no, nd;         // the next ray (when cont)
    float3 c;              // contribution of the shadow ray in flight
};

__device__ __forceinline__ void start_path(const RenderDev &R, uint64_t g, PathLane &P, RayState &r)
{
    const uint32_t sid = scene_of(R, g);
    const SceneRec &S = R.scenes[sid];
    uint32_t pixel, x, y;
    uint64_t key;
    path_ident(S, g, pixel, key, x, y);
    float4 o, d;
    if (S.ray_o) {
        o = S.ray_o[pixel];
        d = S.ray_d[pixel];
    } else {
        const float xi1 = rnd(key, kDimCam) - 0.5f, xi2 = rnd(key, kDimCam + 1) - 0.5f;
        const float fx = x * S.rcp_w + xi1 * S.rcp_w, fy = y * S.rcp_h + xi2 * S.rcp_h;
        const float3 target = S.corner + S.across * fx + S.up * fy;
        const float3 dd = normalize3(target - S.centre);
        o = make_float4(S.centre.x, S.centre.y, S.centre.z, 0.f);
        d = make_float4(dd.x, dd.y, dd.z, FLT_MAX);
    }
    P.sid = sid;
    P.pixel = pixel + S.pixel_base;
    P.depth = 0;
    P.key = key;
    P.beta = make_float3(1.f, 1.f, 1.f);
    P.after_specular = false;
    ray_init(r, o, d, S.n_nodes);
    r.any = false;
}

// The next light sample of the vertex with a contribution, as a shadow ray
// in r; false when none is left.
__device__ __forceinline__ bool next_light_sample(const RenderDev &R, PathLane &P, RayState &r)
{
    const SceneRec &S = R.scenes[P.sid];
    if (P.specular) return false;
    float3 U, V;
    onb_from_w(P.W, U, V);
    const Mat m = S.mats[P.mat_id < S.n_mats ? P.mat_id : 0];
    for (uint32_t l = P.next_light; l < S.n_lights && l < kMaxLights; l++) {
        if (l == P.light_id) continue;
        float4 so, sd;
        if (light_sample(S, l, P.key, P.depth, P.p, U, V, P.W, P.wo_l, m, P.nee_beta, so, sd, P.c)) {
            P.next_light = l + 1;
            ray_init(r, so, sd, S.n_nodes);
            r.any = true;
            return true;
        }
    }
    return false;
}

// After the vertex's light samples: the next ray, or the end of the path.
__device__ __forceinline__ bool next_bounce(const RenderDev &R, PathLane &P, RayState &r)
{
    if (!P.cont) return false;
    P.beta = P.next_beta;
    P.after_specular = P.specular;
    P.depth++;
    ray_init(r, P.no, P.nd, R.scenes[P.sid].n_nodes);
    r.any = false;
    return true;
}

// The closest hit of the path's ray is in r: what the vertex adds, and the
// vertex's state for its light samples and next ray (k_shade's rules).
// Returns whether the path goes on from this vertex.
__device__ __forceinline__ bool shade_vertex(const RenderDev &R, PathLane &P, const RayState &r, float4 o, float4 d)
{
    const SceneRec &S = R.scenes[P.sid];
    const int ti = r.best;
    const uint32_t depth = P.depth;
    float3 add = make_float3(0.f, 0.f, 0.f);
    if (ti < 0) {
        if (ti == -1) {
            add = P.beta * S.sky;
            if ((depth == 0 || P.after_specular) && S.inf_escape > 0.f) add = add + P.beta * S.inf_escape;
            if (!is_black(add)) add_pixel(R.accum, P.pixel, add);
        }
        return false;
    }
    if (depth > S.max_depth) return false;
    const uint32_t attr = S.tri_attr[ti];
    const uint32_t mat_id = attr & 0xffffu, light_id = attr >> 16;
    const Mat m = S.mats[mat_id < S.n_mats ? mat_id : 0];
    const Tri tr = S.tris[ti];
    const float3 ng = normalize3(make_float3(tr.a.w, tr.b.w, tr.c.w));
    const float t = r.tcur;
    const float3 p = make_float3(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
    const float3 wo = normalize3(make_float3(d.x, d.y, d.z)) * -1.f;
    const float3 W = ng;
    float3 U, V;
    onb_from_w(W, U, V);
    const float3 wo_l = make_float3(dot3(U, wo), dot3(V, wo), dot3(W, wo));
    if ((depth == 0 || P.after_specular) && light_id != 0xffffu && light_id < S.n_lights && dot3(W, wo) > 0.f)
        add = add + P.beta * S.lights[light_id].emit;
    if (!is_black(add)) add_pixel(R.accum, P.pixel, add);
    if (depth >= S.max_depth) return false;
    P.specular = m.kind >= 2u;
    P.p = p;
    P.W = W;
    P.wo_l = wo_l;
    P.mat_id = mat_id;
    P.light_id = light_id;
    P.next_light = 0;
    P.nee_beta = P.beta;
    P.next_beta = P.beta;
    P.cont = continue_path(S, P.key, depth, m, P.specular, p, ng, U, V, W, wo_l, P.next_beta, P.no, P.nd);
    return true;
}

constexpr int kPersistThreads = 128;
// A warp of the one-launch renderer takes new paths once 16 of its lanes are
// idle (a path start costs a camera ray and a scene lookup; 8 measured 2 %
// slower on the 32-scene batch, 4 5 % slower).
constexpr uint32_t kRefillLanesPersistent = 16;

__global__ void __launch_bounds__(kPersistThreads) k_render_persistent(RenderDev R, uint64_t total, unsigned long long *next)
{
    const uint32_t lane = threadIdx.x & 31u;
    uint2 stack[kMaxStack];
    RayState r;
    // The path state lives in shared memory, one slot per thread (the kernel
    // runs 128 threads a block): in registers it spilled the traversal's
    // working set; in shared memory the kernel renders 1.17x faster.
    __shared__ PathLane lanes[kPersistThreads];
    __shared__ float4 ray_io[kPersistThreads][2];  // the closest-hit ray in flight (for shading)
    PathLane &P = lanes[threadIdx.x];
    float4 &ro = ray_io[threadIdx.x][0], &rd = ray_io[threadIdx.x][1];
    ro = make_float4(0.f, 0.f, 0.f, 0.f);
    rd = ro;
    bool active = false, exhausted = false;  // exhausted is warp-uniform
    // 0: tracing; 1: closest hit found, waiting to shade; 2: shadow ray done, waiting to be counted
    uint32_t state = 0;
    const Node8 *nodes = nullptr;
    const Tri *tris = nullptr;
    uint32_t n_nodes = 0, n_tris = 0;
    auto bind_scene = [&]() {
        const SceneRec &S = R.scenes[P.sid];
        nodes = S.nodes;
        tris = S.tris;
        n_nodes = S.n_nodes;
        n_tris = S.n_tris;
    };
    while (true) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !active);
        if (!exhausted && (__popc(idle) >= kRefillLanesPersistent || idle == 0xffffffffu)) {
            const uint32_t leader = __ffs(idle) - 1u;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(next, (unsigned long long)__popc(idle));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base >= total) exhausted = true;
            if (!active) {
                const uint64_t k = base + __popc(idle & ((1u << lane) - 1u));
                if (k < total) {
                    start_path(R, k, P, r);
                    bind_scene();
                    ro = make_float4(r.ox, r.oy, r.oz, r.tmin);
                    rd = make_float4(r.dx, r.dy, r.dz, r.tcur);
                    active = true;
                    state = 0;
                }
            }
        }
        const uint32_t live = __ballot_sync(0xffffffffu, active);
        if (live == 0u) break;
        if (active && state == 0 &&
            ray_step<false, false, false, false, kTrisPerStep, true>(r, stack, nodes, tris, n_nodes, n_tris, R.err))
            state = r.any ? 2u : 1u;
        // Shading and shadow results run for the waiting lanes together, once
        // three quarters of the warp's paths wait or none is tracing, so that
        // this code runs with most lanes converged instead of one lane at a
        // time (measured on a B200: half the warp 215, three quarters 233,
        // seven eighths 243, all 239 Msamples/s on the 32-scene batch; on the
        // field 175 / 184 / 179 / 152).
        const uint32_t waiting = __ballot_sync(0xffffffffu, active && state != 0u);
        const uint32_t tracing = live & ~waiting;
        if (waiting && (4u * __popc(waiting) >= 3u * __popc(live) || tracing == 0u)) {
            // a shadow ray's light sample counts when nothing is in the way;
            // a closest hit is shaded; then either lane takes the vertex's
            // next light sample or its next ray (one copy of that code, so
            // the kernel stays small enough for the instruction cache)
            if (active && state == 2u && r.best == -1) add_pixel(R.accum, P.pixel, P.c);
            if (active && state == 1u) active = shade_vertex(R, P, r, ro, rd);
            if (active && state != 0u) {
                active = next_light_sample(R, P, r) || next_bounce(R, P, r);
                state = 0;
                if (active && !r.any) {
                    ro = make_float4(r.ox, r.oy, r.oz, r.tmin);
                    rd = make_float4(r.dx, r.dy, r.dz, r.tcur);
                }
            }
        }
    }
}

__global__ void k_resolve(const float4 *__restrict__ accum, uint32_t wh, float scale, float *__restrict__ out)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= wh) return;
    const float4 a = accum[p];
    out[3 * p] = a.x * scale;
    out[3 * p + 1] = a.y * scale;
    out[3 * p + 2] = a.z * scale;
}

__global__ void k_tri_attr(const uint32_t *__restrict__ prim_of, uint32_t n, const uint32_t *__restrict__ mat_ids,
                           const uint32_t *__restrict__ light_of_prim, uint32_t *__restrict__ attr)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t p = prim_of[i];
    attr[i] = (mat_ids ? (mat_ids[p] & 0xffffu) : 0u) | (light_of_prim[p] << 16);
}

__global__ void k_light_of_prim(uint32_t *lop, uint32_t n_prims, const uint2 *range, uint32_t n_lights)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_prims) return;
    uint32_t id = 0xffffu;
    for (uint32_t l = 0; l < n_lights; l++)
        if (i - range[l].x < range[l].y) id = l;
    lop[i] = id;
}

__global__ void k_tri_area(const float *__restrict__ pos, const uint32_t *__restrict__ idx, uint32_t first,
                           uint32_t count, float *__restrict__ area)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const uint32_t *tv = idx + 3ull * (first + k);
    const float *a = pos + 3ull * tv[0], *b = pos + 3ull * tv[1], *c = pos + 3ull * tv[2];
    const float3 e1 = make_float3(b[0] - a[0], b[1] - a[1], b[2] - a[2]);
    const float3 e2 = make_float3(c[0] - a[0], c[1] - a[1], c[2] - a[2]);
    const float3 n = cross3(e1, e2);
    area[k] = sqrtf(dot3(n, n)) * 0.5f;
}

inline uint32_t blocks_for(uint64_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

// Grid of a persistent kernel of 128-thread blocks over at most n items.
inline uint32_t persistent_blocks(uint64_t n)
{
    const int sms = current_sm_count();
    const uint32_t b = blocks_for(n, 128);
    const uint32_t cap = (uint32_t)sms * 16u;
    return b < 1u ? 1u : (b < cap ? b : cap);
}

}  // namespace

cudaError_t triangle_areas(const float *pos, const uint32_t *idx, uint32_t first, uint32_t count, float *area,
                           cudaStream_t st)
{
    if (count == 0) return cudaSuccess;
    k_tri_area<<<blocks_for(count, 256), 256, 0, st>>>(pos, idx, first, count, area);
    return cudaGetLastError();
}

cudaError_t build_tri_attr(const uint32_t *prim_of, uint32_t n_tris, const uint32_t *mat_ids,
                           const uint2 *light_range, uint32_t n_lights, uint32_t *light_of_prim,
                           uint32_t *attr, cudaStream_t st)
{
    k_light_of_prim<<<blocks_for(n_tris, 256), 256, 0, st>>>(light_of_prim, n_tris, light_range, n_lights);
    k_tri_attr<<<blocks_for(n_tris, 256), 256, 0, st>>>(prim_of, n_tris, mat_ids, light_of_prim, attr);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Hash-grid radiance cache: a non-learned stand-in for the network, the
// baseline the learned cache is measured against. A cell is a voxel of the
// scene's bounding box (256 per axis) crossed with the normal's dominant
// axis and sign (6) and the octant of the outgoing direction (8); it holds
// the running mean of the training records that fell in it. Lookup is
// open addressing over kHashCacheCells cells, 8 probes; a query that finds
// no filled cell answers 0.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long hc_key(const float *f)
{
    const uint32_t x = (uint32_t)fminf(fmaxf(f[0] * 256.f, 0.f), 255.f);
    const uint32_t y = (uint32_t)fminf(fmaxf(f[1] * 256.f, 0.f), 255.f);
    const uint32_t z = (uint32_t)fminf(fmaxf(f[2] * 256.f, 0.f), 255.f);
    const float ax = fabsf(f[6]), ay = fabsf(f[7]), az = fabsf(f[8]);
    const uint32_t axis = ax >= ay && ax >= az ? 0u : (ay >= az ? 1u : 2u);
    const uint32_t nsign = (axis == 0u ? f[6] : axis == 1u ? f[7] : f[8]) < 0.f ? 1u : 0u;
    const uint32_t oct = (f[3] < 0.f ? 1u : 0u) | (f[4] < 0.f ? 2u : 0u) | (f[5] < 0.f ? 4u : 0u);
    return (unsigned long long)x | ((unsigned long long)y << 8) | ((unsigned long long)z << 16) |
           ((unsigned long long)(axis * 2u + nsign) << 24) | ((unsigned long long)oct << 27);
}

__device__ __forceinline__ uint32_t hc_slot(unsigned long long key, uint32_t mask)
{
    unsigned long long h = key * 0x9E3779B97F4A7C15ull;
    h ^= h >> 29;
    return (uint32_t)h & mask;
}

__global__ void k_hc_update(RenderDev R, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *f = R.rec_feat + (size_t)i * kMlpRaw;
    const unsigned long long key = hc_key(f) + 1ull;
    const uint32_t mask = kHashCacheCells - 1u;
    uint32_t s = hc_slot(key, mask);
    for (int probe = 0; probe < 8; probe++, s = (s + 1u) & mask) {
        const unsigned long long prev = atomicCAS(R.hc_keys + s, 0ull, key);
        if (prev == 0ull || prev == key) {
            float *v = reinterpret_cast<float *>(R.hc_vals + s);
            atomicAdd(v, fmaxf(R.rec_tgt[3 * i], 0.f));
            atomicAdd(v + 1, fmaxf(R.rec_tgt[3 * i + 1], 0.f));
            atomicAdd(v + 2, fmaxf(R.rec_tgt[3 * i + 2], 0.f));
            atomicAdd(v + 3, 1.f);
            return;
        }
    }
    // all 8 probed cells hold other keys: the record is dropped (and counted)
    atomicAdd(R.hc_dropped, 1u);
}

__global__ void k_hc_query(RenderDev R, uint32_t cap)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *R.qry_count || i >= cap) return;
    const float *f = R.qry_feat + (size_t)i * kMlpRaw;
    const unsigned long long key = hc_key(f) + 1ull;
    const uint32_t mask = kHashCacheCells - 1u;
    uint32_t s = hc_slot(key, mask);
    float3 y = make_float3(0.f, 0.f, 0.f);
    for (int probe = 0; probe < 8; probe++, s = (s + 1u) & mask) {
        const unsigned long long k = R.hc_keys[s];
        if (k == 0ull) break;
        if (k == key) {
            const float4 v = R.hc_vals[s];
            if (v.w > 0.f) y = make_float3(v.x / v.w, v.y / v.w, v.z / v.w);
            break;
        }
    }
    R.qry_out[3 * i] = y.x;
    R.qry_out[3 * i + 1] = y.y;
    R.qry_out[3 * i + 2] = y.z;
}

cudaError_t hash_cache_update(const RenderDev &R, uint32_t n_rec, cudaStream_t st)
{
    if (n_rec == 0) return cudaSuccess;
    k_hc_update<<<blocks_for(n_rec, 256), 256, 0, st>>>(R, n_rec);
    return cudaGetLastError();
}

cudaError_t render_wave(const RenderDev &R, uint32_t n_paths, uint64_t wave_begin, cudaStream_t st,
                        uint32_t *launches, const MlpDev *cache, uint32_t block)
{
    const uint32_t T = block;
    cudaError_t e;
    if ((e = cudaMemsetAsync(R.count, 0, 2 * sizeof(uint32_t), st)) != cudaSuccess) return e;
    if (R.cache_depth) {
        if ((e = cudaMemsetAsync(R.train_count, 0, sizeof(uint32_t), st)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(R.qry_count, 0, sizeof(uint32_t), st)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(R.rec_of, 0xff, sizeof(uint32_t) * R.train_cap * (R.depth_max + 1), st)) !=
            cudaSuccess)
            return e;
    }
    k_camera<<<blocks_for(n_paths, 128), 128, 0, st>>>(R, n_paths, wave_begin);  // also sets count[0]
    uint32_t n_launch = 1;
    int cur = 0;
    // with short training tails every path has stopped by the tail vertex
    const uint32_t tail = R.cache_depth + R.train_tail;
    const uint32_t last = (R.cache_depth && R.train_tail && cache) ? std::min(R.depth_max, tail) : R.depth_max;
    // persistent traversal: the shadow rays of depth d and the extension rays
    // of depth d + 1 go in one launch (k_trace_mixed)
    const bool merge = R.persistent && !R.stats;
    bool traced = false;  // this depth's extension rays were traced with the previous depth's shadow rays
    for (uint32_t depth = 0; depth <= last; depth++) {
        if (!traced) {
            if ((e = cudaMemsetAsync(R.count + (cur ^ 1), 0, sizeof(uint32_t), st)) != cudaSuccess) return e;
            if ((e = cudaMemsetAsync(R.sh_count, 0, sizeof(uint32_t), st)) != cudaSuccess) return e;
            if (R.stats) {
                k_extend<true><<<blocks_for(n_paths, T), T, 0, st>>>(R, cur);
            } else if (!R.persistent) {
                k_extend<false><<<blocks_for(n_paths, T), T, 0, st>>>(R, cur);
            } else {
                if ((e = cudaMemsetAsync(R.count + 6, 0, sizeof(uint32_t), st)) != cudaSuccess) return e;
                k_extend_dyn<<<persistent_blocks(n_paths), kStackColumns, 0, st>>>(R, cur, R.count + 6);
            }
            n_launch++;
        }
        traced = false;
        k_shade<<<blocks_for(n_paths, T), T, 0, st>>>(R, cur, depth, wave_begin);
        n_launch++;
        if (R.cache_depth && cache && (depth == R.cache_depth || (R.train_tail && depth == tail))) {
            if (R.hc_keys)
                k_hc_query<<<blocks_for(n_paths, 256), 256, 0, st>>>(R, R.capacity);
            else if ((e = mlp_infer(*cache, R.qry_feat, n_paths, R.qry_out, st, R.qry_count)) != cudaSuccess)
                return e;
            k_cache_apply<<<blocks_for(n_paths, 128), 128, 0, st>>>(R);
            if ((e = cudaMemsetAsync(R.qry_count, 0, sizeof(uint32_t), st)) != cudaSuccess) return e;
            n_launch += 2;
        }
        if (depth < last && merge) {
            if ((e = cudaMemsetAsync(R.count + 6, 0, sizeof(uint32_t), st)) != cudaSuccess) return e;
            k_trace_mixed<<<persistent_blocks((uint64_t)n_paths + R.sh_capacity), kStackColumns, 0, st>>>(
                R, cur ^ 1, R.count + 6);
            // the queues the next k_shade appends to, now that they are consumed
            if ((e = cudaMemsetAsync(R.count + cur, 0, sizeof(uint32_t), st)) != cudaSuccess) return e;
            if ((e = cudaMemsetAsync(R.sh_count, 0, sizeof(uint32_t), st)) != cudaSuccess) return e;
            n_launch++;
            traced = true;
        } else if (depth < last) {
            if (R.stats) {
                k_shadow<true><<<blocks_for((uint64_t)R.sh_capacity, T), T, 0, st>>>(R);
            } else if (!R.persistent) {
                k_shadow<false><<<blocks_for((uint64_t)R.sh_capacity, T), T, 0, st>>>(R);
            } else {
                if ((e = cudaMemsetAsync(R.count + 7, 0, sizeof(uint32_t), st)) != cudaSuccess) return e;
                k_shadow_dyn<<<persistent_blocks(R.sh_capacity), kStackColumns, 0, st>>>(R, R.count + 7);
            }
            n_launch++;
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        cur ^= 1;
    }
    if (launches) *launches += n_launch;
    return cudaSuccess;
}

cudaError_t render_persistent(const RenderDev &R, uint64_t total, unsigned long long *next, uint32_t *launches,
                              cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(next, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_render_persistent, kPersistThreads, 0)) != cudaSuccess)
        return e;
    const uint64_t want = (total + 127) / 128;
    const uint64_t cap = (uint64_t)current_sm_count() * (uint64_t)(per_sm > 0 ? per_sm : 1);
    const uint32_t blocks = (uint32_t)(want < cap ? (want > 0 ? want : 1) : cap);
    k_render_persistent<<<blocks, kPersistThreads, 0, st>>>(R, total, next);
    if (launches) *launches += 1;
    return cudaGetLastError();
}

cudaError_t render_resolve(const float4 *accum, uint32_t wh, float scale, float *out, cudaStream_t st)
{
    k_resolve<<<blocks_for(wh, 256), 256, 0, st>>>(accum, wh, scale, out);
    return cudaGetLastError();
}

}  // namespace ilg
