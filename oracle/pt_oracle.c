/* CPU restatement of the path-tracing bounce loop - TEST INFRASTRUCTURE ONLY.
 *
 * Restates the reference's PathIntegrator::Radiance
 * (Core/Integrator/PathIntegrator.cpp:44-367) driven per pixel and sample as
 * BaseRenderer::RenderRegion does (Core/Renderer/BaseRenderer.cpp:62-169):
 *   camera ray          PerspectiveCamera::GetRay      Core/Camera/PerspectiveCamera.cpp:44-60
 *   box filter          sample - 0.5                    Core/Filter/BoxFilter.cpp:20-28
 *   emission            depth 0 only, one-sided         PathIntegrator.cpp:126-128,
 *                                                       DiffuseAreaLight.cpp:47-50
 *   NEE                 every light but the hit one     Integrator.cpp:114-185
 *   light sample        Quad::SamplePoint patch, pdf = 1/area
 *                                                       Quad.cpp:144-153, DiffuseAreaLight.cpp:52-69
 *   visibility          segment [eps, 1 - eps]          Visibility.cpp:50-53
 *   Lambertian          cosine hemisphere, flip to wo   LambertianBxDF.cpp:27-55, BSDF.cpp:141-234
 *   throughput, RR      beta *= f |cos| / pdf; q = min(0.5, lum) after depth 3
 *                                                       PathIntegrator.cpp:164-177
 *   spawn               p + n_g * eps                   PathIntegrator.cpp:184-187
 * with the device's counter-based random numbers (same hash, same
 * dimensions), so that a GPU render and this one follow the same paths and
 * differ only where float rounding flips a decision. GGX and the constant
 * sky are this project's own (the reference has neither) and are restated
 * here from the same formulas as the device code.
 *
 * Test infrastructure: only tests/ and bench.py's CPU-baseline legs call it. */
#define _POSIX_C_SOURCE 199309L /* clock_gettime under -std=c11 */
#include "ilg_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <time.h>
#include <stdlib.h>
#include <string.h>

/* provided by ilg_oracle.c */
void *orc_bvh_create(const float *pos, uint32_t nverts, const uint32_t *idx, uint32_t ntris);
void orc_bvh_destroy(void *h);
int32_t orc_bvh_closest1(void *h, const float o[3], const float d[3], float rmin, float rmax, float *t);
int orc_bvh_any1(void *h, const float o[3], const float d[3], float rmin, float rmax);

typedef struct { float x, y, z; } f3;
static f3 mk(float x, float y, float z) { f3 r = {x, y, z}; return r; }
static f3 add(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static f3 sub(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static f3 mul(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static f3 mulv(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static f3 cross(f3 a, f3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static f3 nrm(f3 a) { return mul(a, 1.0f / sqrtf(dot(a, a))); }
static int black(f3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
static f3 ld(const float *p) { return mk(p[0], p[1], p[2]); }

static uint64_t mix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
static float rnd(uint64_t key, uint32_t dim)
{
    return (float)(uint32_t)(mix64(key + (uint64_t)dim * 0xD1B54A32D192ED03ull) >> 40) * 0x1p-24f;
}
static uint64_t path_key(uint32_t seed, uint64_t g) { return mix64(g ^ ((uint64_t)seed * 0xA24BAED4963EE407ull)); }
#define DIM_CAM 0xFFFFFF00u
static uint32_t dim_of(uint32_t depth, uint32_t k) { return depth * 32u + k; }

static void onb(f3 w, f3 *u, f3 *v)
{
    if (fabsf(w.x) > fabsf(w.y)) {
        float inv = 1.f / sqrtf(w.x * w.x + w.z * w.z);
        *v = mk(-w.z * inv, 0.f, w.x * inv);
    } else {
        float inv = 1.f / sqrtf(w.y * w.y + w.z * w.z);
        *v = mk(0.f, w.z * inv, -w.y * inv);
    }
    *u = cross(w, *v);
}

/* GGX conductor: Trowbridge-Reitz D, separable Smith G, Schlick F, VNDF
 * sampling (Heitz 2018) - the device's formulas. */
static float ggx_d(f3 h, float a)
{
    float a2 = a * a, t = h.x * h.x / a2 + h.y * h.y / a2 + h.z * h.z;
    return 1.f / (3.14159265358979f * a2 * t * t);
}
static float ggx_g1(f3 w, float a)
{
    float z2 = w.z * w.z;
    if (z2 <= 0.f) return 0.f;
    float t2 = (w.x * w.x + w.y * w.y) * a * a / z2;
    return 2.f / (1.f + sqrtf(1.f + t2));
}
static f3 schlick(f3 f0, float c)
{
    float m = 1.f - fminf(fmaxf(c, 0.f), 1.f), m5 = m * m * m * m * m;
    return add(f0, mul(sub(mk(1, 1, 1), f0), m5));
}
static f3 ggx_f(f3 wo, f3 wi, f3 f0, float a)
{
    if (wo.z <= 0.f || wi.z <= 0.f) return mk(0, 0, 0);
    f3 h = nrm(add(wo, wi));
    float g = ggx_g1(wo, a) * ggx_g1(wi, a);
    return mul(schlick(f0, dot(wi, h)), ggx_d(h, a) * g / (4.f * wo.z * wi.z));
}
static float ggx_pdf(f3 wo, f3 wi, float a)
{
    if (wo.z <= 0.f || wi.z <= 0.f) return 0.f;
    f3 h = nrm(add(wo, wi));
    return ggx_g1(wo, a) * fmaxf(dot(wo, h), 0.f) * ggx_d(h, a) / wo.z / (4.f * dot(wo, h));
}
static f3 ggx_sample(f3 wo, float a, float u1, float u2)
{
    f3 vh = nrm(mk(a * wo.x, a * wo.y, wo.z));
    float lensq = vh.x * vh.x + vh.y * vh.y;
    f3 t1 = lensq > 0.f ? mul(mk(-vh.y, vh.x, 0.f), 1.f / sqrtf(lensq)) : mk(1, 0, 0);
    f3 t2 = cross(vh, t1);
    float r = sqrtf(u1), ang = 6.28318530717958647692f * u2;
    float p1 = r * cosf(ang), p2 = r * sinf(ang), sh = 0.5f * (1.f + vh.z);
    p2 = (1.f - sh) * sqrtf(fmaxf(0.f, 1.f - p1 * p1)) + sh * p2;
    f3 nh = add(add(mul(t1, p1), mul(t2, p2)), mul(vh, sqrtf(fmaxf(0.f, 1.f - p1 * p1 - p2 * p2))));
    f3 h = nrm(mk(a * nh.x, a * nh.y, fmaxf(0.f, nh.z)));
    return sub(mul(h, 2.f * dot(wo, h)), wo);
}

typedef struct {
    const float *pos;
    const uint32_t *idx;
    const uint32_t *mat_ids;
    const orc_material *mats;
    uint32_t nmats;
    const orc_quad_light *lights;
    uint32_t nlights;
    f3 ln[8];
    float larea[8];
    int32_t light_of_tri_first[8];
    void *bvh;
    f3 centre, corner, across, up;
    uint32_t W, H, spp, max_depth, seed;
    float eps;
    f3 sky;
    float *out;
    int next_row;
    pthread_mutex_t lock;
} pt_ctx;

static f3 bsdf_f(const orc_material *m, f3 wo, f3 wi)
{
    if (m->kind == 1u) return ggx_f(wo, wi, ld(m->f0), m->alpha);
    if (m->kind == 0u && wi.z > 0.f) return mul(ld(m->albedo), 0.318309886183790671538f);
    return mk(0, 0, 0);  /* mirror, glass: SpecularReflection / SpecularTransmission::F are 0 */
}

/* Mirror (kind 2): SpecularReflectionBxDF.cpp:26-33. Glass (kind 3): BSDF::SampleF
 * (BSDF.cpp:141-211) picks SpecularTransmission ((int)(w * 2) % 2 == 0, with the
 * transmittance in f0) or SpecularReflection (the reflectivity in albedo) and
 * halves the pdf; SpecularTransmissionBxDF.cpp:24-58 refracts by the index
 * ratio (alpha = eta_i / eta_t) with no Fresnel weight; total internal
 * reflection gives f = 0. Returns 1 when the sampled ray is transmitted. */
static int sample_specular(const orc_material *m, f3 wo, float w, f3 *wi, f3 *f, float *pdf)
{
    if (m->kind == 2u || (int)(w * 2.f) % 2 == 1) {
        *wi = mk(-wo.x, -wo.y, wo.z);
        *f = mul(ld(m->albedo), 1.f / fabsf(wi->z));
        *pdf = m->kind == 2u ? 1.f : 0.5f;
        return 0;
    }
    const int entering = wo.z > 0.f;
    const float eta = entering ? m->alpha : 1.f / m->alpha;
    const float sin_t2 = (1.f - wo.z * wo.z) * eta * eta;
    *pdf = 0.5f;
    if (sin_t2 > 1.f) {
        *wi = mk(0, 0, 0);
        *f = mk(0, 0, 0);
        return 0;
    }
    float cos_t = sqrtf(fmaxf(0.f, 1.f - sin_t2));
    if (entering) cos_t = -cos_t;
    *wi = mk(eta * -wo.x, eta * -wo.y, cos_t);
    *f = mul(ld(m->f0), 1.f / fabsf(cos_t));
    return 1;
}

static int light_of(const pt_ctx *c, int32_t tri)
{
    for (uint32_t l = 0; l < c->nlights; l++)
        if ((uint32_t)tri == c->lights[l].first_tri || (uint32_t)tri == c->lights[l].first_tri + 1u) return (int)l;
    return -1;
}

static f3 radiance(pt_ctx *c, uint32_t pixel, uint64_t sample)
{
    const uint32_t x = pixel % c->W, y = pixel / c->W;
    const uint64_t key = path_key(c->seed, sample * (uint64_t)(c->W * c->H) + pixel);
    const float rw = 1.f / c->W, rh = 1.f / c->H;
    const float xi1 = rnd(key, DIM_CAM) - 0.5f, xi2 = rnd(key, DIM_CAM + 1) - 0.5f;
    const float fx = x * rw + xi1 * rw, fy = y * rh + xi2 * rh;
    f3 target = add(add(c->corner, mul(c->across, fx)), mul(c->up, fy));
    f3 o = c->centre, d = nrm(sub(target, c->centre));
    float tmin = 0.f;
    f3 beta = mk(1, 1, 1), L = mk(0, 0, 0);
    int after_specular = 0;
    for (uint32_t depth = 0; depth <= c->max_depth; depth++) {
        float t;
        float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
        int32_t tri = orc_bvh_closest1(c->bvh, oo, dd, tmin, FLT_MAX, &t);
        if (tri < 0) {
            L = add(L, mulv(beta, c->sky));
            break;
        }
        if (depth == c->max_depth) break;
        const orc_material *m = &c->mats[c->mat_ids[tri] < c->nmats ? c->mat_ids[tri] : 0];
        const float *p0 = c->pos + 3 * c->idx[3 * tri], *p1 = c->pos + 3 * c->idx[3 * tri + 1],
                    *p2 = c->pos + 3 * c->idx[3 * tri + 2];
        f3 e1 = sub(ld(p1), ld(p0)), e2 = sub(ld(p2), ld(p0));
        f3 ng = nrm(cross(e1, e2));
        f3 p = mk(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
        f3 wo = mul(nrm(d), -1.f);
        f3 W = ng, U, V;
        onb(W, &U, &V);
        f3 wo_l = mk(dot(U, wo), dot(V, wo), dot(W, wo));
        int lid = light_of(c, tri);
        /* emission at depth 0 or after a specular bounce (PathIntegrator.cpp:126-128) */
        if ((depth == 0 || after_specular) && lid >= 0 && dot(W, wo) > 0.f)
            L = add(L, mulv(beta, ld(c->lights[lid].emit)));
        const int specular = m->kind >= 2u;
        for (uint32_t l = 0; l < c->nlights && !specular; l++) {
            if ((int)l == lid) continue;
            const orc_quad_light *ql = &c->lights[l];
            float u = rnd(key, dim_of(depth, 2 * l)), v = rnd(key, dim_of(depth, 2 * l + 1));
            f3 q0 = ld(ql->v[0]), q1 = ld(ql->v[1]), q2 = ld(ql->v[2]), q3 = ld(ql->v[3]);
            f3 P = add(add(add(q0, mul(sub(q2, q0), u)), mul(sub(q3, q2), v)), mul(add(sub(q0, q2), sub(q1, q3)), u * v));
            f3 win = sub(p, P);
            float dist2 = dot(win, win);
            win = nrm(win);
            float cl = fmaxf(0.f, dot(win, c->ln[l]));
            f3 Ls = mul(ld(ql->emit), cl * c->larea[l] / dist2);
            if (black(Ls)) continue;
            f3 wi = mul(win, -1.f);
            f3 wi_l = mk(dot(U, wi), dot(V, wi), dot(W, wi));
            f3 contrib = mulv(mul(mulv(beta, Ls), fmaxf(0.f, dot(wi, W))), bsdf_f(m, wo_l, wi_l));
            if (black(contrib)) continue;
            f3 seg = sub(P, p);
            float so[3] = {p.x, p.y, p.z}, sd[3] = {seg.x, seg.y, seg.z};
            if (!orc_bvh_any1(c->bvh, so, sd, c->eps, 1.f - c->eps)) L = add(L, contrib);
        }
        float u1 = rnd(key, dim_of(depth, 20)), u2 = rnd(key, dim_of(depth, 21));
        f3 wi_l, f;
        float pdf;
        int transmit = 0;
        if (specular) {
            transmit = sample_specular(m, wo_l, rnd(key, dim_of(depth, 22)), &wi_l, &f, &pdf);
        } else if (m->kind == 1u) {
            wi_l = ggx_sample(wo_l, m->alpha, u1, u2);
            pdf = ggx_pdf(wo_l, wi_l, m->alpha);
            f = ggx_f(wo_l, wi_l, ld(m->f0), m->alpha);
        } else {
            float r = sqrtf(u1), ang = 6.28318530717958647692f * u2;
            wi_l = mk(r * cosf(ang), r * sinf(ang), sqrtf(1.f - u1));
            if (wo_l.z < 0.f) wi_l.z = -wi_l.z;
            pdf = fabsf(wi_l.z) * 0.318309886183790671538f;
            f = bsdf_f(m, wo_l, wi_l);
        }
        if (black(f) || !(pdf > 0.f)) break;
        f3 wi = add(add(mul(U, wi_l.x), mul(V, wi_l.y)), mul(W, wi_l.z));
        beta = mul(mulv(beta, f), fabsf(dot(wi, W)) / pdf);
        if (depth > 3) {
            float q = fminf(0.5f, 0.212671f * beta.x + 0.715160f * beta.y + 0.072169f * beta.z);
            if (rnd(key, dim_of(depth, 23)) > q) break;
            beta = mul(beta, 1.f / q);
        }
        /* a transmitted ray starts below the surface (PathIntegrator.cpp:184-187) */
        o = add(p, mul(ng, transmit ? -c->eps : c->eps));
        d = wi;
        tmin = c->eps;
        after_specular = specular;
    }
    return L;
}

static void *pt_worker(void *arg)
{
    pt_ctx *c = (pt_ctx *)arg;
    for (;;) {
        pthread_mutex_lock(&c->lock);
        int row = c->next_row++;
        pthread_mutex_unlock(&c->lock);
        if (row >= (int)c->H) break;
        for (uint32_t x = 0; x < c->W; x++) {
            uint32_t pixel = (uint32_t)row * c->W + x;
            f3 acc = mk(0, 0, 0);
            for (uint32_t s = 0; s < c->spp; s++) acc = add(acc, radiance(c, pixel, s));
            c->out[3 * pixel] = acc.x / c->spp;
            c->out[3 * pixel + 1] = acc.y / c->spp;
            c->out[3 * pixel + 2] = acc.z / c->spp;
        }
    }
    return NULL;
}

/* Wall seconds of the last orc_render's paths (its tree build excluded). */
static double g_render_seconds;
double orc_last_render_seconds(void) { return g_render_seconds; }

static double now_seconds(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int orc_render(const float *pos, uint32_t nverts, const uint32_t *idx, uint32_t ntris, const uint32_t *mat_ids,
               const orc_material *mats, uint32_t nmats, const orc_quad_light *lights, uint32_t nlights,
               const float cam[11], uint32_t W, uint32_t H, uint32_t spp, uint32_t max_depth, float eps,
               uint32_t seed, const float sky[3], int nthreads, float *out)
{
    if (nlights > 8 || !W || !H || !spp) return 1;
    pt_ctx c;
    memset(&c, 0, sizeof(c));
    c.pos = pos; c.idx = idx; c.mat_ids = mat_ids; c.mats = mats; c.nmats = nmats;
    c.lights = lights; c.nlights = nlights;
    for (uint32_t l = 0; l < nlights; l++) {
        f3 p0 = ld(lights[l].v[0]), p1 = ld(lights[l].v[1]), p2 = ld(lights[l].v[2]), p3 = ld(lights[l].v[3]);
        f3 n0 = cross(sub(p2, p0), sub(p1, p0)), n1 = cross(sub(p3, p0), sub(p2, p0));
        c.larea[l] = 0.5f * sqrtf(dot(n0, n0)) + 0.5f * sqrtf(dot(n1, n1));
        c.ln[l] = nrm(n0);
    }
    /* camera: PerspectiveCamera + SetFieldOfView (Camera.cpp:30-44, Basis.cpp:28-44) */
    f3 eye = ld(cam), tgt = ld(cam + 3), up = ld(cam + 6);
    float fov = cam[9], aspect = cam[10];
    f3 w = nrm(nrm(sub(tgt, eye)));
    f3 v = nrm(up);
    v = sub(v, mul(w, dot(v, w)));
    if (dot(v, v) <= 1.1920929e-7f) {
        v = mk(w.z, w.x, w.y);
        v = nrm(cross(v, w));
        v = nrm(sub(v, mul(w, dot(v, w))));
    }
    f3 u = cross(v, w);
    float half = fov * (atanf(1.0f) / 45.0f) * 0.5f;
    float v1 = tanf(half), v0 = -v1, u0 = v0 * aspect, u1 = v1 * aspect;
    c.centre = eye;
    c.corner = add(add(add(eye, mul(u, u0)), mul(v, v0)), w);
    c.across = mul(u, u1 - u0);
    c.up = mul(v, v1 - v0);
    c.W = W; c.H = H; c.spp = spp; c.max_depth = max_depth; c.seed = seed; c.eps = eps;
    c.sky = sky ? ld(sky) : mk(0, 0, 0);
    c.out = out;
    c.bvh = orc_bvh_create(pos, nverts, idx, ntris);
    pthread_mutex_init(&c.lock, NULL);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    const double t0 = now_seconds();
    for (int i = 0; i < nthreads; i++) pthread_create(&th[i], NULL, pt_worker, &c);
    for (int i = 0; i < nthreads; i++) pthread_join(th[i], NULL);
    g_render_seconds = now_seconds() - t0;
    pthread_mutex_destroy(&c.lock);
    orc_bvh_destroy(c.bvh);
    return 0;
}
