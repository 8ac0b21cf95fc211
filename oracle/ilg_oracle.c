/* CPU oracle for the closest-hit / any-hit path - TEST INFRASTRUCTURE ONLY.
 * See ilg_oracle.h for the reference lines each function follows. Built with
 * -ffp-contract=off so each float operation rounds as the reference's does. */
#include "ilg_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define CROSS(dst, a, b)                      \
    dst[0] = a[1] * b[2] - a[2] * b[1];       \
    dst[1] = a[2] * b[0] - a[0] * b[2];       \
    dst[2] = a[0] * b[1] - a[1] * b[0];
#define DOT(a, b) (a[0] * b[0] + a[1] * b[1] + a[2] * b[2])
#define SUB(dst, a, b)    \
    dst[0] = a[0] - b[0]; \
    dst[1] = a[1] - b[1]; \
    dst[2] = a[2] - b[2];

typedef struct {
    float v0[3], e1[3], e2[3];
} otri;

static void make_tri(const float *pos, const uint32_t *idx, uint32_t t, otri *out)
{
    const float *p0 = pos + 3 * idx[3 * t], *p1 = pos + 3 * idx[3 * t + 1], *p2 = pos + 3 * idx[3 * t + 2];
    memcpy(out->v0, p0, 12);
    SUB(out->e1, p1, p0);
    SUB(out->e2, p2, p0);
}

/* IndexedTriangle::Intersects, Core/Shape/IndexedTriangle.cpp:92-128. */
static int shirley_tri(const otri *tr, const float o[3], const float d[3], float rmax,
                       float *t_out, float *b_out, float *g_out)
{
    float n[3], edge2[3], interm[3];
    CROSS(n, tr->e1, tr->e2);
    const float rcp = 1.0f / DOT(n, d);
    SUB(edge2, tr->v0, o);
    const float t = DOT(n, edge2) * rcp;
    if (t > rmax - 1e-5 || t < 1e-5) /* double comparisons, as written in the reference */
        return 0;
    CROSS(interm, d, edge2);
    const float beta = DOT(interm, tr->e2) * -rcp;
    if (beta < 0.0f) return 0;
    const float gamma = DOT(interm, tr->e1) * rcp;
    if (beta + gamma > 1.0f || gamma < 0.0f) return 0;
    /* A zero-area triangle gives n = 0 and t = 0 * inf = NaN, which passes
     * every comparison above in the reference and is then reported as a hit
     * whose distance poisons ray.Max; which rays meet it depends on the tree.
     * The oracle (like the device) rejects it. */
    if (t != t) return 0;
    *t_out = t;
    *b_out = beta;
    *g_out = gamma;
    return 1;
}

int orc_shirley(const float *pos, const uint32_t *idx, uint32_t tri, const float o[3], const float d[3],
                float tmax, float *t, float *beta, float *gamma)
{
    otri tr;
    make_tri(pos, idx, tri, &tr);
    return shirley_tri(&tr, o, d, tmax, t, beta, gamma);
}

void orc_intersect_brute(const float *pos, const uint32_t *idx, uint32_t ntris, const float *o4, const float *d4,
                         int64_t n, int32_t *prim, float *t, float *u, float *v)
{
    otri *tris = (otri *)malloc(sizeof(otri) * (ntris ? ntris : 1));
    for (uint32_t i = 0; i < ntris; i++) make_tri(pos, idx, i, &tris[i]);
    for (int64_t r = 0; r < n; r++) {
        const float *o = o4 + 4 * r, *d = d4 + 4 * r;
        float rmax = d[3], th, bh, gh;
        int32_t best = -1;
        float bt = INFINITY, bu = 0, bv = 0;
        for (uint32_t i = 0; i < ntris; i++) {
            if (shirley_tri(&tris[i], o, d, rmax, &th, &bh, &gh)) {
                best = (int32_t)i; bt = th; bu = bh; bv = gh;
                rmax = th < rmax ? th : rmax;
            }
        }
        prim[r] = best; t[r] = bt; u[r] = bu; v[r] = bv;
    }
    free(tris);
}

/* ---------------- watertight test (Woop, Benthin, Wald 2013) ----------------
 * Not in the reference: the restatement the device's ILG_WATERTIGHT mode
 * follows, operation for operation (shear into the ray's frame with the
 * largest direction component as z, 2D edge functions from the vertices,
 * double-precision recomputation of edge functions that are exactly zero),
 * with the reference's window t in [1e-5, Max - 1e-5]. */
typedef struct {
    int kx, ky, kz;
    float sx, sy, sz;
} oshear;

static oshear shear_of(const float d[3])
{
    oshear s;
    const float ax = fabsf(d[0]), ay = fabsf(d[1]), az = fabsf(d[2]);
    s.kz = ax >= ay ? (ax >= az ? 0 : 2) : (ay >= az ? 1 : 2);
    s.kx = s.kz == 2 ? 0 : s.kz + 1;
    s.ky = s.kx == 2 ? 0 : s.kx + 1;
    if (d[s.kz] < 0.f) {
        const int k = s.kx;
        s.kx = s.ky;
        s.ky = k;
    }
    s.sx = d[s.kx] / d[s.kz];
    s.sy = d[s.ky] / d[s.kz];
    s.sz = 1.0f / d[s.kz];
    return s;
}

static int watertight_tri(const float *p0, const float *p1, const float *p2, const float o[3], const oshear *sh,
                          float rmax, float *t_out, float *b_out, float *g_out)
{
    float A[3], B[3], C[3];
    SUB(A, p0, o);
    SUB(B, p1, o);
    SUB(C, p2, o);
    const float Ax = A[sh->kx] - sh->sx * A[sh->kz], Ay = A[sh->ky] - sh->sy * A[sh->kz];
    const float Bx = B[sh->kx] - sh->sx * B[sh->kz], By = B[sh->ky] - sh->sy * B[sh->kz];
    const float Cx = C[sh->kx] - sh->sx * C[sh->kz], Cy = C[sh->ky] - sh->sy * C[sh->kz];
    float U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
    if (U == 0.f || V == 0.f || W == 0.f) {
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return 0;
    const float det = U + V + W;
    if (det == 0.f) return 0;
    const float Az = sh->sz * A[sh->kz], Bz = sh->sz * B[sh->kz], Cz = sh->sz * C[sh->kz];
    const float T = U * Az + V * Bz + W * Cz;
    const float rcp = 1.0f / det;
    const float t = T * rcp;
    if (!(t <= rmax - 1e-5) || t < 1e-5) return 0; /* double comparisons; NaN rejected */
    *t_out = t;
    *b_out = V * rcp;
    *g_out = W * rcp;
    return 1;
}

void orc_watertight_brute(const float *pos, const uint32_t *idx, uint32_t ntris, const float *o4, const float *d4,
                          int64_t n, int32_t *prim, float *t, float *u, float *v, uint8_t *occ)
{
    for (int64_t r = 0; r < n; r++) {
        const float *o = o4 + 4 * r, *d = d4 + 4 * r;
        const oshear sh = shear_of(d);
        float rmax = d[3], th, bh, gh;
        int32_t best = -1;
        float bt = INFINITY, bu = 0, bv = 0;
        int any = 0;
        for (uint32_t i = 0; i < ntris; i++) {
            const float *p0 = pos + 3 * idx[3 * i], *p1 = pos + 3 * idx[3 * i + 1], *p2 = pos + 3 * idx[3 * i + 2];
            if (!any && watertight_tri(p0, p1, p2, o, &sh, d[3], &th, &bh, &gh)) any = 1;
            if (watertight_tri(p0, p1, p2, o, &sh, rmax, &th, &bh, &gh)) {
                best = (int32_t)i; bt = th; bu = bh; bv = gh;
                rmax = th < rmax ? th : rmax;
            }
        }
        prim[r] = best; t[r] = bt; u[r] = bu; v[r] = bv;
        if (occ) occ[r] = (uint8_t)any;
    }
}

/* ---------------- binary BVH (ours: median split, <= 4 triangles a leaf) --- */
typedef struct {
    float lo[3], hi[3];
    int32_t left;   /* internal: index of left child (right = left + 1); leaf: -1 */
    int32_t first;  /* leaf: first entry in order[] */
    int32_t count;  /* leaf: number of triangles */
} onode;

typedef struct {
    onode *nodes;
    int32_t nnodes;
    uint32_t *order;
    otri *tris;
    uint32_t ntris;
} obvh;

typedef struct {
    float *cent;
    float *blo, *bhi;
} build_ctx;

static int cmp_axis;
static const float *cmp_cent;
static int cmp_key(const void *a, const void *b)
{
    float ca = cmp_cent[3 * *(const uint32_t *)a + cmp_axis], cb = cmp_cent[3 * *(const uint32_t *)b + cmp_axis];
    if (ca < cb) return -1;
    if (ca > cb) return 1;
    uint32_t ia = *(const uint32_t *)a, ib = *(const uint32_t *)b;
    return ia < ib ? -1 : (ia > ib);
}

/* Total order of the median split: centroid on the axis, then index. */
static int key_less(const float *cent, int axis, uint32_t a, uint32_t b)
{
    float ca = cent[3 * a + axis], cb = cent[3 * b + axis];
    return ca < cb || (ca == cb && a < b);
}

/* Rearranges v[0..n) so that v[k] is the element a full sort by key_less
 * would put there, with every element before it smaller and every one after
 * it larger (quickselect, median-of-three pivots). The two sides hold the
 * same sets as after a full sort, which is all the split uses. */
static void select_kth(uint32_t *v, uint32_t n, uint32_t k, const float *cent, int axis)
{
    uint32_t lo = 0, hi = n - 1;
    while (hi > lo) {
        uint32_t mid = lo + (hi - lo) / 2;
        if (key_less(cent, axis, v[mid], v[lo])) { uint32_t t = v[mid]; v[mid] = v[lo]; v[lo] = t; }
        if (key_less(cent, axis, v[hi], v[lo])) { uint32_t t = v[hi]; v[hi] = v[lo]; v[lo] = t; }
        if (key_less(cent, axis, v[hi], v[mid])) { uint32_t t = v[hi]; v[hi] = v[mid]; v[mid] = t; }
        uint32_t pivot = v[mid];
        uint32_t i = lo, j = hi;
        while (i <= j) {
            while (key_less(cent, axis, v[i], pivot)) i++;
            while (key_less(cent, axis, pivot, v[j])) j--;
            if (i <= j) {
                uint32_t t = v[i]; v[i] = v[j]; v[j] = t;
                i++;
                if (j == 0) break;
                j--;
            }
        }
        if (k <= j) hi = j;
        else if (k >= i) lo = i;
        else return;
    }
}

/* Build with explicit sibling slots: children of node k live at (left, left+1). */
static void build_iter(obvh *b, build_ctx *c)
{
    typedef struct { int32_t node; uint32_t first, count; } item;
    item *stack = (item *)malloc(sizeof(item) * 256);
    int sp = 0;
    b->nnodes = 1;
    stack[sp++] = (item){0, 0, b->ntris};
    while (sp) {
        item it = stack[--sp];
        onode *nd = &b->nodes[it.node];
        for (int k = 0; k < 3; k++) { nd->lo[k] = FLT_MAX; nd->hi[k] = -FLT_MAX; }
        float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (uint32_t i = it.first; i < it.first + it.count; i++) {
            uint32_t t = b->order[i];
            for (int k = 0; k < 3; k++) {
                if (c->blo[3 * t + k] < nd->lo[k]) nd->lo[k] = c->blo[3 * t + k];
                if (c->bhi[3 * t + k] > nd->hi[k]) nd->hi[k] = c->bhi[3 * t + k];
                if (c->cent[3 * t + k] < clo[k]) clo[k] = c->cent[3 * t + k];
                if (c->cent[3 * t + k] > chi[k]) chi[k] = c->cent[3 * t + k];
            }
        }
        if (it.count <= 4) {
            nd->left = -1; nd->first = (int32_t)it.first; nd->count = (int32_t)it.count;
            continue;
        }
        int axis = 0;
        for (int k = 1; k < 3; k++) if (chi[k] - clo[k] > chi[axis] - clo[axis]) axis = k;
        uint32_t half = it.count / 2;
        /* the median split of a full sort by (centroid on the axis, index);
         * a child that becomes a leaf keeps the sorted order, as the leaf's
         * triangle order decides which of two equal hits is tested first */
        select_kth(b->order + it.first, it.count, half, c->cent, axis);
        cmp_axis = axis;
        cmp_cent = c->cent;
        if (half <= 4) qsort(b->order + it.first, half, sizeof(uint32_t), cmp_key);
        if (it.count - half <= 4) qsort(b->order + it.first + half, it.count - half, sizeof(uint32_t), cmp_key);
        int32_t l = b->nnodes;
        b->nnodes += 2;
        nd->left = l; nd->first = 0; nd->count = 0;
        stack[sp++] = (item){l, it.first, half};
        stack[sp++] = (item){l + 1, it.first + half, it.count - half};
    }
    free(stack);
}

void *orc_bvh_create(const float *pos, uint32_t nverts, const uint32_t *idx, uint32_t ntris)
{
    (void)nverts;
    obvh *b = (obvh *)calloc(1, sizeof(obvh));
    b->ntris = ntris;
    b->tris = (otri *)malloc(sizeof(otri) * (ntris ? ntris : 1));
    b->order = (uint32_t *)malloc(sizeof(uint32_t) * (ntris ? ntris : 1));
    b->nodes = (onode *)calloc(2 * (size_t)(ntris ? ntris : 1) + 1, sizeof(onode));
    build_ctx c;
    c.cent = (float *)malloc(12 * (size_t)(ntris ? ntris : 1));
    c.blo = (float *)malloc(12 * (size_t)(ntris ? ntris : 1));
    c.bhi = (float *)malloc(12 * (size_t)(ntris ? ntris : 1));
    for (uint32_t t = 0; t < ntris; t++) {
        make_tri(pos, idx, t, &b->tris[t]);
        b->order[t] = t;
        for (int k = 0; k < 3; k++) {
            float a = pos[3 * idx[3 * t] + k], bb = pos[3 * idx[3 * t + 1] + k], cc = pos[3 * idx[3 * t + 2] + k];
            float lo = fminf(a, fminf(bb, cc)), hi = fmaxf(a, fmaxf(bb, cc));
            c.blo[3 * t + k] = lo;
            c.bhi[3 * t + k] = hi;
            c.cent[3 * t + k] = 0.5f * (lo + hi);
        }
    }
    if (ntris) build_iter(b, &c);
    free(c.cent); free(c.blo); free(c.bhi);
    return b;
}

void orc_bvh_destroy(void *h)
{
    obvh *b = (obvh *)h;
    free(b->nodes); free(b->order); free(b->tris); free(b);
}

/* Slab test in the reference's form (BoundingBox.cpp:215-238), evaluated in
 * double so that float rounding never culls a box the triangle test would
 * hit: the oracle must not lose hits to its own tree. */
static int slab(const onode *nd, const float o[3], const double inv[3], double rmin, double rmax, double *tnear)
{
    double lo = -INFINITY, hi = INFINITY;
    for (int k = 0; k < 3; k++) {
        double a = ((double)nd->lo[k] - o[k]) * inv[k], b = ((double)nd->hi[k] - o[k]) * inv[k];
        if (isnan(a)) a = -INFINITY;
        if (isnan(b)) b = INFINITY;
        double mn = a < b ? a : b, mx = a < b ? b : a;
        if (mn > lo) lo = mn;
        if (mx < hi) hi = mx;
    }
    double pad = 1e-6 * (fabs(hi) + 1e-6);
    hi += pad;
    lo -= pad;
    if (lo > rmax || hi < rmin) return 0;
    *tnear = lo;
    return hi >= 0.0 && hi >= lo;
}

typedef struct {
    obvh *b;
    const float *o4, *d4;
    int64_t begin, end;
    int32_t *prim;
    float *t, *u, *v;
    uint8_t *occ;
    uint64_t visits, tests;
} job;

/* Closest hit (returns triangle index or -1) of one ray on the oracle BVH. */
static int32_t bvh_closest1(obvh *b, const float o[3], const float d[3], float rmin, float rmax0, float *t_out,
                            float *u_out, float *v_out, uint64_t *visits, uint64_t *tests)
{
    int32_t stack[128];
    double inv[3] = {1.0 / d[0], 1.0 / d[1], 1.0 / d[2]};
    float rmax = rmax0;
    int32_t best = -1;
    float bt = INFINITY, bu = 0, bv = 0;
    int sp = 0;
    if (b->ntris) stack[sp++] = 0;
    while (sp) {
        const onode *nd = &b->nodes[stack[--sp]];
        double tn;
        if (visits) (*visits)++;
        if (!slab(nd, o, inv, rmin, rmax, &tn)) continue;
        if (nd->left < 0) {
            for (int32_t i = nd->first; i < nd->first + nd->count; i++) {
                uint32_t tri = b->order[i];
                float th, bh, gh;
                if (tests) (*tests)++;
                if (shirley_tri(&b->tris[tri], o, d, rmax, &th, &bh, &gh)) {
                    best = (int32_t)tri; bt = th; bu = bh; bv = gh;
                    rmax = th < rmax ? th : rmax;
                }
            }
        } else {
            if (sp + 2 > 128) abort();
            stack[sp++] = nd->left + 1;
            stack[sp++] = nd->left;
        }
    }
    *t_out = bt; *u_out = bu; *v_out = bv;
    return best;
}

static int bvh_any1(obvh *b, const float o[3], const float d[3], float rmin, float rmax)
{
    int32_t stack[128];
    double inv[3] = {1.0 / d[0], 1.0 / d[1], 1.0 / d[2]};
    int sp = 0;
    if (b->ntris) stack[sp++] = 0;
    while (sp) {
        const onode *nd = &b->nodes[stack[--sp]];
        double tn;
        if (!slab(nd, o, inv, rmin, rmax, &tn)) continue;
        if (nd->left < 0) {
            for (int32_t i = nd->first; i < nd->first + nd->count; i++) {
                float th, bh, gh;
                if (shirley_tri(&b->tris[b->order[i]], o, d, rmax, &th, &bh, &gh)) return 1;
            }
        } else {
            if (sp + 2 > 128) abort();
            stack[sp++] = nd->left + 1;
            stack[sp++] = nd->left;
        }
    }
    return 0;
}

static void trace_range(job *j)
{
    for (int64_t r = j->begin; r < j->end; r++) {
        const float *o = j->o4 + 4 * r, *d = j->d4 + 4 * r;
        if (j->occ) {
            j->occ[r] = (uint8_t)bvh_any1(j->b, o, d, o[3], d[3]);
        } else {
            float t, u, v;
            int32_t p = bvh_closest1(j->b, o, d, o[3], d[3], &t, &u, &v, &j->visits, &j->tests);
            j->prim[r] = p; j->t[r] = t; j->u[r] = u; j->v[r] = v;
        }
    }
}

static void *trace_thread(void *arg) { trace_range((job *)arg); return NULL; }

static void run_jobs(obvh *b, const float *o4, const float *d4, int64_t n, int32_t *prim, float *t, float *u,
                     float *v, uint8_t *occ, int nthreads, uint64_t *stats)
{
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    job jobs[256];
    pthread_t th[256];
    int64_t chunk = (n + nthreads - 1) / nthreads;
    int used = 0;
    for (int i = 0; i < nthreads; i++) {
        int64_t s = i * chunk, e = s + chunk < n ? s + chunk : n;
        if (s >= e) break;
        jobs[i] = (job){b, o4, d4, s, e, prim, t, u, v, occ, 0, 0};
        used++;
    }
    if (used <= 1) {
        if (used) trace_range(&jobs[0]);
    } else {
        for (int i = 0; i < used; i++) pthread_create(&th[i], NULL, trace_thread, &jobs[i]);
        for (int i = 0; i < used; i++) pthread_join(th[i], NULL);
    }
    if (stats) {
        stats[0] = stats[1] = 0;
        for (int i = 0; i < used; i++) { stats[0] += jobs[i].visits; stats[1] += jobs[i].tests; }
    }
}

void orc_bvh_intersect(void *h, const float *o4, const float *d4, int64_t n, int32_t *prim, float *t, float *u,
                       float *v, int nthreads, uint64_t *stats)
{
    run_jobs((obvh *)h, o4, d4, n, prim, t, u, v, NULL, nthreads, stats);
}

void orc_bvh_occluded(void *h, const float *o4, const float *d4, int64_t n, uint8_t *occ, int nthreads)
{
    run_jobs((obvh *)h, o4, d4, n, NULL, NULL, NULL, NULL, occ, nthreads, NULL);
}

int32_t orc_bvh_closest1(void *h, const float o[3], const float d[3], float rmin, float rmax, float *t)
{
    float u, v;
    return bvh_closest1((obvh *)h, o, d, rmin, rmax, t, &u, &v, NULL, NULL);
}

int orc_bvh_any1(void *h, const float o[3], const float d[3], float rmin, float rmax)
{
    return bvh_any1((obvh *)h, o, d, rmin, rmax);
}
