// C ABI (include/ilg.h): context, scene upload, device build, batched queries.
#include "ilg.h"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>

#include "build.cuh"
#include "trace_api.cuh"
#include "ctx.cuh"

using namespace ilg;

namespace {

int fail(ilg_ctx *c, int code, const char *fmt, ...)
{
    if (c) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(c->err, sizeof(c->err), fmt, ap);
        va_end(ap);
    }
    return code;
}

}  // namespace

#define CK(call)                                                                                     \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess)                                                                       \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? ILG_ENOMEM : ILG_ECUDA, "%s: %s", #call, \
                        cudaGetErrorString(e_));                                                     \
    } while (0)

extern "C" {

int ilg_create(ilg_ctx **out, const ilg_opts *opts)
{
    if (!out) return ILG_EINVAL;
    *out = nullptr;
    int dev = opts ? opts->device : 0;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return ILG_ECUDA;
    if (dev < 0 || dev >= count) return ILG_EINVAL;
    ilg_ctx *ctx = new (std::nothrow) ilg_ctx();
    if (!ctx) return ILG_ENOMEM;
    ctx->device = dev;
    if (cudaSetDevice(dev) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
        ctx->derr.reserve(4) != cudaSuccess || ctx->dstats.reserve(2) != cudaSuccess) {
        delete ctx;
        return ILG_ECUDA;
    }
    cudaMemsetAsync(ctx->derr.ptr, 0, 4 * sizeof(uint32_t), ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    *out = ctx;
    return ILG_OK;
}

int ilg_destroy(ilg_ctx *ctx)
{
    if (!ctx) return ILG_EINVAL;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->release_all();
    cudaEventDestroy(ctx->ev0);
    cudaEventDestroy(ctx->ev1);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return ILG_OK;
}

const char *ilg_last_error(const ilg_ctx *ctx) { return ctx ? ctx->err : "null context"; }

void *ilg_stream(ilg_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int ilg_sync(ilg_ctx *ctx)
{
    if (!ctx) return ILG_EINVAL;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    return ctx->check_device_error();
}

int ilg_set_mesh(ilg_ctx *ctx, const float *pos_xyz, uint32_t n_verts, const uint32_t *idx, uint32_t n_tris,
                 const uint32_t *mat_ids)
{
    if (!ctx) return ILG_EINVAL;
    if (!pos_xyz || !idx || n_verts == 0 || n_tris == 0)
        return fail(ctx, ILG_EINVAL, "ilg_set_mesh: empty or null mesh");
    if (n_tris > (1u << 30)) return fail(ctx, ILG_EINVAL, "ilg_set_mesh: %u triangles exceed 2^30", n_tris);
    for (uint64_t i = 0; i < 3ull * n_tris; i++)
        if (idx[i] >= n_verts) return fail(ctx, ILG_EINVAL, "ilg_set_mesh: index %u out of range at %llu", idx[i], (unsigned long long)i);
    float maxabs = 0.f;
    for (uint64_t i = 0; i < 3ull * n_verts; i++) {
        float a = fabsf(pos_xyz[i]);
        if (!(a <= 3.0e38f)) return fail(ctx, ILG_EINVAL, "ilg_set_mesh: non-finite position at %llu", (unsigned long long)i);
        maxabs = std::max(maxabs, a);
    }
    CK(cudaSetDevice(ctx->device));
    CK(ctx->pos.reserve(3ull * n_verts));
    CK(ctx->idx.reserve(3ull * n_tris));
    CK(cudaMemcpyAsync(ctx->pos.ptr, pos_xyz, 12ull * n_verts, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->idx.ptr, idx, 12ull * n_tris, cudaMemcpyHostToDevice, ctx->stream));
    if (mat_ids) {
        CK(ctx->mat.reserve(n_tris));
        CK(cudaMemcpyAsync(ctx->mat.ptr, mat_ids, 4ull * n_tris, cudaMemcpyHostToDevice, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->n_verts = n_verts;
    ctx->n_tris = n_tris;
    ctx->has_mat = mat_ids != nullptr;
    ctx->max_abs = maxabs;
    ctx->built = false;
    return ILG_OK;
}

int ilg_build(ilg_ctx *ctx)
{
    if (!ctx) return ILG_EINVAL;
    if (ctx->n_tris == 0) return fail(ctx, ILG_ESTATE, "ilg_build: no mesh set");
    CK(cudaSetDevice(ctx->device));
    BuildResult res;
    res.min_step = std::max(ctx->max_abs * 0x1p-19f, 1e-30f);
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    int rc = bvh_build(ctx->bb, ctx->pos.ptr, ctx->n_verts, ctx->idx.ptr, ctx->n_tris, ctx->stream, res, ctx->err,
                       sizeof(ctx->err));
    if (rc) return rc;
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    CK(cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->bb.release_scratch();
    ctx->stats.n_tris = ctx->n_tris;
    ctx->stats.n_nodes = res.n_nodes;
    ctx->stats.n_leaf_tris = res.n_tris;
    ctx->stats.max_depth = res.depth;
    ctx->stats.build_ms = ms;
    ctx->stats.node_bytes = (uint64_t)res.n_nodes * sizeof(Node8);
    ctx->stats.tri_bytes = (uint64_t)res.n_tris * sizeof(Tri);
    ctx->built = true;
    return ILG_OK;
}

int ilg_get_stats(const ilg_ctx *ctx, ilg_stats *out)
{
    if (!ctx || !out) return ILG_EINVAL;
    *out = ctx->stats;
    return ILG_OK;
}

int ilg_intersect(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n, int32_t *prim,
                  float *t, float *u, float *v, uint32_t flags)
{
    if (!ctx) return ILG_EINVAL;
    if (flags & ~ILG_DEVICE_PTRS) return fail(ctx, ILG_EINVAL, "ilg_intersect: unknown flags 0x%x", flags);
    if (!ctx->built) return fail(ctx, ILG_ESTATE, "ilg_intersect: scene not built");
    if (n == 0) return ILG_OK;
    if (!ray_o_tmin || !ray_d_tmax || !prim || !t || !u || !v) return fail(ctx, ILG_EINVAL, "ilg_intersect: null array");
    if (((uintptr_t)ray_o_tmin | (uintptr_t)ray_d_tmax) & 15u)
        return fail(ctx, ILG_EINVAL, "ilg_intersect: ray arrays must be 16-byte aligned");
    CK(cudaSetDevice(ctx->device));
    const SceneView sv = ctx->view();
    if (flags & ILG_DEVICE_PTRS) {
        CK(launch_closest(sv, (const float4 *)ray_o_tmin, (const float4 *)ray_d_tmax, n, prim, t, u, v, ctx->derr.ptr,
                          nullptr, ctx->stream));
        return ILG_OK;
    }
    CK(ctx->ro.reserve(n));
    CK(ctx->rd.reserve(n));
    CK(ctx->hprim.reserve(n));
    CK(ctx->ht.reserve(n));
    CK(ctx->hu.reserve(n));
    CK(ctx->hv.reserve(n));
    cudaStream_t st = ctx->stream;
    CK(cudaMemcpyAsync(ctx->ro.ptr, ray_o_tmin, 16ull * n, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->rd.ptr, ray_d_tmax, 16ull * n, cudaMemcpyHostToDevice, st));
    CK(launch_closest(sv, ctx->ro.ptr, ctx->rd.ptr, n, ctx->hprim.ptr, ctx->ht.ptr, ctx->hu.ptr, ctx->hv.ptr,
                      ctx->derr.ptr, nullptr, st));
    CK(cudaMemcpyAsync(prim, ctx->hprim.ptr, 4ull * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(t, ctx->ht.ptr, 4ull * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(u, ctx->hu.ptr, 4ull * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(v, ctx->hv.ptr, 4ull * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return ctx->check_device_error();
}

int ilg_intersect_counted(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n, int32_t *prim,
                          float *t, float *u, float *v, uint64_t counts[2], uint32_t flags)
{
    if (!ctx) return ILG_EINVAL;
    if (!counts) return fail(ctx, ILG_EINVAL, "ilg_intersect_counted: null counts");
    if (!(flags & ILG_DEVICE_PTRS)) return fail(ctx, ILG_EINVAL, "ilg_intersect_counted: needs ILG_DEVICE_PTRS");
    if (!ctx->built) return fail(ctx, ILG_ESTATE, "ilg_intersect_counted: scene not built");
    if (!ray_o_tmin || !ray_d_tmax || !prim || !t || !u || !v) return fail(ctx, ILG_EINVAL, "ilg_intersect_counted: null array");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemsetAsync(ctx->dstats.ptr, 0, 2 * sizeof(unsigned long long), ctx->stream));
    CK(launch_closest(ctx->view(), (const float4 *)ray_o_tmin, (const float4 *)ray_d_tmax, n, prim, t, u, v,
                      ctx->derr.ptr, ctx->dstats.ptr, ctx->stream));
    unsigned long long h[2];
    CK(cudaMemcpyAsync(h, ctx->dstats.ptr, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    counts[0] = h[0];
    counts[1] = h[1];
    return ctx->check_device_error();
}

int ilg_occluded(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n, uint8_t *occ,
                 uint32_t flags)
{
    if (!ctx) return ILG_EINVAL;
    if (flags & ~ILG_DEVICE_PTRS) return fail(ctx, ILG_EINVAL, "ilg_occluded: unknown flags 0x%x", flags);
    if (!ctx->built) return fail(ctx, ILG_ESTATE, "ilg_occluded: scene not built");
    if (n == 0) return ILG_OK;
    if (!ray_o_tmin || !ray_d_tmax || !occ) return fail(ctx, ILG_EINVAL, "ilg_occluded: null array");
    if (((uintptr_t)ray_o_tmin | (uintptr_t)ray_d_tmax) & 15u)
        return fail(ctx, ILG_EINVAL, "ilg_occluded: ray arrays must be 16-byte aligned");
    CK(cudaSetDevice(ctx->device));
    const SceneView sv = ctx->view();
    if (flags & ILG_DEVICE_PTRS) {
        CK(launch_any(sv, (const float4 *)ray_o_tmin, (const float4 *)ray_d_tmax, n, occ, ctx->derr.ptr, ctx->stream));
        return ILG_OK;
    }
    CK(ctx->ro.reserve(n));
    CK(ctx->rd.reserve(n));
    CK(ctx->hocc.reserve(n));
    cudaStream_t st = ctx->stream;
    CK(cudaMemcpyAsync(ctx->ro.ptr, ray_o_tmin, 16ull * n, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->rd.ptr, ray_d_tmax, 16ull * n, cudaMemcpyHostToDevice, st));
    CK(launch_any(sv, ctx->ro.ptr, ctx->rd.ptr, n, ctx->hocc.ptr, ctx->derr.ptr, st));
    CK(cudaMemcpyAsync(occ, ctx->hocc.ptr, n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return ctx->check_device_error();
}

}  // extern "C"
