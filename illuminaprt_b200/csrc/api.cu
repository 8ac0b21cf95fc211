// C ABI (include/ilg.h): context, scene upload, device build, batched queries.
#include "ilg.h"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "build.cuh"
#include "trace_api.cuh"
#include "ctx.cuh"
#include "hostpool.h"
#include "render.cuh"

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

#define CK2(c, call)                                                                                 \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess)                                                                       \
            return fail(c, e_ == cudaErrorMemoryAllocation ? ILG_ENOMEM : ILG_ECUDA, "%s: %s", #call,   \
                        cudaGetErrorString(e_));                                                     \
    } while (0)

namespace {

// The watertight test reads each triangle record's own vertices; they are
// copied out of the uploaded mesh once per build, on first use.
int ensure_raw_tris(ilg_ctx *ctx)
{
    if (ctx->raw_ready) return ILG_OK;
    const uint32_t n = ctx->stats.n_tris;
    CK(ctx->raw_tris.reserve(3ull * n));
    CK(build_raw_tris(ctx->bb.prim_of, ctx->idx.ptr, ctx->pos.ptr, n, ctx->raw_tris.ptr, ctx->stream));
    ctx->raw_ready = true;
    return ILG_OK;
}

// Whether p is host memory the device cannot reach directly (not
// page-locked): copies from it go through a staging buffer.
bool pageable(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

// host copies of pageable queries: up to 16 parts (the calling thread and
// the context's pool), 1 MB a part at least
constexpr unsigned kCopyParts = 16u;

void pool_copy_ctx(ilg_ctx *ctx, const CopySeg *seg, int nseg)
{
    if (!ctx->host_pool) ctx->host_pool = new (std::nothrow) HostPool();
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    if (ctx->host_pool) {
        pool_copy(*ctx->host_pool, seg, nseg, std::min(kCopyParts, hw));
    } else {
        for (int i = 0; i < nseg; i++) memcpy(seg[i].dst, seg[i].src, seg[i].bytes);
    }
}

// Closest hit (occ == nullptr) or any hit of rays in pageable host memory:
// chunks of rays go through three page-locked slots owned by the context,
// each with its own stream and device buffers. For chunk c the host waits
// for the slot's previous chunk (c - 3), then copies that chunk's hits out
// and chunk c's rays in as one job over the host threads, and queues chunk
// c's upload, traversal and download on the slot's stream; the device works
// on the other slots' chunks meanwhile.
constexpr uint32_t kPinSlots = 3u;

int query_host_pageable_run(ilg_ctx *ctx, const float *o4, const float *d4, uint32_t n, int32_t *prim, float *t,
                            float *u, float *v, uint8_t *occ, bool wt)
{
    const bool any = occ != nullptr;
    constexpr uint32_t kChunk = 1u << 19;
    const size_t in_bytes = 32ull * kChunk;
    const size_t slot_bytes = in_bytes + 16ull * kChunk;
    if (!ctx->pin_buf) CK(cudaHostAlloc(&ctx->pin_buf, kPinSlots * slot_bytes, cudaHostAllocDefault));
    for (uint32_t k = 0; k < kPinSlots; k++)
        if (!ctx->pin_ev[k]) CK(cudaEventCreateWithFlags(&ctx->pin_ev[k], cudaEventDisableTiming));
    // chunks of 512 K rays (the slots' size), or of an eighth of the batch,
    // 256 K rays at least, when that is smaller: short batches then still
    // run in enough chunks to overlap host copies and device work
    const uint32_t chunk = (uint32_t)std::min<uint64_t>(kChunk, std::max<uint64_t>(1u << 18, ((n + 7ull) / 8u + 127u) & ~127ull));
    const uint32_t m = std::min(n, chunk);
    CK(ctx->ro.reserve(kPinSlots * (size_t)m));
    CK(ctx->rd.reserve(kPinSlots * (size_t)m));
    if (any) {
        CK(ctx->hocc.reserve(kPinSlots * (size_t)m));
    } else {
        CK(ctx->hprim.reserve(kPinSlots * (size_t)m));
        CK(ctx->ht.reserve(kPinSlots * (size_t)m));
        CK(ctx->hu.reserve(kPinSlots * (size_t)m));
        CK(ctx->hv.reserve(kPinSlots * (size_t)m));
    }
    const SceneView sv = ctx->view();
    const uint32_t chunks = (uint32_t)((n + (uint64_t)chunk - 1) / chunk);
    cudaStream_t ss[kPinSlots] = {ctx->stream, ctx->stream, ctx->stream};
    if (chunks > 1) {
        for (int k = 0; k < 2; k++)
            if (!ctx->side[k]) CK(cudaStreamCreateWithFlags(&ctx->side[k], cudaStreamNonBlocking));
        if (!ctx->side_ev[2]) CK(cudaEventCreateWithFlags(&ctx->side_ev[2], cudaEventDisableTiming));
        // the side streams start after everything already queued on the main one
        CK(cudaEventRecord(ctx->side_ev[2], ctx->stream));
        for (int k = 0; k < 2; k++) {
            CK(cudaStreamWaitEvent(ctx->side[k], ctx->side_ev[2], 0));
            ss[1 + k] = ctx->side[k];
        }
    }
    auto slot_of = [&](uint32_t c) { return (unsigned char *)ctx->pin_buf + (c % kPinSlots) * slot_bytes; };
    // the copies from chunk c's slot to the caller's hit arrays
    auto out_segs = [&](uint32_t c, CopySeg *seg) -> int {
        const uint32_t off = c * chunk, len = std::min(chunk, n - off);
        const unsigned char *out = slot_of(c) + in_bytes;
        if (any) {
            seg[0] = {occ + off, out, len};
            return 1;
        }
        seg[0] = {prim + off, out, 4ull * len};
        seg[1] = {t + off, out + 4ull * kChunk, 4ull * len};
        seg[2] = {u + off, out + 8ull * kChunk, 4ull * len};
        seg[3] = {v + off, out + 12ull * kChunk, 4ull * len};
        return 4;
    };
    for (uint32_t c = 0; c < chunks; c++) {
        const uint32_t s = c % kPinSlots;
        cudaStream_t st = ss[s];
        const uint32_t off = c * chunk, len = std::min(chunk, n - off);
        unsigned char *slot = slot_of(c);
        CopySeg seg[6];
        int nseg = 0;
        if (c >= kPinSlots) {
            // the slot's previous chunk has left the device (its download was
            // the last of its work on this stream)
            CK(cudaEventSynchronize(ctx->pin_ev[s]));
            nseg = out_segs(c - kPinSlots, seg);
        }
        seg[nseg++] = {slot, o4 + 4ull * off, 16ull * len};
        seg[nseg++] = {slot + 16ull * kChunk, d4 + 4ull * off, 16ull * len};
        pool_copy_ctx(ctx, seg, nseg);
        float4 *dro = ctx->ro.ptr + (size_t)s * m, *drd = ctx->rd.ptr + (size_t)s * m;
        uint32_t *next = ctx->derr.ptr + 1 + s;  // ray counter of this stream's persistent kernels
        CK(cudaMemcpyAsync(dro, slot, 16ull * len, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(drd, slot + 16ull * kChunk, 16ull * len, cudaMemcpyHostToDevice, st));
        unsigned char *out = slot + in_bytes;
        if (any) {
            uint8_t *docc = ctx->hocc.ptr + (size_t)s * m;
            if (wt) CK(launch_any_wt(sv, ctx->raw_tris.ptr, dro, drd, len, docc, next, ctx->derr.ptr, st));
            else CK(launch_any_dyn(sv, dro, drd, len, docc, next, ctx->derr.ptr, st));
            CK(cudaMemcpyAsync(out, docc, len, cudaMemcpyDeviceToHost, st));
        } else {
            int32_t *dp = ctx->hprim.ptr + (size_t)s * m;
            float *dt = ctx->ht.ptr + (size_t)s * m, *du = ctx->hu.ptr + (size_t)s * m, *dv = ctx->hv.ptr + (size_t)s * m;
            if (wt)
                CK(launch_closest_wt(sv, ctx->raw_tris.ptr, dro, drd, len, dp, dt, du, dv, next, ctx->derr.ptr, st));
            else
                CK(launch_closest_dyn(sv, dro, drd, len, dp, dt, du, dv, next, ctx->derr.ptr, st));
            CK(cudaMemcpyAsync(out, dp, 4ull * len, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(out + 4ull * kChunk, dt, 4ull * len, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(out + 8ull * kChunk, du, 4ull * len, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(out + 12ull * kChunk, dv, 4ull * len, cudaMemcpyDeviceToHost, st));
        }
        CK(cudaEventRecord(ctx->pin_ev[s], st));
    }
    // the last chunks' hits, in order
    for (uint32_t c = chunks > kPinSlots ? chunks - kPinSlots : 0; c < chunks; c++) {
        CK(cudaEventSynchronize(ctx->pin_ev[c % kPinSlots]));
        CopySeg seg[4];
        const int nseg = out_segs(c, seg);
        pool_copy_ctx(ctx, seg, nseg);
    }
    return ctx->check_device_error();
}

int query_host_pageable(ilg_ctx *ctx, const float *o4, const float *d4, uint32_t n, int32_t *prim, float *t,
                        float *u, float *v, uint8_t *occ, bool wt)
{
    const int rc = query_host_pageable_run(ctx, o4, d4, n, prim, t, u, v, occ, wt);
    // after a failure, copies of this call may still be in flight into the
    // page-locked slots that the next call fills from the host
    if (rc != ILG_OK) {
        cudaStreamSynchronize(ctx->stream);
        for (auto sd : ctx->side)
            if (sd) cudaStreamSynchronize(sd);
    }
    return rc;
}

// Closest hit (occ == nullptr) or any hit of rays in host memory. Large
// batches go in chunks round-robin over three streams, so the upload of one
// chunk, the traversal of the previous one and the download of the one
// before that run at once; for host-resident rays the PCIe copies, not the
// traversal, bound the call.
int query_host(ilg_ctx *ctx, const float *o4, const float *d4, uint32_t n, int32_t *prim, float *t, float *u,
               float *v, uint8_t *occ, bool wt)
{
    const bool any = occ != nullptr;
    if (n >= (1u << 16) && (pageable(o4) || pageable(d4) || (any ? pageable(occ) : pageable(prim) || pageable(t) ||
                                                                   pageable(u) || pageable(v))))
        return query_host_pageable(ctx, o4, d4, n, prim, t, u, v, occ, wt);
    CK(ctx->ro.reserve(n));
    CK(ctx->rd.reserve(n));
    if (any) {
        CK(ctx->hocc.reserve(n));
    } else {
        CK(ctx->hprim.reserve(n));
        CK(ctx->ht.reserve(n));
        CK(ctx->hu.reserve(n));
        CK(ctx->hv.reserve(n));
    }
    // up to 8 chunks of >= 256 K rays, more for large batches so that no chunk
    // exceeds about 512 K rays (measured on a B200: 8.4 M rays in one call ran
    // 3 % slower in 8 chunks than as two calls of 4.2 M in 8 chunks each)
    const uint32_t kMinChunk = 1u << 18, kTargetChunk = 1u << 19, kMaxChunks = 64u;
    const uint32_t chunks =
        n >= 2u * kMinChunk ? std::min<uint32_t>(kMaxChunks, std::max<uint32_t>(std::min<uint32_t>(8u, n / kMinChunk),
                                                                                n / kTargetChunk))
                            : 1u;
    const uint32_t chunk = ((n + chunks - 1) / chunks + 127u) & ~127u;
    cudaStream_t ss[3] = {ctx->stream, ctx->stream, ctx->stream};
    if (chunks > 1) {
        for (int k = 0; k < 2; k++)
            if (!ctx->side[k]) CK(cudaStreamCreateWithFlags(&ctx->side[k], cudaStreamNonBlocking));
        for (int k = 0; k < 3; k++)
            if (!ctx->side_ev[k]) CK(cudaEventCreateWithFlags(&ctx->side_ev[k], cudaEventDisableTiming));
        // the side streams start after everything already queued on the main one
        CK(cudaEventRecord(ctx->side_ev[2], ctx->stream));
        for (int k = 0; k < 2; k++) {
            CK(cudaStreamWaitEvent(ctx->side[k], ctx->side_ev[2], 0));
            ss[1 + k] = ctx->side[k];
        }
    }
    const SceneView sv = ctx->view();
    uint32_t c = 0;
    for (uint32_t off = 0; off < n; off += chunk, c++) {
        const uint32_t len = std::min(chunk, n - off);
        cudaStream_t st = ss[c % 3];
        uint32_t *next = ctx->derr.ptr + 1 + (c % 3);  // ray counter of this stream's persistent kernels
        CK(cudaMemcpyAsync(ctx->ro.ptr + off, o4 + 4ull * off, 16ull * len, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->rd.ptr + off, d4 + 4ull * off, 16ull * len, cudaMemcpyHostToDevice, st));
        if (any && wt) {
            CK(launch_any_wt(sv, ctx->raw_tris.ptr, ctx->ro.ptr + off, ctx->rd.ptr + off, len, ctx->hocc.ptr + off,
                             next, ctx->derr.ptr, st));
            CK(cudaMemcpyAsync(occ + off, ctx->hocc.ptr + off, len, cudaMemcpyDeviceToHost, st));
        } else if (any) {
            CK(launch_any_dyn(sv, ctx->ro.ptr + off, ctx->rd.ptr + off, len, ctx->hocc.ptr + off, next, ctx->derr.ptr,
                              st));
            CK(cudaMemcpyAsync(occ + off, ctx->hocc.ptr + off, len, cudaMemcpyDeviceToHost, st));
        } else {
            if (wt)
                CK(launch_closest_wt(sv, ctx->raw_tris.ptr, ctx->ro.ptr + off, ctx->rd.ptr + off, len,
                                     ctx->hprim.ptr + off, ctx->ht.ptr + off, ctx->hu.ptr + off, ctx->hv.ptr + off,
                                     next, ctx->derr.ptr, st));
            else
                CK(launch_closest_dyn(sv, ctx->ro.ptr + off, ctx->rd.ptr + off, len, ctx->hprim.ptr + off,
                                      ctx->ht.ptr + off, ctx->hu.ptr + off, ctx->hv.ptr + off, next, ctx->derr.ptr,
                                      st));
            CK(cudaMemcpyAsync(prim + off, ctx->hprim.ptr + off, 4ull * len, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(t + off, ctx->ht.ptr + off, 4ull * len, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(u + off, ctx->hu.ptr + off, 4ull * len, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(v + off, ctx->hv.ptr + off, 4ull * len, cudaMemcpyDeviceToHost, st));
        }
    }
    if (chunks > 1) {
        // the main stream ends after the side streams' work
        for (int k = 0; k < 2; k++) {
            CK(cudaEventRecord(ctx->side_ev[k], ctx->side[k]));
            CK(cudaStreamWaitEvent(ctx->stream, ctx->side_ev[k], 0));
        }
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return ctx->check_device_error();
}

}  // namespace

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
    ctx->build_flags = opts ? opts->build_flags : 0u;
    if (cudaSetDevice(dev) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
        ctx->derr.reserve(4) != cudaSuccess || ctx->dstats.reserve(2) != cudaSuccess) {
        delete ctx;
        return ILG_ECUDA;
    }
    cudaMemsetAsync(ctx->derr.ptr, 0, 4 * sizeof(uint32_t), ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    // the allocation-free query's fixed array becomes resident here, not at
    // its first call; a failure only disables that entry point
    if (noalloc_prepare(&ctx->noalloc_scratch) != cudaSuccess) {
        ctx->noalloc_scratch = nullptr;
        cudaGetLastError();
    }
    *out = ctx;
    return ILG_OK;
}

int ilg_destroy(ilg_ctx *ctx)
{
    if (!ctx) return ILG_EINVAL;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto s : ctx->side)
        if (s) cudaStreamSynchronize(s);
    ctx->release_all();
    cudaEventDestroy(ctx->ev0);
    cudaEventDestroy(ctx->ev1);
    for (auto e : ctx->side_ev)
        if (e) cudaEventDestroy(e);
    for (auto e : ctx->pin_ev)
        if (e) cudaEventDestroy(e);
    if (ctx->pin_buf) cudaFreeHost(ctx->pin_buf);
    delete ctx->host_pool;
    for (auto s : ctx->side)
        if (s) cudaStreamDestroy(s);
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
    float lo[3] = {3.0e38f, 3.0e38f, 3.0e38f}, hi[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
    for (uint64_t i = 0; i < 3ull * n_verts; i++) {
        float a = fabsf(pos_xyz[i]);
        if (!(a <= 3.0e38f)) return fail(ctx, ILG_EINVAL, "ilg_set_mesh: non-finite position at %llu", (unsigned long long)i);
        maxabs = std::max(maxabs, a);
        lo[i % 3] = std::min(lo[i % 3], pos_xyz[i]);
        hi[i % 3] = std::max(hi[i % 3], pos_xyz[i]);
    }
    for (int k = 0; k < 3; k++) {
        ctx->scene_lo[k] = lo[k];
        ctx->scene_hi[k] = hi[k];
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
    ctx->mesh_gen++;
    ctx->has_mat = mat_ids != nullptr;
    ctx->max_abs = maxabs;
    ctx->built = false;
    ctx->attr_dirty = true;
    return ILG_OK;
}

int ilg_build(ilg_ctx *ctx)
{
    if (!ctx) return ILG_EINVAL;
    if (ctx->n_tris == 0) return fail(ctx, ILG_ESTATE, "ilg_build: no mesh set");
    CK(cudaSetDevice(ctx->device));
    BuildResult res;
    res.min_step = std::max(ctx->max_abs * 0x1p-19f, 1e-30f);
    res.treelets = !(ctx->build_flags & ILG_BUILD_FAST);
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
    ctx->attr_dirty = true;
    ctx->raw_ready = false;
    return ILG_OK;
}

// ---------------------------------------------------------------------------
// Persistent scenes: the uploaded mesh and the built 8-wide BVH in one file,
// so a scene is loaded instead of rebuilt. Layout (little-endian): a 64-byte
// header, then positions (12 B a vertex), indices (12 B a triangle), material
// ids (4 B a triangle, when present), node records (80 B), triangle records
// (48 B), record -> input triangle map (4 B), and an FNV-1a 64 checksum of
// everything after the header.
// ---------------------------------------------------------------------------
namespace {

struct SceneFileHeader {
    char magic[8];  // "ILGBVH8\0"
    uint32_t version, header_bytes;
    uint32_t n_verts, n_tris, n_nodes, n_leaf_tris;
    uint32_t max_depth, has_mat, node_bytes, tri_bytes;
    uint64_t payload_bytes;
    uint64_t reserved;
};
static_assert(sizeof(SceneFileHeader) == 64, "scene file header is 64 bytes");

constexpr uint32_t kSceneFileVersion = 1;

uint64_t fnv1a(uint64_t h, const void *data, size_t n)
{
    const unsigned char *p = static_cast<const unsigned char *>(data);
    for (size_t i = 0; i < n; i++) {
        h ^= p[i];
        h *= 0x100000001B3ull;
    }
    return h;
}

}  // namespace

int ilg_save(ilg_ctx *ctx, const char *path)
{
    if (!ctx || !path) return ILG_EINVAL;
    if (!ctx->built) return fail(ctx, ILG_ESTATE, "ilg_save: scene not built");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    SceneFileHeader h;
    memset(&h, 0, sizeof(h));
    memcpy(h.magic, "ILGBVH8", 8);
    h.version = kSceneFileVersion;
    h.header_bytes = sizeof(h);
    h.n_verts = ctx->n_verts;
    h.n_tris = ctx->n_tris;
    h.n_nodes = ctx->stats.n_nodes;
    h.n_leaf_tris = ctx->stats.n_leaf_tris;
    h.max_depth = ctx->stats.max_depth;
    h.has_mat = ctx->has_mat ? 1u : 0u;
    h.node_bytes = sizeof(Node8);
    h.tri_bytes = sizeof(Tri);
    std::vector<float> pos(3ull * h.n_verts);
    std::vector<uint32_t> idx(3ull * h.n_tris), mat(h.has_mat ? h.n_tris : 0), prim(h.n_leaf_tris);
    std::vector<Node8> nodes(h.n_nodes);
    std::vector<Tri> tris(h.n_leaf_tris);
    CK(cudaMemcpyAsync(pos.data(), ctx->pos.ptr, 12ull * h.n_verts, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(idx.data(), ctx->idx.ptr, 12ull * h.n_tris, cudaMemcpyDeviceToHost, st));
    if (h.has_mat) CK(cudaMemcpyAsync(mat.data(), ctx->mat.ptr, 4ull * h.n_tris, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(nodes.data(), ctx->bb.nodes, sizeof(Node8) * h.n_nodes, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(tris.data(), ctx->bb.tris, sizeof(Tri) * h.n_leaf_tris, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(prim.data(), ctx->bb.prim_of, 4ull * h.n_leaf_tris, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const std::pair<const void *, size_t> parts[6] = {
        {pos.data(), 12ull * h.n_verts}, {idx.data(), 12ull * h.n_tris}, {mat.data(), 4ull * mat.size()},
        {nodes.data(), sizeof(Node8) * nodes.size()}, {tris.data(), sizeof(Tri) * tris.size()},
        {prim.data(), 4ull * prim.size()}};
    uint64_t sum = 0xCBF29CE484222325ull;
    for (auto &q : parts) {
        h.payload_bytes += q.second;
        sum = fnv1a(sum, q.first, q.second);
    }
    FILE *f = fopen(path, "wb");
    if (!f) return fail(ctx, ILG_EINVAL, "ilg_save: cannot open %s for writing", path);
    bool ok = fwrite(&h, sizeof(h), 1, f) == 1;
    for (auto &q : parts)
        if (ok && q.second) ok = fwrite(q.first, 1, q.second, f) == q.second;
    ok = ok && fwrite(&sum, sizeof(sum), 1, f) == 1;
    ok = (fclose(f) == 0) && ok;
    if (!ok) return fail(ctx, ILG_EINVAL, "ilg_save: writing %s failed", path);
    return ILG_OK;
}

int ilg_load(ilg_ctx *ctx, const char *path)
{
    if (!ctx || !path) return ILG_EINVAL;
    FILE *f = fopen(path, "rb");
    if (!f) return fail(ctx, ILG_EINVAL, "ilg_load: cannot open %s", path);
    SceneFileHeader h;
    auto bad = [&](const char *why) {
        fclose(f);
        return fail(ctx, ILG_EINVAL, "ilg_load: %s: %s", path, why);
    };
    if (fread(&h, sizeof(h), 1, f) != 1) return bad("short header");
    if (memcmp(h.magic, "ILGBVH8", 8) != 0) return bad("not a scene file");
    if (h.version != kSceneFileVersion || h.header_bytes != sizeof(h)) return bad("unsupported version");
    if (h.node_bytes != sizeof(Node8) || h.tri_bytes != sizeof(Tri)) return bad("record sizes differ");
    if (h.n_verts == 0 || h.n_tris == 0 || h.n_tris > (1u << 30) || h.n_leaf_tris != h.n_tris || h.n_nodes == 0 ||
        h.n_nodes > h.n_tris + 1u || h.has_mat > 1u)
        return bad("inconsistent counts");
    const uint64_t expect = 12ull * h.n_verts + 12ull * h.n_tris + (h.has_mat ? 4ull * h.n_tris : 0ull) +
                            sizeof(Node8) * (uint64_t)h.n_nodes + sizeof(Tri) * (uint64_t)h.n_leaf_tris +
                            4ull * h.n_leaf_tris;
    if (h.payload_bytes != expect) return bad("payload size differs from the counts");
    std::vector<float> pos(3ull * h.n_verts);
    std::vector<uint32_t> idx(3ull * h.n_tris), mat(h.has_mat ? h.n_tris : 0), prim(h.n_leaf_tris);
    std::vector<Node8> nodes(h.n_nodes);
    std::vector<Tri> tris(h.n_leaf_tris);
    const std::pair<void *, size_t> parts[6] = {
        {pos.data(), 12ull * h.n_verts}, {idx.data(), 12ull * h.n_tris}, {mat.data(), 4ull * mat.size()},
        {nodes.data(), sizeof(Node8) * nodes.size()}, {tris.data(), sizeof(Tri) * tris.size()},
        {prim.data(), 4ull * prim.size()}};
    uint64_t sum = 0xCBF29CE484222325ull, stored = 0;
    for (auto &q : parts) {
        if (q.second && fread(q.first, 1, q.second, f) != q.second) return bad("truncated");
        sum = fnv1a(sum, q.first, q.second);
    }
    if (fread(&stored, sizeof(stored), 1, f) != 1) return bad("truncated checksum");
    fclose(f);
    if (stored != sum) return fail(ctx, ILG_EINVAL, "ilg_load: %s: checksum mismatch", path);
    // record -> triangle map: a permutation of the triangles (the renderer indexes with it)
    {
        std::vector<unsigned char> seen(h.n_tris, 0);
        for (uint32_t p : prim) {
            if (p >= h.n_tris || seen[p]) return fail(ctx, ILG_EINVAL, "ilg_load: %s: bad triangle map", path);
            seen[p] = 1;
        }
    }
    int rc = ilg_set_mesh(ctx, pos.data(), h.n_verts, idx.data(), h.n_tris, h.has_mat ? mat.data() : nullptr);
    if (rc) return rc;
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    CK(ctx->bb.nodes_b.reserve(h.n_nodes));
    CK(ctx->bb.tris_b.reserve(h.n_leaf_tris));
    CK(ctx->bb.prim_of_b.reserve(h.n_leaf_tris));
    ctx->bb.nodes = ctx->bb.nodes_b.ptr;
    ctx->bb.tris = ctx->bb.tris_b.ptr;
    ctx->bb.prim_of = ctx->bb.prim_of_b.ptr;
    CK(cudaMemcpyAsync(ctx->bb.nodes, nodes.data(), sizeof(Node8) * h.n_nodes, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->bb.tris, tris.data(), sizeof(Tri) * h.n_leaf_tris, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->bb.prim_of, prim.data(), 4ull * h.n_leaf_tris, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    ctx->stats.n_tris = h.n_tris;
    ctx->stats.n_nodes = h.n_nodes;
    ctx->stats.n_leaf_tris = h.n_leaf_tris;
    ctx->stats.max_depth = h.max_depth;
    ctx->stats.build_ms = 0.f;
    ctx->stats.node_bytes = (uint64_t)h.n_nodes * sizeof(Node8);
    ctx->stats.tri_bytes = (uint64_t)h.n_leaf_tris * sizeof(Tri);
    ctx->built = true;
    ctx->attr_dirty = true;
    ctx->raw_ready = false;
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
    if (flags & ~(ILG_DEVICE_PTRS | ILG_WATERTIGHT))
        return fail(ctx, ILG_EINVAL, "ilg_intersect: unknown flags 0x%x", flags);
    if (!ctx->built) return fail(ctx, ILG_ESTATE, "ilg_intersect: scene not built");
    if (n == 0) return ILG_OK;
    if (!ray_o_tmin || !ray_d_tmax || !prim || !t || !u || !v) return fail(ctx, ILG_EINVAL, "ilg_intersect: null array");
    if (((uintptr_t)ray_o_tmin | (uintptr_t)ray_d_tmax) & 15u)
        return fail(ctx, ILG_EINVAL, "ilg_intersect: ray arrays must be 16-byte aligned");
    CK(cudaSetDevice(ctx->device));
    const SceneView sv = ctx->view();
    uint32_t *next = ctx->derr.ptr + 1;  // ray counter of the persistent kernels
    const bool wt = (flags & ILG_WATERTIGHT) != 0;
    if (wt) {
        int rc = ensure_raw_tris(ctx);
        if (rc) return rc;
    }
    if (flags & ILG_DEVICE_PTRS) {
        if (wt)
            CK(launch_closest_wt(sv, ctx->raw_tris.ptr, (const float4 *)ray_o_tmin, (const float4 *)ray_d_tmax, n,
                                 prim, t, u, v, next, ctx->derr.ptr, ctx->stream));
        else
            CK(launch_closest_dyn(sv, (const float4 *)ray_o_tmin, (const float4 *)ray_d_tmax, n, prim, t, u, v, next,
                                  ctx->derr.ptr, ctx->stream));
        return ILG_OK;
    }
    return query_host(ctx, ray_o_tmin, ray_d_tmax, n, prim, t, u, v, nullptr, wt);
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
    if (flags & ~(ILG_DEVICE_PTRS | ILG_WATERTIGHT))
        return fail(ctx, ILG_EINVAL, "ilg_occluded: unknown flags 0x%x", flags);
    if (!ctx->built) return fail(ctx, ILG_ESTATE, "ilg_occluded: scene not built");
    if (n == 0) return ILG_OK;
    if (!ray_o_tmin || !ray_d_tmax || !occ) return fail(ctx, ILG_EINVAL, "ilg_occluded: null array");
    if (((uintptr_t)ray_o_tmin | (uintptr_t)ray_d_tmax) & 15u)
        return fail(ctx, ILG_EINVAL, "ilg_occluded: ray arrays must be 16-byte aligned");
    CK(cudaSetDevice(ctx->device));
    const SceneView sv = ctx->view();
    uint32_t *next = ctx->derr.ptr + 1;
    const bool wt = (flags & ILG_WATERTIGHT) != 0;
    if (wt) {
        int rc = ensure_raw_tris(ctx);
        if (rc) return rc;
    }
    if (flags & ILG_DEVICE_PTRS) {
        if (wt)
            CK(launch_any_wt(sv, ctx->raw_tris.ptr, (const float4 *)ray_o_tmin, (const float4 *)ray_d_tmax, n, occ,
                             next, ctx->derr.ptr, ctx->stream));
        else
            CK(launch_any_dyn(sv, (const float4 *)ray_o_tmin, (const float4 *)ray_d_tmax, n, occ, next, ctx->derr.ptr,
                              ctx->stream));
        return ILG_OK;
    }
    return query_host(ctx, ray_o_tmin, ray_d_tmax, n, nullptr, nullptr, nullptr, nullptr, occ, wt);
}

int ilg_intersect_excluding(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n,
                            uint32_t skip_first, uint32_t skip_count, int32_t *prim, float *t, float *u, float *v,
                            uint32_t flags)
{
    if (!ctx) return ILG_EINVAL;
    if (flags & ~ILG_DEVICE_PTRS) return fail(ctx, ILG_EINVAL, "ilg_intersect_excluding: unknown flags 0x%x", flags);
    if (!ctx->built) return fail(ctx, ILG_ESTATE, "ilg_intersect_excluding: scene not built");
    if (n == 0) return ILG_OK;
    if (!ray_o_tmin || !ray_d_tmax || !prim || !t || !u || !v)
        return fail(ctx, ILG_EINVAL, "ilg_intersect_excluding: null array");
    if (((uintptr_t)ray_o_tmin | (uintptr_t)ray_d_tmax) & 15u)
        return fail(ctx, ILG_EINVAL, "ilg_intersect_excluding: ray arrays must be 16-byte aligned");
    CK(cudaSetDevice(ctx->device));
    const SceneView sv = ctx->view();
    cudaStream_t st = ctx->stream;
    if (flags & ILG_DEVICE_PTRS) {
        CK(launch_closest_skip(sv, (const float4 *)ray_o_tmin, (const float4 *)ray_d_tmax, n, skip_first, skip_count,
                               prim, t, u, v, ctx->derr.ptr, st));
        return ILG_OK;
    }
    CK(ctx->ro.reserve(n));
    CK(ctx->rd.reserve(n));
    CK(ctx->hprim.reserve(n));
    CK(ctx->ht.reserve(n));
    CK(ctx->hu.reserve(n));
    CK(ctx->hv.reserve(n));
    CK(cudaMemcpyAsync(ctx->ro.ptr, ray_o_tmin, 16ull * n, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->rd.ptr, ray_d_tmax, 16ull * n, cudaMemcpyHostToDevice, st));
    CK(launch_closest_skip(sv, ctx->ro.ptr, ctx->rd.ptr, n, skip_first, skip_count, ctx->hprim.ptr, ctx->ht.ptr,
                           ctx->hu.ptr, ctx->hv.ptr, ctx->derr.ptr, st));
    CK(cudaMemcpyAsync(prim, ctx->hprim.ptr, 4ull * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(t, ctx->ht.ptr, 4ull * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(u, ctx->hu.ptr, 4ull * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(v, ctx->hv.ptr, 4ull * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return ctx->check_device_error();
}

int ilg_occluded_excluding(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n,
                           uint32_t skip_first, uint32_t skip_count, uint8_t *occ, uint32_t flags)
{
    if (!ctx) return ILG_EINVAL;
    if (flags & ~ILG_DEVICE_PTRS) return fail(ctx, ILG_EINVAL, "ilg_occluded_excluding: unknown flags 0x%x", flags);
    if (!ctx->built) return fail(ctx, ILG_ESTATE, "ilg_occluded_excluding: scene not built");
    if (n == 0) return ILG_OK;
    if (!ray_o_tmin || !ray_d_tmax || !occ) return fail(ctx, ILG_EINVAL, "ilg_occluded_excluding: null array");
    if (((uintptr_t)ray_o_tmin | (uintptr_t)ray_d_tmax) & 15u)
        return fail(ctx, ILG_EINVAL, "ilg_occluded_excluding: ray arrays must be 16-byte aligned");
    CK(cudaSetDevice(ctx->device));
    const SceneView sv = ctx->view();
    cudaStream_t st = ctx->stream;
    if (flags & ILG_DEVICE_PTRS) {
        CK(launch_any_skip(sv, (const float4 *)ray_o_tmin, (const float4 *)ray_d_tmax, n, skip_first, skip_count, occ,
                           ctx->derr.ptr, st));
        return ILG_OK;
    }
    CK(ctx->ro.reserve(n));
    CK(ctx->rd.reserve(n));
    CK(ctx->hocc.reserve(n));
    CK(cudaMemcpyAsync(ctx->ro.ptr, ray_o_tmin, 16ull * n, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->rd.ptr, ray_d_tmax, 16ull * n, cudaMemcpyHostToDevice, st));
    CK(launch_any_skip(sv, ctx->ro.ptr, ctx->rd.ptr, n, skip_first, skip_count, ctx->hocc.ptr, ctx->derr.ptr, st));
    CK(cudaMemcpyAsync(occ, ctx->hocc.ptr, n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return ctx->check_device_error();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// path tracing
// ---------------------------------------------------------------------------
namespace {
int mlp_reserve_train(ilg_ctx *ctx, uint32_t n);

struct V3 {
    float x, y, z;
};
inline V3 v3(const float *a) { return V3{a[0], a[1], a[2]}; }
inline V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator*(float s, V3 a) { return V3{s * a.x, s * a.y, s * a.z}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V3 normalize(V3 a)
{
    float l = std::sqrt(dot(a, a));
    return l > 0.f ? (1.f / l) * a : a;
}
inline float3 f3(V3 a) { return make_float3(a.x, a.y, a.z); }

}  // namespace

extern "C" {

int ilg_set_materials(ilg_ctx *ctx, const ilg_material *mats, uint32_t n)
{
    if (!ctx) return ILG_EINVAL;
    if (!mats || n == 0 || n > 0xffffu) return fail(ctx, ILG_EINVAL, "ilg_set_materials: need 1..65535 materials");
    static_assert(sizeof(ilg_material) == sizeof(Mat), "ilg_material layout");
    for (uint32_t i = 0; i < n; i++) {
        if (mats[i].kind > ILG_MAT_GLASS) return fail(ctx, ILG_EINVAL, "ilg_set_materials: material %u has unknown kind %u", i, mats[i].kind);
        if (mats[i].kind == ILG_MAT_GGX && !(mats[i].alpha > 0.f && mats[i].alpha <= 1.f))
            return fail(ctx, ILG_EINVAL, "ilg_set_materials: material %u needs 0 < alpha <= 1", i);
        if (mats[i].kind == ILG_MAT_GLASS && !(mats[i].alpha > 0.f && mats[i].alpha < 1e30f))
            return fail(ctx, ILG_EINVAL, "ilg_set_materials: glass material %u needs eta_i / eta_t > 0 in alpha", i);
    }
    CK(cudaSetDevice(ctx->device));
    CK(ctx->mats.reserve(n));
    CK(cudaMemcpyAsync(ctx->mats.ptr, mats, n * sizeof(Mat), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->n_mats = n;
    return ILG_OK;
}

int ilg_set_lights(ilg_ctx *ctx, const ilg_light *lights, uint32_t n)
{
    if (!ctx) return ILG_EINVAL;
    if (n > kMaxLights) return fail(ctx, ILG_EINVAL, "ilg_set_lights: at most %u lights", kMaxLights);
    if (n && !lights) return fail(ctx, ILG_EINVAL, "ilg_set_lights: null lights");
    Light hl[kMaxLights];
    uint2 range[kMaxLights];
    float inf = 0.f;
    bool uses_mesh = false;
    CK(cudaSetDevice(ctx->device));
    for (uint32_t i = 0; i < n; i++) {
        const ilg_light &L = lights[i];
        Light &d = hl[i];
        memset(&d, 0, sizeof(d));
        d.kind = L.kind;
        d.emit = make_float3(L.emit[0], L.emit[1], L.emit[2]);
        if (!(std::isfinite(L.emit[0]) && std::isfinite(L.emit[1]) && std::isfinite(L.emit[2])))
            return fail(ctx, ILG_EINVAL, "ilg_set_lights: light %u has a non-finite radiance", i);
        range[i] = make_uint2(0u, 0u);
        if (L.kind == ILG_LIGHT_QUAD) {
            if (ctx->n_tris && (uint64_t)L.first_tri + 2 > ctx->n_tris)
                return fail(ctx, ILG_EINVAL, "ilg_set_lights: light %u triangles out of range", i);
            V3 p0 = v3(L.v[0]), p1 = v3(L.v[1]), p2 = v3(L.v[2]), p3 = v3(L.v[3]);
            V3 n0 = cross(p2 - p0, p1 - p0);   // triangle (v1, v3, v2)
            V3 n1 = cross(p3 - p0, p2 - p0);   // triangle (v1, v4, v3)
            float area = 0.5f * std::sqrt(dot(n0, n0)) + 0.5f * std::sqrt(dot(n1, n1));
            if (!(area > 0.f)) return fail(ctx, ILG_EINVAL, "ilg_set_lights: light %u has zero area", i);
            d.p[0] = f3(p0); d.p[1] = f3(p1); d.p[2] = f3(p2); d.p[3] = f3(p3);
            d.n = f3(normalize(n0));
            d.area = area;
            d.first_tri = L.first_tri;
            d.tri_count = 2;
            range[i] = make_uint2(L.first_tri, 2u);
        } else if (L.kind == ILG_LIGHT_MESH) {
            if (!ctx->n_tris || L.tri_count == 0 || (uint64_t)L.first_tri + L.tri_count > ctx->n_tris)
                return fail(ctx, ILG_EINVAL, "ilg_set_lights: mesh light %u triangles out of range", i);
            // ITriangleMesh::ComputeArea (Core/Shape/TriangleMesh.cpp:163-168): the
            // triangles' areas summed in order in float
            ilg::DevBuf<float> areas;
            CK(areas.reserve(L.tri_count));
            CK(triangle_areas(ctx->pos.ptr, ctx->idx.ptr, L.first_tri, L.tri_count, areas.ptr, ctx->stream));
            std::vector<float> ha(L.tri_count);
            CK(cudaMemcpyAsync(ha.data(), areas.ptr, 4ull * L.tri_count, cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            areas.release();
            float area = 0.f;
            for (float a : ha) area += a;
            if (!(area > 0.f)) return fail(ctx, ILG_EINVAL, "ilg_set_lights: mesh light %u has zero area", i);
            d.area = area;
            d.first_tri = L.first_tri;
            d.tri_count = L.tri_count;
            range[i] = make_uint2(L.first_tri, L.tri_count);
            uses_mesh = true;
        } else if (L.kind == ILG_LIGHT_INFINITE) {
            inf += 1.f;
        } else {
            return fail(ctx, ILG_EINVAL, "ilg_set_lights: light %u has unknown kind %u", i, L.kind);
        }
    }
    CK(ctx->lights.reserve(kMaxLights));
    CK(ctx->light_range.reserve(kMaxLights));
    if (n) {
        CK(cudaMemcpyAsync(ctx->lights.ptr, hl, n * sizeof(Light), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(ctx->light_range.ptr, range, n * sizeof(uint2), cudaMemcpyHostToDevice, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->n_lights = n;
    memcpy(ctx->light_range_host, range, n * sizeof(uint2));
    ctx->inf_escape = inf;
    ctx->lights_use_mesh = uses_mesh;
    ctx->lights_mesh_gen = ctx->mesh_gen;
    ctx->attr_dirty = true;
    return ILG_OK;
}

int ilg_set_quad_lights(ilg_ctx *ctx, const ilg_quad_light *lights, uint32_t n)
{
    if (!ctx) return ILG_EINVAL;
    if (n > kMaxLights) return fail(ctx, ILG_EINVAL, "ilg_set_quad_lights: at most %u lights", kMaxLights);
    if (n && !lights) return fail(ctx, ILG_EINVAL, "ilg_set_quad_lights: null lights");
    ilg_light all[kMaxLights];
    for (uint32_t i = 0; i < n; i++) {
        memset(&all[i], 0, sizeof(ilg_light));
        all[i].kind = ILG_LIGHT_QUAD;
        memcpy(all[i].emit, lights[i].emit, sizeof(all[i].emit));
        memcpy(all[i].v, lights[i].v, sizeof(all[i].v));
        all[i].first_tri = lights[i].first_tri;
        all[i].tri_count = 2;
    }
    return ilg_set_lights(ctx, n ? all : nullptr, n);
}

// The camera frame PerspectiveCamera(eye, normalize(target - eye), up,
// -1,1,-1,1, 1) + SetFieldOfView builds (Core/Camera/Camera.cpp:30-44,
// Core/Geometry/Basis.cpp:28-44).
static void camera_frame_of(const ilg_camera &cam, ilg_camera_frame &f)
{
    V3 eye = v3(cam.eye);
    V3 w = normalize(normalize(v3(cam.target) - eye));
    V3 v = normalize(v3(cam.up));
    v = v - dot(v, w) * w;
    if (dot(v, v) <= 1.1920929e-7f) {
        v = V3{w.z, w.x, w.y};
        v = normalize(cross(v, w));
        v = normalize(v - dot(v, w) * w);
    }
    V3 u = cross(v, w);
    const float half = cam.fov_deg * (std::atan(1.0f) / 45.0f) * 0.5f;
    const float v1 = std::tan(half), v0 = -v1, u0 = v0 * cam.aspect, u1 = v1 * cam.aspect;
    const V3 corner = eye + u0 * u + v0 * v + 1.0f * w, across = (u1 - u0) * u, up = (v1 - v0) * v;
    const V3 *src[4] = {&eye, &corner, &across, &up};
    float *dst[4] = {f.centre, f.corner, f.across, f.up};
    for (int k = 0; k < 4; k++) {
        dst[k][0] = src[k]->x;
        dst[k][1] = src[k]->y;
        dst[k][2] = src[k]->z;
    }
}

// Validates a scene context for rendering and fills its scene record for the
// region (rx, ry, rw, rh) of a W x H image. Builds the per-triangle
// attributes on `st`.
static int prepare_scene(ilg_ctx *runner, ilg_ctx *ctx, const ilg_camera_frame &cam, uint32_t W, uint32_t H,
                         uint32_t rx, uint32_t ry, uint32_t rw, uint32_t rh, uint32_t spp, uint32_t max_depth,
                         float eps, uint32_t seed, const float sky[3], cudaStream_t st, SceneRec &S)
{
    if (!ctx) return fail(runner, ILG_EINVAL, "render: null scene");
    if (ctx->device != runner->device) return fail(runner, ILG_EINVAL, "render: scene on another device");
    if (!ctx->built) return fail(runner, ILG_ESTATE, "ilg_render: scene not built");
    if (!ctx->has_mat || ctx->n_mats == 0) return fail(runner, ILG_ESTATE, "ilg_render: materials not set");
    if (W == 0 || H == 0 || spp == 0 || (uint64_t)W * H > (1u << 26))
        return fail(runner, ILG_EINVAL, "ilg_render: bad image size %ux%u or spp %u", W, H, spp);
    if (rw == 0 || rh == 0 || (uint64_t)rx + rw > W || (uint64_t)ry + rh > H)
        return fail(runner, ILG_EINVAL, "ilg_render: region %u,%u %ux%u outside the %ux%u image", rx, ry, rw, rh, W, H);
    if (max_depth == 0 || max_depth > 64) return fail(runner, ILG_EINVAL, "ilg_render: max_depth must be 1..64");
    for (uint32_t l = 0; l < ctx->n_lights; l++)
        if ((uint64_t)ctx->light_range_host[l].x + ctx->light_range_host[l].y > ctx->n_tris)
            return fail(runner, ILG_EINVAL, "ilg_render: light %u triangles out of range of the mesh", l);
    if (ctx->lights_use_mesh && ctx->lights_mesh_gen != ctx->mesh_gen)
        return fail(runner, ILG_ESTATE, "ilg_render: mesh lights were set for an earlier mesh (call ilg_set_lights again)");
    const uint32_t n = ctx->n_tris;
    if (ctx->attr_dirty) {
        CK2(runner, ctx->tri_attr.reserve(n));
        CK2(runner, ctx->light_of_prim.reserve(n));
        CK2(runner, build_tri_attr(ctx->bb.prim_of, n, ctx->mat.ptr, ctx->light_range.ptr, ctx->n_lights,
                                   ctx->light_of_prim.ptr, ctx->tri_attr.ptr, st));
        ctx->attr_dirty = false;
    }
    S = SceneRec{};
    S.nodes = ctx->bb.nodes; S.tris = ctx->bb.tris; S.n_nodes = ctx->stats.n_nodes; S.n_tris = ctx->stats.n_tris;
    S.tri_attr = ctx->tri_attr.ptr; S.mats = ctx->mats.ptr; S.n_mats = ctx->n_mats;
    S.lights = ctx->lights.ptr; S.n_lights = ctx->n_lights;
    S.sky = make_float3(sky[0], sky[1], sky[2]);
    S.inf_escape = ctx->inf_escape;
    S.pos = ctx->pos.ptr; S.idx = ctx->idx.ptr;
    S.centre = make_float3(cam.centre[0], cam.centre[1], cam.centre[2]);
    S.corner = make_float3(cam.corner[0], cam.corner[1], cam.corner[2]);
    S.across = make_float3(cam.across[0], cam.across[1], cam.across[2]);
    S.up = make_float3(cam.up[0], cam.up[1], cam.up[2]);
    S.width = W; S.height = H; S.full_wh = W * H; S.rcp_w = 1.f / W; S.rcp_h = 1.f / H;
    S.region_x = rx; S.region_y = ry; S.region_w = rw; S.wh = rw * rh;
    S.max_depth = max_depth; S.eps = eps; S.spp = spp; S.seed = seed;
    return ILG_OK;
}

// Renders the scenes of `recs` (path ranges and pixel bases filled here) in
// waves of at most `cap_req` paths on the runner's buffers and stream.
static int run_render(ilg_ctx *ctx, std::vector<SceneRec> &recs, uint32_t cap_req, uint32_t block,
                      uint32_t cache_depth, uint32_t train_every, uint32_t train_steps, uint32_t train_batch,
                      uint64_t *total_paths_out, bool aux = false, bool count = false, uint32_t train_tail = 0,
                      uint32_t train_epochs = 1, bool hash_cache = false, bool one_launch = false)
{
    if (one_launch && (cache_depth || aux || count))
        return fail(ctx, ILG_EINVAL,
                    "render: ILG_RENDER_PERSISTENT renders plain images only (no cache, Direct / Albedo or counts)");
    cudaStream_t st = ctx->stream;
    uint64_t total = 0, pixels64 = 0;
    uint32_t pixels = 0, depth_max = 0, nl = 1;
    for (auto &S : recs) {
        S.path_begin = total;
        S.pixel_base = pixels;
        total += (uint64_t)S.wh * S.spp;
        pixels64 += S.wh;
        pixels = (uint32_t)std::min<uint64_t>(pixels64, 0xffffffffu);
        depth_max = std::max(depth_max, S.max_depth);
        nl = std::max(nl, S.n_lights);
    }
    // shadow segments carry the pixel in 31 bits (bit 31 tags Direct)
    if (pixels64 >= 0x80000000u) return fail(ctx, ILG_EINVAL, "render: more than 2^31 pixels in one call");
    if (total_paths_out) *total_paths_out = total;
    // wave size: whole samples for a single scene (so a wave never splits a pixel's sample)
    uint32_t cap = cap_req ? cap_req : (1u << 22);
    if (recs.size() == 1) {
        const uint32_t wh = recs[0].wh;
        uint32_t spw = std::max<uint32_t>(1u, cap / wh);
        spw = std::min(spw, recs[0].spp);
        cap = wh * spw;
    } else {
        cap = (uint32_t)std::min<uint64_t>(cap, total);
    }
    CK(ctx->q_o0.reserve(cap)); CK(ctx->q_d0.reserve(cap)); CK(ctx->q_o1.reserve(cap)); CK(ctx->q_d1.reserve(cap));
    CK(ctx->q_p0.reserve(cap)); CK(ctx->q_p1.reserve(cap)); CK(ctx->beta.reserve(cap));
    CK(ctx->hit_tri.reserve(cap)); CK(ctx->hit_t.reserve(cap)); CK(ctx->path_scene.reserve(cap));
    CK(ctx->s_o.reserve((size_t)cap * nl)); CK(ctx->s_d.reserve((size_t)cap * nl)); CK(ctx->s_c.reserve((size_t)cap * nl));
    CK(ctx->s_sid.reserve((size_t)cap * nl));
    CK(ctx->counts.reserve(9)); CK(ctx->accum.reserve((size_t)pixels + 1));
    CK(ctx->scene_table.reserve(recs.size()));
    CK(cudaMemcpyAsync(ctx->scene_table.ptr, recs.data(), recs.size() * sizeof(SceneRec), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(ctx->accum.ptr, 0, sizeof(float4) * ((size_t)pixels + 1), st));

    RenderDev R = {};
    R.scenes = ctx->scene_table.ptr; R.n_scenes = (uint32_t)recs.size(); R.depth_max = depth_max;
    R.path_scene = ctx->path_scene.ptr; R.s_sid = ctx->s_sid.ptr;
    R.q_o[0] = ctx->q_o0.ptr; R.q_o[1] = ctx->q_o1.ptr; R.q_d[0] = ctx->q_d0.ptr; R.q_d[1] = ctx->q_d1.ptr;
    R.q_path[0] = ctx->q_p0.ptr; R.q_path[1] = ctx->q_p1.ptr;
    R.count = ctx->counts.ptr; R.capacity = cap;
    R.hit_tri = ctx->hit_tri.ptr; R.hit_t = ctx->hit_t.ptr; R.beta = ctx->beta.ptr;
    R.s_o = ctx->s_o.ptr; R.s_d = ctx->s_d.ptr; R.s_c = ctx->s_c.ptr;
    R.sh_count = ctx->counts.ptr + 2; R.sh_capacity = cap * nl;
    R.accum = ctx->accum.ptr; R.err = ctx->derr.ptr;
    R.discard_pixel = pixels;
    // measured on a B200: persistent traversal gains 18-25 % on the 21 M- and
    // 13.8 M-triangle workloads and loses 6 % on the 16-triangle box scene
    for (auto &S : recs) R.persistent |= S.n_tris >= 4096u ? 1u : 0u;
    if (count) {
        CK(ctx->render_stats.reserve(6));
        CK(cudaMemsetAsync(ctx->render_stats.ptr, 0, 6 * sizeof(unsigned long long), st));
        R.stats = ctx->render_stats.ptr;
    }
    if (aux) {
        CK(ctx->accum_direct.reserve(pixels));
        CK(ctx->accum_albedo.reserve(pixels));
        CK(cudaMemsetAsync(ctx->accum_direct.ptr, 0, sizeof(float4) * pixels, st));
        CK(cudaMemsetAsync(ctx->accum_albedo.ptr, 0, sizeof(float4) * pixels, st));
        R.accum_direct = ctx->accum_direct.ptr;
        R.accum_albedo = ctx->accum_albedo.ptr;
    }

    MlpDev mlp = {};
    if (cache_depth) {
        const uint32_t train_cap = cap / train_every * 2u + 1024u;
        const uint32_t rec_cap = std::max<uint32_t>(1u, train_steps) * train_batch;
        CK(ctx->train_slot.reserve(cap));
        CK(ctx->rec_of.reserve((size_t)train_cap * (depth_max + 1)));
        CK(ctx->s_meta.reserve((size_t)cap * nl));
        CK(ctx->rec_feat.reserve((size_t)rec_cap * kMlpRaw));
        CK(ctx->rec_tgt.reserve((size_t)rec_cap * 3));
        CK(ctx->rec_beta.reserve(rec_cap));
        CK(ctx->qry_feat.reserve((size_t)cap * kMlpRaw));
        CK(ctx->qry_out.reserve((size_t)cap * 3));
        CK(ctx->qry_beta.reserve(cap));
        CK(ctx->qry_meta.reserve(cap));
        CK(ctx->mlp_enc.reserve((size_t)cap * kGridLevels));
        if (!hash_cache) {
            int rc = mlp_reserve_train(ctx, train_batch);
            if (rc) return rc;
        }
        R.cache_depth = cache_depth;
        R.train_every = train_every;
        R.train_tail = train_tail;
        R.qry_meta = ctx->qry_meta.ptr;
        if (hash_cache) {
            if (!ctx->hc_keys.ptr) return fail(ctx, ILG_ESTATE, "render: hash cache not reset (ilg_hash_cache_reset)");
            R.hc_keys = ctx->hc_keys.ptr;
            R.hc_vals = ctx->hc_vals.ptr;
            R.hc_dropped = ctx->counts.ptr + 8;
        }
        R.scene_lo = make_float3(ctx->scene_lo[0], ctx->scene_lo[1], ctx->scene_lo[2]);
        R.scene_inv_ext = make_float3(1.f / std::max(ctx->scene_hi[0] - ctx->scene_lo[0], 1e-20f),
                                      1.f / std::max(ctx->scene_hi[1] - ctx->scene_lo[1], 1e-20f),
                                      1.f / std::max(ctx->scene_hi[2] - ctx->scene_lo[2], 1e-20f));
        R.train_slot = ctx->train_slot.ptr;
        R.train_count = ctx->counts.ptr + 3;
        R.train_cap = train_cap;
        R.rec_of = ctx->rec_of.ptr;
        R.rec_feat = ctx->rec_feat.ptr;
        R.rec_beta = ctx->rec_beta.ptr;
        R.rec_tgt = ctx->rec_tgt.ptr;
        R.rec_count = ctx->counts.ptr + 4;
        R.rec_cap = rec_cap;
        R.qry_feat = ctx->qry_feat.ptr;
        R.qry_beta = ctx->qry_beta.ptr;
        R.qry_out = ctx->qry_out.ptr;
        R.qry_count = ctx->counts.ptr + 5;
        R.s_meta = ctx->s_meta.ptr;
        CK(cudaMemsetAsync(R.rec_count, 0, sizeof(uint32_t), st));
        mlp = ctx->mlp_view();
    }


    // The frame (every wave, every bounce) is one CUDA graph. Nothing in it
    // depends on the host between launches (queue counts stay on the device),
    // so a call whose launch configuration equals the previous one replays
    // the instantiated graph; a different one is captured afresh.
    uint32_t launches = 0;
    unsigned char key[sizeof(RenderDev) + sizeof(MlpDev) + 4 * sizeof(uint64_t)];
    {
        const uint64_t extra[4] = {cap, total, block, cache_depth | (one_launch ? 0x100000000ull : 0ull)};
        memcpy(key, &R, sizeof(RenderDev));
        memcpy(key + sizeof(RenderDev), &mlp, sizeof(MlpDev));
        memcpy(key + sizeof(RenderDev) + sizeof(MlpDev), extra, sizeof(extra));
    }
    if (!ctx->graph_exec || ctx->graph_key.size() != sizeof(key) || memcmp(ctx->graph_key.data(), key, sizeof(key))) {
        ctx->drop_graph();
        if (one_launch) CK(ctx->persist_next.reserve(1));
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
        cudaError_t ce = cudaSuccess;
        if (one_launch) {
            ce = render_persistent(R, total, ctx->persist_next.ptr, &launches, st);
        } else {
            for (uint64_t g0 = 0; g0 < total && ce == cudaSuccess; g0 += cap) {
                const uint32_t k = (uint32_t)std::min<uint64_t>(cap, total - g0);
                ce = render_wave(R, k, g0, st, &launches, cache_depth ? &mlp : nullptr, block);
            }
        }
        cudaGraph_t graph = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(st, &graph);
        if (ce == cudaSuccess) ce = ee;
        if (ce == cudaSuccess) ce = cudaGraphInstantiate(&ctx->graph_exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (ce != cudaSuccess) {
            ctx->graph_exec = nullptr;
            CK(ce);
        }
        ctx->graph_key.assign(key, key + sizeof(key));
        ctx->graph_kernels = launches;
    } else {
        launches = ctx->graph_kernels;
    }
    CK(cudaGraphLaunch(ctx->graph_exec, st));
    if (cache_depth) {
        // online training on this call's records (the next call renders with the update)
        uint32_t n_rec = 0;
        CK(cudaMemcpyAsync(&n_rec, R.rec_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        n_rec = std::min(n_rec, R.rec_cap);
        ctx->last_train_records = n_rec;
        ctx->last_hash_update = hash_cache;
        if (hash_cache) {
            CK(cudaMemsetAsync(R.hc_dropped, 0, sizeof(uint32_t), st));
            CK(hash_cache_update(R, n_rec, st));
            launches += 1;
            train_epochs = 0;
        }
        for (uint32_t ep = 0; ep < train_epochs; ep++)
        for (uint32_t s = 0; s < train_steps && (uint64_t)s * train_batch < n_rec; s++) {
            const uint32_t nb = std::min(train_batch, n_rec - s * train_batch);
            CK(mlp_grads(mlp, R.rec_feat + (size_t)s * train_batch * kMlpRaw, R.rec_tgt + (size_t)s * train_batch * 3,
                         nb, st));
            ctx->mlp_step++;
            CK(mlp_adam(mlp, ctx->mlp_step, ctx->mlp_lr, st));
            launches += 9;
        }
    }
    ctx->last_render_launches = launches;
    return ILG_OK;
}

}  // extern "C"

namespace {

// One scene, one region: the body of ilg_render and ilg_render_region.
int render_one(ilg_ctx *ctx, const ilg_camera_frame &frame, const ilg_render_opts *opts, const ilg_region &reg,
               float *final_rgb, float *direct_rgb, float *albedo_rgb, uint32_t flags,
               const float4 *ray_o = nullptr, const float4 *ray_d = nullptr)
{
    ctx->counted = (flags & ILG_RENDER_COUNT) != 0;
    const bool hash_cache = (flags & ILG_RENDER_HASH_CACHE) != 0;
    const uint32_t cache_depth = opts->cache_depth;
    if (hash_cache && !cache_depth) return fail(ctx, ILG_EINVAL, "ilg_render: ILG_RENDER_HASH_CACHE needs cache_depth");
    if (cache_depth) {
        if (!hash_cache && !ctx->mlp_ready)
            return fail(ctx, ILG_ESTATE, "ilg_render: cache_depth set but ilg_mlp_init not called");
        if (hash_cache && !ctx->hc_keys.ptr)
            return fail(ctx, ILG_ESTATE, "ilg_render: ILG_RENDER_HASH_CACHE but ilg_hash_cache_reset not called");
        if (cache_depth >= opts->max_depth)
            return fail(ctx, ILG_EINVAL, "ilg_render: cache_depth %u must be below max_depth %u", cache_depth, opts->max_depth);
        if (opts->train_tail > 64) return fail(ctx, ILG_EINVAL, "ilg_render: train_tail %u above 64", opts->train_tail);
        if (opts->train_epochs > 64)
            return fail(ctx, ILG_EINVAL, "ilg_render: train_epochs %u above 64", opts->train_epochs);
    }
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    std::vector<SceneRec> recs(1);
    int rc = prepare_scene(ctx, ctx, frame, opts->width, opts->height, reg.x, reg.y, reg.width, reg.height,
                           opts->spp, opts->max_depth, opts->epsilon, opts->seed, opts->sky, st, recs[0]);
    if (rc) return rc;
    recs[0].ray_o = ray_o;
    recs[0].ray_d = ray_d;
    const uint32_t wh = recs[0].wh;
    const bool aux = direct_rgb || albedo_rgb;
    rc = run_render(ctx, recs, opts->paths_per_wave, 128, cache_depth, opts->train_every ? opts->train_every : 16u,
                    opts->train_steps, opts->train_batch ? opts->train_batch : 16384u, nullptr, aux,
                    ctx->counted, opts->train_tail, opts->train_epochs ? opts->train_epochs : 1u, hash_cache,
                    (flags & ILG_RENDER_PERSISTENT) != 0);
    if (rc) return rc;
    const bool dev = (flags & ILG_DEVICE_PTRS) != 0;
    const float4 *sums[3] = {ctx->accum.ptr, ctx->accum_direct.ptr, ctx->accum_albedo.ptr};
    float *outs[3] = {final_rgb, direct_rgb, albedo_rgb};
    if (!dev) CK(ctx->out_dev.reserve(3ull * wh));
    for (int k = 0; k < 3; k++) {
        if (!outs[k]) continue;
        float *dst = dev ? outs[k] : ctx->out_dev.ptr;
        CK(render_resolve(sums[k], wh, 1.f / opts->spp, dst, st));
        ctx->last_render_launches += 1;
        if (!dev) {
            CK(cudaMemcpyAsync(outs[k], dst, 12ull * wh, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));  // out_dev is reused for the next output
        }
    }
    if (!dev) return ctx->check_device_error();
    return ILG_OK;
}

}  // namespace

extern "C" {

int ilg_camera_frame_of(const ilg_camera *cam, ilg_camera_frame *out)
{
    if (!cam || !out) return ILG_EINVAL;
    camera_frame_of(*cam, *out);
    return ILG_OK;
}

int ilg_render(ilg_ctx *ctx, const ilg_camera *cam, const ilg_render_opts *opts, float *out_rgb, uint32_t flags)
{
    if (!ctx) return ILG_EINVAL;
    if (!cam || !opts || !out_rgb) return fail(ctx, ILG_EINVAL, "ilg_render: null argument");
    if (flags & ~(ILG_DEVICE_PTRS | ILG_RENDER_COUNT | ILG_RENDER_HASH_CACHE | ILG_RENDER_PERSISTENT))
        return fail(ctx, ILG_EINVAL, "ilg_render: unknown flags 0x%x", flags);
    ilg_camera_frame frame;
    camera_frame_of(*cam, frame);
    const ilg_region whole = {0u, 0u, opts->width, opts->height};
    return render_one(ctx, frame, opts, whole, out_rgb, nullptr, nullptr, flags);
}

int ilg_render_counts(ilg_ctx *ctx, uint64_t counts[6])
{
    if (!ctx || !counts) return ILG_EINVAL;
    if (!ctx->counted) return fail(ctx, ILG_ESTATE, "ilg_render_counts: the last render was not counted");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(counts, ctx->render_stats.ptr, 6 * sizeof(uint64_t), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return ILG_OK;
}

int ilg_render_region(ilg_ctx *ctx, const ilg_camera_frame *frame, const ilg_render_opts *opts,
                      const ilg_region *region, float *final_rgb, float *direct_rgb, float *albedo_rgb,
                      uint32_t flags)
{
    if (!ctx) return ILG_EINVAL;
    if (!frame || !opts || !region || !final_rgb) return fail(ctx, ILG_EINVAL, "ilg_render_region: null argument");
    if (flags & ~(ILG_DEVICE_PTRS | ILG_RENDER_HASH_CACHE))
        return fail(ctx, ILG_EINVAL, "ilg_render_region: unknown flags 0x%x", flags);
    return render_one(ctx, *frame, opts, *region, final_rgb, direct_rgb, albedo_rgb, flags);
}

int ilg_radiance(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n,
                 const ilg_render_opts *opts, float *final_rgb, float *direct_rgb, float *albedo_rgb, uint32_t flags)
{
    if (!ctx) return ILG_EINVAL;
    if (!ray_o_tmin || !ray_d_tmax || !opts || !final_rgb) return fail(ctx, ILG_EINVAL, "ilg_radiance: null argument");
    if (flags & ~(ILG_DEVICE_PTRS | ILG_RENDER_HASH_CACHE))
        return fail(ctx, ILG_EINVAL, "ilg_radiance: unknown flags 0x%x", flags);
    if (n == 0) return ILG_OK;
    if (n > (1u << 26)) return fail(ctx, ILG_EINVAL, "ilg_radiance: %u rays exceed 2^26", n);
    const bool dev = (flags & ILG_DEVICE_PTRS) != 0;
    if (((uintptr_t)ray_o_tmin | (uintptr_t)ray_d_tmax) & 15u)
        return fail(ctx, ILG_EINVAL, "ilg_radiance: ray arrays must be 16-byte aligned");
    CK(cudaSetDevice(ctx->device));
    const float4 *ro = (const float4 *)ray_o_tmin, *rd = (const float4 *)ray_d_tmax;
    if (!dev) {
        CK(ctx->ro.reserve(n));
        CK(ctx->rd.reserve(n));
        CK(cudaMemcpyAsync(ctx->ro.ptr, ray_o_tmin, 16ull * n, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(ctx->rd.ptr, ray_d_tmax, 16ull * n, cudaMemcpyHostToDevice, ctx->stream));
        ro = ctx->ro.ptr;
        rd = ctx->rd.ptr;
    }
    ilg_render_opts o = *opts;
    o.width = n;
    o.height = 1;
    ilg_camera_frame frame;
    memset(&frame, 0, sizeof(frame));
    const ilg_region whole = {0u, 0u, n, 1u};
    return render_one(ctx, frame, &o, whole, final_rgb, direct_rgb, albedo_rgb, flags, ro, rd);
}

int ilg_last_train_stats(ilg_ctx *ctx, uint32_t *records, uint32_t *dropped)
{
    if (!ctx || !records || !dropped) return ILG_EINVAL;
    *records = ctx->last_train_records;
    *dropped = 0;
    if (ctx->last_hash_update && ctx->counts.ptr) {
        CK(cudaSetDevice(ctx->device));
        CK(cudaMemcpyAsync(dropped, ctx->counts.ptr + 8, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return ILG_OK;
}

int ilg_hash_cache_reset(ilg_ctx *ctx)
{
    if (!ctx) return ILG_EINVAL;
    CK(cudaSetDevice(ctx->device));
    CK(ctx->hc_keys.reserve(kHashCacheCells));
    CK(ctx->hc_vals.reserve(kHashCacheCells));
    CK(cudaMemsetAsync(ctx->hc_keys.ptr, 0, sizeof(unsigned long long) * kHashCacheCells, ctx->stream));
    CK(cudaMemsetAsync(ctx->hc_vals.ptr, 0, sizeof(float4) * kHashCacheCells, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return ILG_OK;
}

int ilg_render_batch(ilg_ctx *runner, const ilg_batch_item *items, uint32_t n, uint32_t paths_per_wave,
                     uint32_t block, uint32_t flags)
{
    if (!runner) return ILG_EINVAL;
    if (!items || n == 0 || n > 4096) return fail(runner, ILG_EINVAL, "ilg_render_batch: need 1..4096 items");
    if (flags & ~(ILG_DEVICE_PTRS | ILG_RENDER_COUNT | ILG_RENDER_PERSISTENT))
        return fail(runner, ILG_EINVAL, "ilg_render_batch: unknown flags 0x%x", flags);
    if (block != 0 && block != 64 && block != 128 && block != 256)
        return fail(runner, ILG_EINVAL, "ilg_render_batch: block must be 64, 128 or 256");
    CK2(runner, cudaSetDevice(runner->device));
    cudaStream_t st = runner->stream;
    std::vector<SceneRec> recs(n);
    for (uint32_t i = 0; i < n; i++) {
        const ilg_batch_item &it = items[i];
        if (!it.out_rgb) return fail(runner, ILG_EINVAL, "ilg_render_batch: item %u has no output", i);
        ilg_camera_frame frame;
        camera_frame_of(it.camera, frame);
        int rc = prepare_scene(runner, it.scene, frame, it.width, it.height, 0, 0, it.width, it.height, it.spp,
                               it.max_depth, it.epsilon, it.seed, it.sky, st, recs[i]);
        if (rc) return rc;
    }
    runner->counted = (flags & ILG_RENDER_COUNT) != 0;
    int rc = run_render(runner, recs, paths_per_wave, block ? block : 128, 0, 16, 0, 16384, nullptr, false,
                        runner->counted, 0, 1, false, (flags & ILG_RENDER_PERSISTENT) != 0);
    if (rc) return rc;
    uint32_t max_wh = 0;
    for (auto &S : recs) max_wh = std::max(max_wh, S.wh);
    if (!(flags & ILG_DEVICE_PTRS)) CK2(runner, runner->out_dev.reserve(3ull * max_wh));
    for (uint32_t i = 0; i < n; i++) {
        const SceneRec &S = recs[i];
        float *dst = (flags & ILG_DEVICE_PTRS) ? items[i].out_rgb : runner->out_dev.ptr;
        CK2(runner, render_resolve(runner->accum.ptr + S.pixel_base, S.wh, 1.f / S.spp, dst, st));
        if (!(flags & ILG_DEVICE_PTRS))
            CK2(runner, cudaMemcpyAsync(items[i].out_rgb, dst, 12ull * S.wh, cudaMemcpyDeviceToHost, st));
        if (!(flags & ILG_DEVICE_PTRS)) CK2(runner, cudaStreamSynchronize(st));  // runner->out_dev is reused per item
    }
    runner->last_render_launches += n;
    if (!(flags & ILG_DEVICE_PTRS)) return runner->check_device_error();
    return ILG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// post-processing: progressive accumulation and tone mapping
// ---------------------------------------------------------------------------
extern "C" {

int ilg_accumulate_reset(ilg_ctx *ctx)
{
    if (!ctx) return ILG_EINVAL;
    CK(cudaSetDevice(ctx->device));
    if (ctx->post_pixels) CK(cudaMemsetAsync(ctx->post_acc.ptr, 0, 12ull * ctx->post_pixels, ctx->stream));
    ctx->post_frames = 0;
    return ILG_OK;
}

int ilg_accumulate(ilg_ctx *ctx, const float *frame_rgb, uint32_t n_pixels, float *out_rgb, uint32_t flags)
{
    if (!ctx) return ILG_EINVAL;
    if (!frame_rgb || !out_rgb || n_pixels == 0 || n_pixels > (1u << 28))
        return fail(ctx, ILG_EINVAL, "ilg_accumulate: bad arguments");
    if (flags & ~ILG_DEVICE_PTRS) return fail(ctx, ILG_EINVAL, "ilg_accumulate: unknown flags 0x%x", flags);
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    if (n_pixels != ctx->post_pixels) {  // a new image size starts a new accumulation
        CK(ctx->post_acc.reserve(3ull * n_pixels));
        CK(cudaMemsetAsync(ctx->post_acc.ptr, 0, 12ull * n_pixels, st));
        ctx->post_pixels = n_pixels;
        ctx->post_frames = 0;
    }
    ctx->post_frames++;
    const bool dev = (flags & ILG_DEVICE_PTRS) != 0;
    const float *in = frame_rgb;
    float *out = out_rgb;
    if (!dev) {
        CK(ctx->post_in.reserve(3ull * n_pixels));
        CK(ctx->post_out.reserve(3ull * n_pixels));
        CK(cudaMemcpyAsync(ctx->post_in.ptr, frame_rgb, 12ull * n_pixels, cudaMemcpyHostToDevice, st));
        in = ctx->post_in.ptr;
        out = ctx->post_out.ptr;
    }
    CK(post_accumulate(in, ctx->post_acc.ptr, out, n_pixels, ctx->post_frames, st));
    if (!dev) {
        CK(cudaMemcpyAsync(out_rgb, out, 12ull * n_pixels, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    return ILG_OK;
}

int ilg_tonemap(ilg_ctx *ctx, const float *in_rgb, uint32_t n_pixels, float *out_rgb, uint32_t op, uint32_t flags)
{
    if (!ctx) return ILG_EINVAL;
    if (!in_rgb || !out_rgb || n_pixels == 0 || n_pixels > (1u << 28))
        return fail(ctx, ILG_EINVAL, "ilg_tonemap: bad arguments");
    if (op > ILG_TONE_DRAGO) return fail(ctx, ILG_EINVAL, "ilg_tonemap: unknown operator %u", op);
    if (flags & ~ILG_DEVICE_PTRS) return fail(ctx, ILG_EINVAL, "ilg_tonemap: unknown flags 0x%x", flags);
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const bool dev = (flags & ILG_DEVICE_PTRS) != 0;
    const float *in = in_rgb;
    float *out = out_rgb;
    if (!dev) {
        CK(ctx->post_in.reserve(3ull * n_pixels));
        CK(ctx->post_out.reserve(3ull * n_pixels));
        CK(cudaMemcpyAsync(ctx->post_in.ptr, in_rgb, 12ull * n_pixels, cudaMemcpyHostToDevice, st));
        in = ctx->post_in.ptr;
        out = ctx->post_out.ptr;
    }
    CK(ctx->post_scratch.reserve(post_scratch_floats(n_pixels)));
    CK(post_tonemap(in, out, n_pixels, op, ctx->post_scratch.ptr, st));
    if (!dev) {
        CK(cudaMemcpyAsync(out_rgb, out, 12ull * n_pixels, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    return ILG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// radiance-cache network
// ---------------------------------------------------------------------------
namespace {

int mlp_reserve_train(ilg_ctx *ctx, uint32_t n)
{
    const size_t cap = ((size_t)n + 15) / 16 * 16;
    if (ctx->mlp_xcm.cap >= cap * kMlpIn) return ILG_OK;
    CK(ctx->mlp_xcm.reserve(cap * kMlpIn));
    CK(ctx->mlp_hcm.reserve(cap * 5 * kMlpHid));
    CK(ctx->mlp_dzcm.reserve(cap * (5 * kMlpHid + kMlpOutP)));
    return ILG_OK;
}

}  // namespace

extern "C" {

int ilg_mlp_init(ilg_ctx *ctx, uint32_t seed, float learning_rate)
{
    return ilg_mlp_init_encoding(ctx, seed, learning_rate, ILG_MLP_ENC_HASHGRID);
}

int ilg_mlp_init_encoding(ilg_ctx *ctx, uint32_t seed, float learning_rate, uint32_t encoding)
{
    if (!ctx) return ILG_EINVAL;
    if (!(learning_rate > 0.f)) return fail(ctx, ILG_EINVAL, "ilg_mlp_init: learning rate must be > 0");
    if (encoding != ILG_MLP_ENC_HASHGRID && encoding != ILG_MLP_ENC_FREQ12)
        return fail(ctx, ILG_EINVAL, "ilg_mlp_init: unknown encoding %u", encoding);
    static_assert(ILG_MLP_ENC_HASHGRID == kEncHashGrid && ILG_MLP_ENC_FREQ12 == kEncFreq12, "encoding ids");
    CK(cudaSetDevice(ctx->device));
    ctx->mlp_encoding = encoding;
    ctx->drop_graph();
    CK(ctx->mlp_w.reserve(kMlpParams)); CK(ctx->mlp_m.reserve(kMlpParams)); CK(ctx->mlp_v.reserve(kMlpParams));
    CK(ctx->mlp_grad.reserve(kMlpParams)); CK(ctx->mlp_loss.reserve(1));
    CK(ctx->mlp_wf.reserve(kFwdElems)); CK(ctx->mlp_wb.reserve(kBwdElems)); CK(ctx->mlp_wu.reserve(kUmmaElems));
    CK(ctx->mlp_wv.reserve(kUmmaBwdElems));
    CK(ctx->mlp_grid.reserve(kGridParams)); CK(ctx->mlp_grid_grad.reserve(kGridParams));
    CK(ctx->mlp_grid_m.reserve(kGridParams)); CK(ctx->mlp_grid_v.reserve(kGridParams));
    CK(mlp_init(ctx->mlp_view(), seed, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->mlp_ready = true;
    ctx->mlp_step = 0;
    ctx->mlp_lr = learning_rate;
    return ILG_OK;
}

// which = 0: the grid features, 1: their gradient from the last ilg_mlp_grads.
static int grid_copy(ilg_ctx *ctx, float *dst, const float *src, int which)
{
    if (!ctx || (!dst && !src)) return ILG_EINVAL;
    if (!ctx->mlp_ready) return fail(ctx, ILG_ESTATE, "ilg_mlp grid: network not initialised");
    CK(cudaSetDevice(ctx->device));
    float *dev = which == 0 ? ctx->mlp_grid.ptr : ctx->mlp_grid_grad.ptr;
    if (dst) CK(cudaMemcpyAsync(dst, dev, sizeof(float) * kGridParams, cudaMemcpyDeviceToHost, ctx->stream));
    else CK(cudaMemcpyAsync(dev, src, sizeof(float) * kGridParams, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return ILG_OK;
}

int ilg_mlp_get_grid(ilg_ctx *ctx, float *grid) { return grid_copy(ctx, grid, nullptr, 0); }
int ilg_mlp_set_grid(ilg_ctx *ctx, const float *grid) { return grid_copy(ctx, nullptr, grid, 0); }
int ilg_mlp_get_grid_grads(ilg_ctx *ctx, float *grad) { return grid_copy(ctx, grad, nullptr, 1); }

int ilg_mlp_get_params(ilg_ctx *ctx, float *params)
{
    if (!ctx || !params) return ILG_EINVAL;
    if (!ctx->mlp_ready) return fail(ctx, ILG_ESTATE, "ilg_mlp_get_params: network not initialised");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(params, ctx->mlp_w.ptr, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return ILG_OK;
}

int ilg_mlp_set_params(ilg_ctx *ctx, const float *params)
{
    if (!ctx || !params) return ILG_EINVAL;
    if (!ctx->mlp_ready) return fail(ctx, ILG_ESTATE, "ilg_mlp_set_params: network not initialised");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(ctx->mlp_w.ptr, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice, ctx->stream));
    CK(mlp_refresh_copies(ctx->mlp_view(), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return ILG_OK;
}

int ilg_mlp_infer(ilg_ctx *ctx, const float *raw, uint32_t n, float *out, uint32_t flags)
{
    if (!ctx) return ILG_EINVAL;
    if (!ctx->mlp_ready) return fail(ctx, ILG_ESTATE, "ilg_mlp_infer: network not initialised");
    if (n == 0) return ILG_OK;
    if (!raw || !out) return fail(ctx, ILG_EINVAL, "ilg_mlp_infer: null array");
    if (flags & ~(ILG_DEVICE_PTRS | ILG_MLP_WARP_MMA)) return fail(ctx, ILG_EINVAL, "ilg_mlp_infer: unknown flags");
    if ((flags & ILG_DEVICE_PTRS) && ((uintptr_t)raw & 15u))
        return fail(ctx, ILG_EINVAL, "ilg_mlp_infer: device query rows must start 16-byte aligned");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const bool warp_mma = (flags & ILG_MLP_WARP_MMA) != 0;
    if (!warp_mma) CK(ctx->mlp_enc.reserve((size_t)n * kGridLevels));
    auto run = [&](const float *r, float *o) {
        return warp_mma ? mlp_infer_warp(ctx->mlp_view(), r, n, o, st) : mlp_infer(ctx->mlp_view(), r, n, o, st);
    };
    if (flags & ILG_DEVICE_PTRS) {
        CK(run(raw, out));
        return ILG_OK;
    }
    CK(ctx->mlp_raw.reserve((size_t)n * kMlpRaw));
    CK(ctx->mlp_out.reserve((size_t)n * 3));
    CK(cudaMemcpyAsync(ctx->mlp_raw.ptr, raw, sizeof(float) * kMlpRaw * n, cudaMemcpyHostToDevice, st));
    CK(run(ctx->mlp_raw.ptr, ctx->mlp_out.ptr));
    CK(cudaMemcpyAsync(out, ctx->mlp_out.ptr, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return ctx->check_device_error();
}

static int mlp_grads_common(ilg_ctx *ctx, const float *raw, const float *target, uint32_t n, uint32_t flags,
                            float *loss)
{
    if (!ctx->mlp_ready) return fail(ctx, ILG_ESTATE, "network not initialised");
    if (n == 0 || !raw || !target) return fail(ctx, ILG_EINVAL, "empty batch or null array");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    int rc = mlp_reserve_train(ctx, n);
    if (rc) return rc;
    const float *draw = raw, *dtgt = target;
    if (!(flags & ILG_DEVICE_PTRS)) {
        CK(ctx->mlp_raw.reserve((size_t)n * kMlpRaw));
        CK(ctx->mlp_tgt.reserve((size_t)n * 3));
        CK(cudaMemcpyAsync(ctx->mlp_raw.ptr, raw, sizeof(float) * kMlpRaw * n, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->mlp_tgt.ptr, target, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, st));
        draw = ctx->mlp_raw.ptr;
        dtgt = ctx->mlp_tgt.ptr;
    }
    if ((flags & ILG_DEVICE_PTRS) && ((uintptr_t)draw & 15u) && !(flags & ILG_MLP_WARP_MMA))
        return fail(ctx, ILG_EINVAL, "device training rows must start 16-byte aligned");
    CK(mlp_grads(ctx->mlp_view(), draw, dtgt, n, st, (flags & ILG_MLP_WARP_MMA) != 0));
    if (loss) {
        CK(cudaMemcpyAsync(loss, ctx->mlp_loss.ptr, sizeof(float), cudaMemcpyDefault, st));
        if (!(flags & ILG_DEVICE_PTRS)) CK(cudaStreamSynchronize(st));
    }
    return ILG_OK;
}

int ilg_mlp_grads(ilg_ctx *ctx, const float *raw, const float *target, uint32_t n, float *grad, float *loss,
                  uint32_t flags)
{
    if (!ctx) return ILG_EINVAL;
    if (!grad) return fail(ctx, ILG_EINVAL, "ilg_mlp_grads: null grad");
    int rc = mlp_grads_common(ctx, raw, target, n, flags, loss);
    if (rc) return rc;
    // (cudaMemcpyDefault: grad is a device pointer with ILG_DEVICE_PTRS)
    CK(cudaMemcpyAsync(grad, ctx->mlp_grad.ptr, sizeof(float) * kMlpParams, cudaMemcpyDefault, ctx->stream));
    if (!(flags & ILG_DEVICE_PTRS)) CK(cudaStreamSynchronize(ctx->stream));
    return ILG_OK;
}

int ilg_mlp_train_step(ilg_ctx *ctx, const float *raw, const float *target, uint32_t n, float *loss, uint32_t flags)
{
    if (!ctx) return ILG_EINVAL;
    int rc = mlp_grads_common(ctx, raw, target, n, flags, loss);
    if (rc) return rc;
    ctx->mlp_step++;
    CK(mlp_adam(ctx->mlp_view(), ctx->mlp_step, ctx->mlp_lr, ctx->stream));
    if (!(flags & ILG_DEVICE_PTRS)) CK(cudaStreamSynchronize(ctx->stream));
    return ILG_OK;
}

}  // extern "C"
