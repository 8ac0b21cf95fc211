// ilg_intersect_noalloc: the closest-hit query from host buffers without any
// device allocation.
//
// ilg_intersect stages host rays and hits through device buffers that the
// context grows with cudaMalloc on demand. Some callers cannot allow that at
// query time: a renderer that runs its per-frame queries inside a section
// where the device memory budget is fixed and fully handed out up front, or a
// host process whose device memory is owned by another allocator (a caching
// pool that would fail or stall a cudaMalloc issued behind its back). For
// them this entry point stages through one file-scope device array of fixed
// size instead, so the call performs copies, two small memsets and one kernel
// launch and nothing else.
//
// Limits and sharing:
//   * at most ILG_NOALLOC_MAX_RAYS rays per call; larger batches are rejected
//     with ILG_EINVAL before any device work;
//   * the array exists once per GPU that loads this library and stays
//     resident until the process exits (12 MiB + 256 bytes);
//   * ilg_create loads the array's module on its device and looks up the
//     array's device address there (cudaGetSymbolAddress), so the array
//     becomes resident when the first context on a device is created, and a
//     query never triggers that load itself;
//   * every call on a device uses the same array and leaves the previous
//     call's rays and hits in it. The ray counter of the persistent kernel
//     and the call's error word (also in the array) are cleared on the
//     stream before the launch; everything else a call reads it has written
//     itself first;
//   * calls whose device work overlaps (two contexts on one device used from
//     two threads, or calls on different streams) race on the array: the
//     caller must serialise them.
#include "ilg.h"

#include "ctx.cuh"
#include "trace_api.cuh"

namespace {

constexpr uint32_t kMaxRays = ILG_NOALLOC_MAX_RAYS;
// rays (o4, d4) then hits (prim, t, u, v): 32 + 16 bytes per ray; then one
// 256-byte block: word 0 = the persistent kernel's ray counter, word 1 = this
// call's device error flags
constexpr size_t kRayBytes = (size_t)kMaxRays * 48;
constexpr size_t kScratchBytes = kRayBytes + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

}  // namespace

namespace ilg {

// Called by ilg_create with `device` current: the device address of this
// device's copy of g_noalloc_scratch (the host-side name is only a stand-in
// and must never be handed to a kernel), and the traversal kernel's code
// loaded, so that a query loads nothing.
cudaError_t noalloc_prepare(void **out)
{
    *out = nullptr;
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    if ((e = preload_closest_dyn()) != cudaSuccess) return e;
    *out = p;
    return cudaSuccess;
}

}  // namespace ilg

#define NA_CK(call)                                                                                \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            snprintf(ctx->err, sizeof(ctx->err), "ilg_intersect_noalloc: %s: %s", #call,           \
                     cudaGetErrorString(e_));                                                      \
            return ILG_ECUDA;                                                                      \
        }                                                                                          \
    } while (0)

extern "C" int ilg_intersect_noalloc(ilg_ctx *ctx, const float *ray_o_tmin, const float *ray_d_tmax, uint32_t n,
                                     int32_t *prim, float *t, float *u, float *v)
{
    if (!ctx) return ILG_EINVAL;
    if (n > kMaxRays) {
        snprintf(ctx->err, sizeof(ctx->err), "ilg_intersect_noalloc: %u rays exceed the maximum of %u per call", n,
                 kMaxRays);
        return ILG_EINVAL;
    }
    if (!ctx->built) {
        snprintf(ctx->err, sizeof(ctx->err), "ilg_intersect_noalloc: scene not built");
        return ILG_ESTATE;
    }
    if (n == 0) return ILG_OK;
    if (!ray_o_tmin || !ray_d_tmax || !prim || !t || !u || !v) {
        snprintf(ctx->err, sizeof(ctx->err), "ilg_intersect_noalloc: null array");
        return ILG_EINVAL;
    }
    if (!ctx->noalloc_scratch) {
        snprintf(ctx->err, sizeof(ctx->err),
                 "ilg_intersect_noalloc: the fixed device array is unavailable (its lookup in ilg_create failed)");
        return ILG_ECUDA;
    }
    NA_CK(cudaSetDevice(ctx->device));
    unsigned char *b = (unsigned char *)ctx->noalloc_scratch;
    float4 *ro = (float4 *)b;
    float4 *rd = (float4 *)(b + (size_t)kMaxRays * 16);
    int32_t *hprim = (int32_t *)(b + (size_t)kMaxRays * 32);
    float *ht = (float *)(b + (size_t)kMaxRays * 36);
    float *hu = (float *)(b + (size_t)kMaxRays * 40);
    float *hv = (float *)(b + (size_t)kMaxRays * 44);
    uint32_t *next = (uint32_t *)(b + kRayBytes);
    uint32_t *derr = next + 1;
    cudaStream_t st = ctx->stream;
    uint32_t flags = 0;
    NA_CK(cudaMemsetAsync(derr, 0, sizeof(uint32_t), st));
    NA_CK(cudaMemcpyAsync(ro, ray_o_tmin, 16ull * n, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(rd, ray_d_tmax, 16ull * n, cudaMemcpyHostToDevice, st));
    NA_CK(ilg::launch_closest_dyn(ctx->view(), ro, rd, n, hprim, ht, hu, hv, next, derr, st));
    NA_CK(cudaMemcpyAsync(prim, hprim, 4ull * n, cudaMemcpyDeviceToHost, st));
    NA_CK(cudaMemcpyAsync(t, ht, 4ull * n, cudaMemcpyDeviceToHost, st));
    NA_CK(cudaMemcpyAsync(u, hu, 4ull * n, cudaMemcpyDeviceToHost, st));
    NA_CK(cudaMemcpyAsync(v, hv, 4ull * n, cudaMemcpyDeviceToHost, st));
    NA_CK(cudaMemcpyAsync(&flags, derr, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    if (flags) {
        snprintf(ctx->err, sizeof(ctx->err),
                 "ilg_intersect_noalloc: device reported error flags 0x%x (bit0: traversal stack bound, bit1: "
                 "node/triangle index out of range, bit2: node visit budget)",
                 flags);
        return ILG_EOVERFLOW;
    }
    return ILG_OK;
}
