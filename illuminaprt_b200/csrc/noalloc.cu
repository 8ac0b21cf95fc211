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
// size instead, so the call performs copies and one kernel launch and nothing
// else.
//
// Limits and sharing:
//   * at most ILG_NOALLOC_MAX_RAYS rays per call; larger batches are rejected
//     with ILG_EINVAL before any device work;
//   * the array exists once per GPU that loads this library and stays
//     resident until the process exits (12 MiB);
//   * every call on a device uses the same array and leaves the previous
//     call's rays and hits in it; each call writes every element it later
//     reads, so nothing has to be cleared;
//   * calls whose device work overlaps (two contexts on one device used from
//     two threads, or calls on different streams) race on the array: the
//     caller must serialise them;
//   * the first call on a device looks the array's device address up with
//     cudaGetSymbolAddress (once per device, with that device current); make
//     that first call before any stream capture.
#include "ilg.h"

#include <mutex>

#include "ctx.cuh"
#include "trace_api.cuh"

namespace {

constexpr uint32_t kMaxRays = ILG_NOALLOC_MAX_RAYS;
// rays (o4, d4) then hits (prim, t, u, v): 32 + 16 bytes per ray
constexpr size_t kScratchBytes = (size_t)kMaxRays * 48;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_lock;
void *g_scratch_addr[kMaxDevices] = {};

// Device address of this device's copy of g_noalloc_scratch (the host-side
// name is only a stand-in and must never be handed to a kernel).
int scratch_for(int device, void **out, char *err, size_t err_len)
{
    if (device < 0 || device >= kMaxDevices) {
        snprintf(err, err_len, "ilg_intersect_noalloc: device %d out of range", device);
        return ILG_EINVAL;
    }
    std::lock_guard<std::mutex> g(g_lock);
    if (!g_scratch_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            snprintf(err, err_len, "ilg_intersect_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return ILG_ECUDA;
        }
        g_scratch_addr[device] = p;
    }
    *out = g_scratch_addr[device];
    return ILG_OK;
}

}  // namespace

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
    NA_CK(cudaSetDevice(ctx->device));
    void *base = nullptr;
    int rc = scratch_for(ctx->device, &base, ctx->err, sizeof(ctx->err));
    if (rc != ILG_OK) return rc;
    unsigned char *b = (unsigned char *)base;
    float4 *ro = (float4 *)b;
    float4 *rd = (float4 *)(b + (size_t)kMaxRays * 16);
    int32_t *hprim = (int32_t *)(b + (size_t)kMaxRays * 32);
    float *ht = (float *)(b + (size_t)kMaxRays * 36);
    float *hu = (float *)(b + (size_t)kMaxRays * 40);
    float *hv = (float *)(b + (size_t)kMaxRays * 44);
    cudaStream_t st = ctx->stream;
    NA_CK(cudaMemcpyAsync(ro, ray_o_tmin, 16ull * n, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(rd, ray_d_tmax, 16ull * n, cudaMemcpyHostToDevice, st));
    NA_CK(ilg::launch_closest(ctx->view(), ro, rd, n, hprim, ht, hu, hv, ctx->derr.ptr, nullptr, st));
    NA_CK(cudaMemcpyAsync(prim, hprim, 4ull * n, cudaMemcpyDeviceToHost, st));
    NA_CK(cudaMemcpyAsync(t, ht, 4ull * n, cudaMemcpyDeviceToHost, st));
    NA_CK(cudaMemcpyAsync(u, hu, 4ull * n, cudaMemcpyDeviceToHost, st));
    NA_CK(cudaMemcpyAsync(v, hv, 4ull * n, cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    return ctx->check_device_error();
}
