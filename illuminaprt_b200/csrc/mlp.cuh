// Online-trained radiance cache: a 96 -> 64 x 5 (ReLU) -> 3 MLP in BF16 with
// FP32 accumulation on the tensor cores (mlp.cu). The reference has no
// learned component; the closest analogue is its irradiance cache
// (Core/Integrator/ICIntegrator.*), which this does not reproduce.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace ilg {

// Raw features of one query (16 floats): position normalised to [0,1]^3 (3),
// outgoing direction (3), shading normal (3), roughness (1), albedo (3), pad (3).
constexpr int kMlpRaw = 16;
constexpr int kMlpIn = 96;     // encoded input width (82 used + constant 1 + zero pad)
constexpr int kMlpHid = 64;
constexpr int kMlpOutP = 8;    // output columns computed (3 used)
constexpr int kMlpLayers = 6;
constexpr int kMlpBands = 12;

__host__ __device__ constexpr int mlp_in(int l) { return l == 0 ? kMlpIn : kMlpHid; }
__host__ __device__ constexpr int mlp_out(int l) { return l == kMlpLayers - 1 ? kMlpOutP : kMlpHid; }
__host__ __device__ constexpr int mlp_off(int l)
{
    return l == 0 ? 0 : mlp_off(l - 1) + mlp_in(l - 1) * mlp_out(l - 1);
}
constexpr int kMlpParams = mlp_off(kMlpLayers);  // 23040 (row-major [in][out] per layer)

// forward copy: per layer [out][in + 8] bf16 (padded row stride avoids bank conflicts)
__host__ __device__ constexpr int fwd_stride(int l) { return mlp_in(l) + 8; }
__host__ __device__ constexpr int fwd_off(int l)
{
    return l == 0 ? 0 : fwd_off(l - 1) + mlp_out(l - 1) * fwd_stride(l - 1);
}
constexpr int kFwdElems = fwd_off(kMlpLayers);
// backward copy (layers 1..5): per layer [in][outB + 8], outB = out padded to 16
__host__ __device__ constexpr int bwd_outp(int l) { return mlp_out(l) < 16 ? 16 : mlp_out(l); }
__host__ __device__ constexpr int bwd_stride(int l) { return bwd_outp(l) + 8; }
__host__ __device__ constexpr int bwd_off(int l)
{
    return l <= 1 ? 0 : bwd_off(l - 1) + mlp_in(l - 1) * bwd_stride(l - 1);
}
constexpr int kBwdElems = bwd_off(kMlpLayers);
// tensor-core (tcgen05) copy: per layer W^T as N x K, K-major, in 8 x 8-element
// core matrices (no swizzle); the output layer is padded to N = 16
__host__ __device__ constexpr int umma_n(int l) { return l == kMlpLayers - 1 ? 16 : mlp_out(l); }
__host__ __device__ constexpr int umma_off(int l)
{
    return l == 0 ? 0 : umma_off(l - 1) + umma_n(l - 1) * mlp_in(l - 1);
}
constexpr int kUmmaElems = umma_off(kMlpLayers);

struct MlpDev {
    float *w;                 // FP32 master weights (kMlpParams)
    float *m, *v;             // Adam moments
    float *grad;              // FP32 gradient accumulator
    __nv_bfloat16 *wf;        // forward copy (kFwdElems)
    __nv_bfloat16 *wb;        // backward copy (kBwdElems)
    __nv_bfloat16 *wu;        // tensor-core copy (kUmmaElems)
    float *loss;              // [1] loss sum of the last step
    // training scratch, column-major [feature][row_padded]
    __nv_bfloat16 *xcm;       // kMlpIn x cap
    __nv_bfloat16 *hcm;       // 5 x kMlpHid x cap
    __nv_bfloat16 *dzcm;      // (5 x kMlpHid + kMlpOutP) x cap
    uint32_t cap;             // rows the scratch holds (multiple of 16)
    uint32_t *err;            // device error word (bounded waits)
};

// Encoded input columns (c, c+1), c even. Columns 0..71: for axis a and band
// b, column 24a + 2b is sin(2^b pi x_a) and the next cos(2^b pi x_a);
// 72..74 direction, 75..77 normal, 78 roughness, 79..81 albedo, 82 constant 1.
__device__ __forceinline__ float2 encode_pair(const float *f, int c)
{
    if (c < 72) {
        const int axis = c / 24, band = (c % 24) >> 1;
        const float x = axis == 0 ? f[0] : (axis == 1 ? f[1] : f[2]);
        float s, co;
        sincospif(ldexpf(x, band), &s, &co);
        return make_float2(s, co);
    }
    switch (c) {
    case 72: return make_float2(f[3], f[4]);
    case 74: return make_float2(f[5], f[6]);
    case 76: return make_float2(f[7], f[8]);
    case 78: return make_float2(f[9], f[10]);
    case 80: return make_float2(f[11], f[12]);
    case 82: return make_float2(1.f, 0.f);
    default: return make_float2(0.f, 0.f);
    }
}

// Host entry points (mlp.cu). All enqueue on `st`.
cudaError_t mlp_init(const MlpDev &M, uint32_t seed, cudaStream_t st);
cudaError_t mlp_refresh_copies(const MlpDev &M, cudaStream_t st);
// Inference (tcgen05 path). n_dev (optional): a device word holding the
// actual row count (<= n).
cudaError_t mlp_infer(const MlpDev &M, const float *raw, uint32_t n, float *out, cudaStream_t st,
                      const uint32_t *n_dev = nullptr);
// The same inference on warp-level mma.sync (the kernel training's forward uses).
cudaError_t mlp_infer_warp(const MlpDev &M, const float *raw, uint32_t n, float *out, cudaStream_t st,
                           const uint32_t *n_dev = nullptr);
// Forward + loss + backward + weight gradients into M.grad (zeroed first).
// Inference on the 5th-generation tensor cores (tcgen05.mma, accumulators in
// TMEM); err gets bit 64 set if a bounded wait ran out.
cudaError_t mlp_infer_tc(const MlpDev &M, const float *raw, uint32_t n, float *out, cudaStream_t st,
                         const uint32_t *n_dev, uint32_t *err);
cudaError_t mlp_grads(const MlpDev &M, const float *raw, const float *target, uint32_t n, cudaStream_t st);
cudaError_t mlp_adam(const MlpDev &M, uint32_t step, float lr, cudaStream_t st);

}  // namespace ilg
