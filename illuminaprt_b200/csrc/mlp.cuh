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

struct MlpDev {
    float *w;                 // FP32 master weights (kMlpParams)
    float *m, *v;             // Adam moments
    float *grad;              // FP32 gradient accumulator
    __nv_bfloat16 *wf;        // forward copy (kFwdElems)
    __nv_bfloat16 *wb;        // backward copy (kBwdElems)
    float *loss;              // [1] loss sum of the last step
    // training scratch, column-major [feature][row_padded]
    __nv_bfloat16 *xcm;       // kMlpIn x cap
    __nv_bfloat16 *hcm;       // 5 x kMlpHid x cap
    __nv_bfloat16 *dzcm;      // (5 x kMlpHid + kMlpOutP) x cap
    uint32_t cap;             // rows the scratch holds (multiple of 16)
};

// Host entry points (mlp.cu). All enqueue on `st`.
cudaError_t mlp_init(const MlpDev &M, uint32_t seed, cudaStream_t st);
cudaError_t mlp_refresh_copies(const MlpDev &M, cudaStream_t st);
// n_dev (optional): a device word holding the actual row count (<= n).
cudaError_t mlp_infer(const MlpDev &M, const float *raw, uint32_t n, float *out, cudaStream_t st,
                      const uint32_t *n_dev = nullptr);
// Forward + loss + backward + weight gradients into M.grad (zeroed first).
cudaError_t mlp_grads(const MlpDev &M, const float *raw, const float *target, uint32_t n, cudaStream_t st);
cudaError_t mlp_adam(const MlpDev &M, uint32_t step, float lr, cudaStream_t st);

}  // namespace ilg
