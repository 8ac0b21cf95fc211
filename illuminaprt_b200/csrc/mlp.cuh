// Online-trained radiance cache: a multiresolution hash-grid encoding of
// position (Mueller et al. 2022, "Instant neural graphics primitives")
// feeding a 96 -> 64 x 5 (ReLU) -> 3 MLP in BF16 with FP32 accumulation on
// the tensor cores (mlp.cu). The reference has no learned component; the
// closest analogue is its irradiance cache (Core/Integrator/ICIntegrator.*),
// which this does not reproduce.
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
constexpr int kMlpBands = 4;       // frequency bands of position next to the grid
constexpr int kMlpBandsFreq = 12;  // frequency bands of position in the frequency-only encoding

// Input encodings (MlpDev::encoding)
constexpr uint32_t kEncHashGrid = 0;  // hash grid + 4 bands + spherical harmonics (below)
constexpr uint32_t kEncFreq12 = 1;    // 12 sine/cosine bands of position + raw direction, normal, roughness, albedo

// Hash grid: kGridLevels levels of kGridFeat trainable features, each level a
// table of kGridSize entries. Level l has resolution N_l = floor(16 *
// 2^(7 l / 15)) cells per unit (16 .. 2048; grid_resolution() on the host
// fills MlpDev::grid_res). Levels whose (N_l + 1)^3 corners fit the table are
// indexed densely, the others through the spatial hash
// (x * 1) ^ (y * 2654435761) ^ (z * 805459861) mod kGridSize.
constexpr int kGridLevels = 16;
constexpr int kGridFeat = 2;
constexpr int kGridLog2Size = 15;
constexpr uint32_t kGridSize = 1u << kGridLog2Size;
constexpr uint32_t kGridParams = (uint32_t)kGridLevels * kGridSize * kGridFeat;  // 1,048,576

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
// tensor-core backward copy (layers 1..5): W_l as N = in x K = out, K-major
// core matrices, for dH_{l-1} = dZ_l W_l^T; the output layer's K padded to 16
__host__ __device__ constexpr int umma_bk(int l) { return l == kMlpLayers - 1 ? 16 : mlp_out(l); }
__host__ __device__ constexpr int umma_boff(int l)
{
    return l <= 1 ? 0 : umma_boff(l - 1) + mlp_in(l - 1) * umma_bk(l - 1);
}
constexpr int kUmmaBwdElems = umma_boff(kMlpLayers);

struct MlpDev {
    float *w;                 // FP32 master weights (kMlpParams)
    float *m, *v;             // Adam moments
    float *grad;              // FP32 gradient accumulator
    __nv_bfloat16 *wf;        // forward copy (kFwdElems)
    __nv_bfloat16 *wb;        // backward copy (kBwdElems)
    __nv_bfloat16 *wu;        // tensor-core copy (kUmmaElems)
    __nv_bfloat16 *wv;        // tensor-core backward copy (kUmmaBwdElems)
    float *loss;              // [1] loss sum of the last step
    // training scratch, column-major [feature][row_padded]
    __nv_bfloat16 *xcm;       // kMlpIn x cap
    __nv_bfloat16 *hcm;       // 5 x kMlpHid x cap
    __nv_bfloat16 *dzcm;      // (5 x kMlpHid + kMlpOutP) x cap
    uint32_t cap;             // rows the scratch holds (multiple of 16)
    uint32_t *err;            // device error word (bounded waits)
    // hash grid: FP32 features [level][entry][feature], their gradient and Adam moments
    float *grid, *grid_grad, *grid_m, *grid_v;
    uint32_t grid_res[kGridLevels];
    // inference scratch: the grid columns of each query row, one packed BF16
    // pair per level (enc_cap rows); null = the inference kernel gathers itself
    uint32_t *enc;
    uint32_t enc_cap;
    uint32_t encoding;        // kEncHashGrid or kEncFreq12 (no grid: enc null, grid untouched)
};

// N_l of every level (host).
void grid_resolution(uint32_t (&res)[kGridLevels]);

// Table entry of corner (x, y, z) of level l.
__host__ __device__ __forceinline__ uint32_t grid_index(uint32_t res, uint32_t x, uint32_t y, uint32_t z)
{
    const uint32_t side = res + 1u;
    if ((uint64_t)side * side * side <= kGridSize) return x + side * (y + side * z);
    return (x ^ (y * 2654435761u) ^ (z * 805459861u)) & (kGridSize - 1u);
}

// Cell and trilinear fractions of position coordinate x in [0, 1] at resolution res.
__device__ __forceinline__ void grid_cell(float x, uint32_t res, uint32_t &i, float &f)
{
    x = fminf(fmaxf(x, 0.f), 1.f);
    const float p = __fmul_rn(x, (float)res);
    const uint32_t c = (uint32_t)floorf(p);
    i = c < res ? c : res - 1u;
    f = __fsub_rn(p, (float)i);
}

// The two features of level l at normalised position (x, y, z): the eight
// corners weighted trilinearly, summed in corner order (bit 0 = x, 1 = y,
// 2 = z), every product and sum rounded separately.
__device__ __forceinline__ float2 grid_features(const MlpDev &M, int l, float x, float y, float z)
{
    const uint32_t res = M.grid_res[l];
    uint32_t ix, iy, iz;
    float fx, fy, fz;
    grid_cell(x, res, ix, fx);
    grid_cell(y, res, iy, fy);
    grid_cell(z, res, iz, fz);
    const float2 *table = reinterpret_cast<const float2 *>(M.grid) + (size_t)l * kGridSize;
    float a0 = 0.f, a1 = 0.f;
#pragma unroll
    for (int c = 0; c < 8; c++) {
        const float wx = (c & 1) ? fx : __fsub_rn(1.f, fx);
        const float wy = (c & 2) ? fy : __fsub_rn(1.f, fy);
        const float wz = (c & 4) ? fz : __fsub_rn(1.f, fz);
        const float w = __fmul_rn(__fmul_rn(wx, wy), wz);
        const float2 t = __ldg(table + grid_index(res, ix + (c & 1), iy + ((c >> 1) & 1), iz + (c >> 2)));
        a0 = __fadd_rn(a0, __fmul_rn(w, t.x));
        a1 = __fadd_rn(a1, __fmul_rn(w, t.y));
    }
    return make_float2(a0, a1);
}

// Real spherical harmonics of degree < 4 of the unit vector (x, y, z), two at
// a time (pair k = coefficients 2k, 2k + 1; order l = 0..3, m = -l..l), with
// the usual orthonormal constants sqrt((2l + 1) / 4pi * (l - |m|)! / (l + |m|)!)
// folded in.
__device__ __forceinline__ float2 sh_pair(float x, float y, float z, int k)
{
    const float xx = x * x, yy = y * y, zz = z * z;
    switch (k) {
    case 0: return make_float2(0.28209479177387814f, -0.48860251190291987f * y);
    case 1: return make_float2(0.48860251190291987f * z, -0.48860251190291987f * x);
    case 2: return make_float2(1.0925484305920792f * x * y, -1.0925484305920792f * y * z);
    case 3: return make_float2(0.94617469575755997f * zz - 0.31539156525251999f, -1.0925484305920792f * x * z);
    case 4: return make_float2(0.54627421529603959f * (xx - yy), 0.59004358992664352f * y * (3.f * xx - yy));
    case 5: return make_float2(2.8906114426405538f * x * y * z, 0.45704579946446572f * y * (5.f * zz - 1.f));
    case 6: return make_float2(0.3731763325901154f * z * (5.f * zz - 3.f), 0.45704579946446572f * x * (5.f * zz - 1.f));
    default: return make_float2(1.4453057213202769f * z * (xx - yy), 0.59004358992664352f * x * (xx - 3.f * yy));
    }
}

// Encoded input columns (c, c+1), c even. Columns 0..31: the two hash-grid
// features of level c / 2. Columns 32..55: for axis a and band b < 4, column
// 32 + 8a + 2b is sin(2^b pi x_a) and the next cos(2^b pi x_a). Columns
// 56..71: the 16 spherical harmonics of the outgoing direction. Then 72..74
// normal, 75 roughness, 76..78 albedo, 79 constant 1, 80..95 zero.
// sin and cos of 2^b pi x for the frequency-only encoding: bands 0, 4 and 8
// from sincospif, the three bands after each of them by the double-angle
// identities sin 2a = 2 sin a cos a, cos 2a = (cos a - sin a)(cos a + sin a),
// every product and sum rounded separately (a quarter of the sincospif
// calls; three doublings at most keep the error within a few ulp).
__device__ __forceinline__ void freq_double(float &s, float &c)
{
    const float s2 = __fmul_rn(__fmul_rn(2.f, s), c);
    c = __fmul_rn(__fsub_rn(c, s), __fadd_rn(c, s));
    s = s2;
}
__device__ __forceinline__ void freq_band(float x, int b, float &s, float &c)
{
    sincospif(ldexpf(x, b & ~3), &s, &c);
    for (int k = 0; k < (b & 3); k++) freq_double(s, c);
}

// The frequency-only encoding (kEncFreq12): for axis a and band b < 12,
// column 24a + 2b is sin(2^b pi x_a) and the next cos(2^b pi x_a) (by
// freq_band); then 72..74 outgoing direction, 75..77 normal, 78 roughness,
// 79..81 albedo, 82 constant 1, 83..95 zero.
__device__ __forceinline__ float2 encode_pair_freq(const float *f, int c)
{
    if (c < 6 * kMlpBandsFreq) {
        const int axis = c / (2 * kMlpBandsFreq), band = (c % (2 * kMlpBandsFreq)) >> 1;
        float s, co;
        freq_band(f[axis], band, s, co);
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

__device__ __forceinline__ float2 encode_pair(const float *f, int c, const MlpDev &M)
{
    if (M.encoding == kEncFreq12) return encode_pair_freq(f, c);
    if (c < 2 * kGridLevels) return grid_features(M, c >> 1, f[0], f[1], f[2]);
    if (c < 56) {
        const int k = c - 32, axis = k >> 3, band = (k & 7) >> 1;
        const float x = axis == 0 ? f[0] : (axis == 1 ? f[1] : f[2]);
        float s, co;
        sincospif(ldexpf(x, band), &s, &co);
        return make_float2(s, co);
    }
    if (c < 72) return sh_pair(f[3], f[4], f[5], (c - 56) >> 1);
    switch (c) {
    case 72: return make_float2(f[6], f[7]);
    case 74: return make_float2(f[8], f[9]);
    case 76: return make_float2(f[10], f[11]);
    case 78: return make_float2(f[12], 1.f);
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
// warp_mma: the warp-level mma.sync kernels; otherwise the tcgen05 ones
// (mlp_train_tc.cu).
cudaError_t mlp_grads(const MlpDev &M, const float *raw, const float *target, uint32_t n, cudaStream_t st,
                      bool warp_mma = false);
// Forward with activations kept, loss and backward (tcgen05): X, H_0..H_4 and
// dZ_0..dZ_5 into M.xcm / hcm / dzcm, the loss into M.loss.
cudaError_t mlp_train_tc(const MlpDev &M, const float *raw, const float *target, uint32_t n, cudaStream_t st);
// dW_l += H_{l-1}^T dZ_l for every layer from the column-major activations (tcgen05).
cudaError_t mlp_dw_tc(const MlpDev &M, uint32_t n_pad, cudaStream_t st);
cudaError_t mlp_adam(const MlpDev &M, uint32_t step, float lr, cudaStream_t st);

}  // namespace ilg
