// BF16 tensor-core MLP of the radiance cache (see mlp.cuh).
//
// The network is small (23,040 weights), so every warp keeps a 16-row tile's
// activations in registers through all six layers: the FP32 accumulator
// fragments of one m16n8k16 MMA pair up into the BF16 A fragments of the next
// layer without leaving the register file, and the weights stay in shared
// memory for the whole kernel. Training runs three kernels:
//   k_mlp_fwd<true>  forward, storing the encoded input and every hidden
//                    activation column-major for the weight gradients
//   k_mlp_bwd        recomputes the forward, evaluates the relative-L2 loss
//                    (mean over rows and RGB of (y - t)^2 / (y^2 + 0.01), y
//                    held constant in the denominator), back-propagates dZ
//                    through the layers on the tensor cores, stores dZ
//   k_mlp_dw         dW_l = H_{l-1}^T dZ_l as a split-K tensor-core GEMM over
//                    the batch, FP32 partial sums added atomically
//   k_grid_bwd       dX of the grid columns = dZ0 W0^T, scattered to the
//                    hash-grid corners of every level (FP32 atomics)
// followed by k_mlp_adam (FP32 master weights, refreshes the BF16 copies)
// and k_grid_adam (the grid features).
#include "devinfo.cuh"
#include "mlp.cuh"

#include <cmath>
#include <cstdio>

namespace ilg {

namespace {

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}
__device__ __forceinline__ float2 unpack_bf16(uint32_t u)
{
    __nv_bfloat162 v = *reinterpret_cast<__nv_bfloat162 *>(&u);
    return __bfloat1622float2(v);
}

// D = A (16x16 bf16, row) * B (16x8 bf16, col) + D, FP32 accumulate
__device__ __forceinline__ void mma16816(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t ld_u32(const __nv_bfloat16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

// C[8 tiles of n8] += A[KB k16 blocks] x W^T, W given as [n][k] rows with `stride`
template <int KB>
__device__ __forceinline__ void layer64(const uint32_t (&a)[KB][4], const __nv_bfloat16 *w, int stride, int g, int tig,
                                        float (&c)[8][4])
{
#pragma unroll
    for (int j = 0; j < 8; j++) c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.f;
#pragma unroll
    for (int kk = 0; kk < KB; kk++) {
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const __nv_bfloat16 *row = w + (8 * j + g) * stride + 16 * kk + 2 * tig;
            mma16816(c[j], a[kk], ld_u32(row), ld_u32(row + 8));
        }
    }
}

// relu + repack the 8 C tiles (16 x 64) into 4 A blocks
__device__ __forceinline__ void relu_pack(const float (&c)[8][4], uint32_t (&a)[4][4])
{
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
        const float(&lo)[4] = c[2 * kk];
        const float(&hi)[4] = c[2 * kk + 1];
        a[kk][0] = pack_bf16(fmaxf(lo[0], 0.f), fmaxf(lo[1], 0.f));
        a[kk][1] = pack_bf16(fmaxf(lo[2], 0.f), fmaxf(lo[3], 0.f));
        a[kk][2] = pack_bf16(fmaxf(hi[0], 0.f), fmaxf(hi[1], 0.f));
        a[kk][3] = pack_bf16(fmaxf(hi[2], 0.f), fmaxf(hi[3], 0.f));
    }
}

// column-major store of one packed A block (16 rows x 16 columns) at column base c0
__device__ __forceinline__ void store_cm(__nv_bfloat16 *dst, uint32_t cap, int c0, uint32_t r0, int g, int tig,
                                         const uint32_t (&a)[4])
{
    const int c = c0 + 2 * tig;
    const float2 v0 = unpack_bf16(a[0]), v1 = unpack_bf16(a[1]), v2 = unpack_bf16(a[2]), v3 = unpack_bf16(a[3]);
    dst[(size_t)c * cap + r0 + g] = __float2bfloat16_rn(v0.x);
    dst[(size_t)(c + 1) * cap + r0 + g] = __float2bfloat16_rn(v0.y);
    dst[(size_t)c * cap + r0 + g + 8] = __float2bfloat16_rn(v1.x);
    dst[(size_t)(c + 1) * cap + r0 + g + 8] = __float2bfloat16_rn(v1.y);
    dst[(size_t)(c + 8) * cap + r0 + g] = __float2bfloat16_rn(v2.x);
    dst[(size_t)(c + 9) * cap + r0 + g] = __float2bfloat16_rn(v2.y);
    dst[(size_t)(c + 8) * cap + r0 + g + 8] = __float2bfloat16_rn(v3.x);
    dst[(size_t)(c + 9) * cap + r0 + g + 8] = __float2bfloat16_rn(v3.y);
}

__device__ __forceinline__ void load_smem(__nv_bfloat16 *dst, const __nv_bfloat16 *src, int n_elems)
{
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
    uint4 *d = reinterpret_cast<uint4 *>(dst);
    for (int i = threadIdx.x; i < n_elems / 8; i += blockDim.x) d[i] = s[i];
}

// input A fragments (6 k16 blocks) of rows r0+g, r0+g+8 from raw features
__device__ __forceinline__ void encode_rows(const MlpDev &M, const float *raw, uint32_t n, uint32_t r0, int g, int tig,
                                           uint32_t (&a)[6][4])
{
    float f0[kMlpRaw], f1[kMlpRaw];
    const uint32_t ra = r0 + g, rb = r0 + g + 8;
#pragma unroll
    for (int k = 0; k < kMlpRaw; k++) {
        f0[k] = ra < n ? raw[(size_t)ra * kMlpRaw + k] : 0.f;
        f1[k] = rb < n ? raw[(size_t)rb * kMlpRaw + k] : 0.f;
    }
#pragma unroll
    for (int kk = 0; kk < 6; kk++) {
        const int c = 16 * kk + 2 * tig;
        float2 p;
        p = encode_pair(f0, c, M);
        a[kk][0] = ra < n ? pack_bf16(p.x, p.y) : 0u;
        p = encode_pair(f1, c, M);
        a[kk][1] = rb < n ? pack_bf16(p.x, p.y) : 0u;
        p = encode_pair(f0, c + 8, M);
        a[kk][2] = ra < n ? pack_bf16(p.x, p.y) : 0u;
        p = encode_pair(f1, c + 8, M);
        a[kk][3] = rb < n ? pack_bf16(p.x, p.y) : 0u;
    }
}

template <bool kTrain>
__global__ void __launch_bounds__(128) k_mlp_fwd(MlpDev M, const float *__restrict__ raw, uint32_t n,
                                                 float *__restrict__ out, const uint32_t *__restrict__ n_dev)
{
    extern __shared__ __align__(16) __nv_bfloat16 sw[];
    if (n_dev) n = min(n, *n_dev);  // row count produced on the device (capped by the launch size)
    load_smem(sw, M.wf, kFwdElems);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
    const uint32_t n_tiles = (n + 15) / 16;
    for (uint32_t tile = blockIdx.x * 4 + warp; tile < n_tiles; tile += gridDim.x * 4) {
        const uint32_t r0 = tile * 16;
        uint32_t a0[6][4];
        encode_rows(M, raw, n, r0, g, tig, a0);
        if (kTrain) {
#pragma unroll
            for (int kk = 0; kk < 6; kk++) store_cm(M.xcm, M.cap, 16 * kk, r0, g, tig, a0[kk]);
        }
        float c[8][4];
        uint32_t a[4][4];
        layer64<6>(a0, sw + fwd_off(0), fwd_stride(0), g, tig, c);
        relu_pack(c, a);
        if (kTrain) {
#pragma unroll
            for (int kk = 0; kk < 4; kk++) store_cm(M.hcm, M.cap, 16 * kk, r0, g, tig, a[kk]);
        }
#pragma unroll
        for (int l = 1; l < 5; l++) {
            layer64<4>(a, sw + fwd_off(l), fwd_stride(l), g, tig, c);
            relu_pack(c, a);
            if (kTrain) {
#pragma unroll
                for (int kk = 0; kk < 4; kk++)
                    store_cm(M.hcm + (size_t)l * kMlpHid * M.cap, M.cap, 16 * kk, r0, g, tig, a[kk]);
            }
        }
        if (!kTrain) {
            float y[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                const __nv_bfloat16 *row = sw + fwd_off(5) + g * fwd_stride(5) + 16 * kk + 2 * tig;
                mma16816(y, a[kk], ld_u32(row), ld_u32(row + 8));
            }
            const int col = 2 * tig;
            const uint32_t ra = r0 + g, rb = r0 + g + 8;
            if (col < 3) {
                if (ra < n) out[(size_t)ra * 3 + col] = y[0];
                if (rb < n) out[(size_t)rb * 3 + col] = y[2];
            }
            if (col + 1 < 3) {
                if (ra < n) out[(size_t)ra * 3 + col + 1] = y[1];
                if (rb < n) out[(size_t)rb * 3 + col + 1] = y[3];
            }
        }
    }
}

// bit mask of the (row, col) entries of C tile j whose forward activation was > 0
__device__ __forceinline__ void relu_mask(const uint32_t (&h)[4][4], int j, float (&d)[4])
{
    const float2 top = unpack_bf16(h[j >> 1][(j & 1) * 2]);
    const float2 bot = unpack_bf16(h[j >> 1][(j & 1) * 2 + 1]);
    if (!(top.x > 0.f)) d[0] = 0.f;
    if (!(top.y > 0.f)) d[1] = 0.f;
    if (!(bot.x > 0.f)) d[2] = 0.f;
    if (!(bot.y > 0.f)) d[3] = 0.f;
}

__global__ void __launch_bounds__(128) k_mlp_bwd(MlpDev M, const float *__restrict__ raw,
                                                 const float *__restrict__ target, uint32_t n)
{
    extern __shared__ __align__(16) __nv_bfloat16 sw[];
    __nv_bfloat16 *swf = sw, *swb = sw + kFwdElems;
    load_smem(swf, M.wf, kFwdElems);
    load_smem(swb, M.wb, kBwdElems);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
    const uint32_t n_tiles = (n + 15) / 16;
    const float inv_count = 1.f / (3.f * (float)n);
    float loss = 0.f;
    for (uint32_t tile = blockIdx.x * 4 + warp; tile < n_tiles; tile += gridDim.x * 4) {
        const uint32_t r0 = tile * 16, ra = r0 + g, rb = r0 + g + 8;
        // forward, keeping every hidden activation in registers
        uint32_t h[5][4][4];
        {
            uint32_t a0[6][4];
            encode_rows(M, raw, n, r0, g, tig, a0);
            float c[8][4];
            layer64<6>(a0, swf + fwd_off(0), fwd_stride(0), g, tig, c);
            relu_pack(c, h[0]);
#pragma unroll
            for (int l = 1; l < 5; l++) {
                layer64<4>(h[l - 1], swf + fwd_off(l), fwd_stride(l), g, tig, c);
                relu_pack(c, h[l]);
            }
        }
        float y[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
            const __nv_bfloat16 *row = swf + fwd_off(5) + g * fwd_stride(5) + 16 * kk + 2 * tig;
            mma16816(y, h[4][kk], ld_u32(row), ld_u32(row + 8));
        }
        // dL/dy of the relative L2 loss
        float dy[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int col = 2 * tig + (e & 1);
            const uint32_t r = (e < 2) ? ra : rb;
            dy[e] = 0.f;
            if (col < 3 && r < n) {
                const float t = target[(size_t)r * 3 + col];
                const float den = y[e] * y[e] + 0.01f;
                const float diff = y[e] - t;
                loss += diff * diff / den;
                dy[e] = 2.f * diff / den * inv_count;
            }
        }
        uint32_t d[4][4];
        d[0][0] = pack_bf16(dy[0], dy[1]);
        d[0][1] = pack_bf16(dy[2], dy[3]);
        d[0][2] = 0u;
        d[0][3] = 0u;
        {
            // dZ5 (8 columns) column-major
            __nv_bfloat16 *dz5 = M.dzcm + (size_t)5 * kMlpHid * M.cap;
            const int col = 2 * tig;
            dz5[(size_t)col * M.cap + ra] = __float2bfloat16_rn(dy[0]);
            dz5[(size_t)(col + 1) * M.cap + ra] = __float2bfloat16_rn(dy[1]);
            dz5[(size_t)col * M.cap + rb] = __float2bfloat16_rn(dy[2]);
            dz5[(size_t)(col + 1) * M.cap + rb] = __float2bfloat16_rn(dy[3]);
        }
        // back through layers 5..1: dZ_{l-1} = (dZ_l W_l^T) * relu'(H_{l-1})
#pragma unroll
        for (int l = 5; l >= 1; l--) {
            float c[8][4];
#pragma unroll
            for (int j = 0; j < 8; j++) c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.f;
            const int kb = bwd_outp(l) / 16;
            const __nv_bfloat16 *wl = swb + bwd_off(l);
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                if (kk >= kb) break;
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const __nv_bfloat16 *row = wl + (8 * j + g) * bwd_stride(l) + 16 * kk + 2 * tig;
                    mma16816(c[j], d[kk], ld_u32(row), ld_u32(row + 8));
                }
            }
#pragma unroll
            for (int j = 0; j < 8; j++) relu_mask(h[l - 1], j, c[j]);
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                d[kk][0] = pack_bf16(c[2 * kk][0], c[2 * kk][1]);
                d[kk][1] = pack_bf16(c[2 * kk][2], c[2 * kk][3]);
                d[kk][2] = pack_bf16(c[2 * kk + 1][0], c[2 * kk + 1][1]);
                d[kk][3] = pack_bf16(c[2 * kk + 1][2], c[2 * kk + 1][3]);
                store_cm(M.dzcm + (size_t)(l - 1) * kMlpHid * M.cap, M.cap, 16 * kk, r0, g, tig, d[kk]);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if (lane == 0) atomicAdd(M.loss, loss / (3.f * (float)n));
}

// dW_l[in][out] += sum over rows of A[in][row] * B[out][row] (both column-major
// activations); each warp owns 16 input rows, the CTA one chunk of the batch.
constexpr uint32_t kDwChunk = 256;

template <int kOut>
__global__ void k_mlp_dw(const __nv_bfloat16 *__restrict__ A, const __nv_bfloat16 *__restrict__ B, uint32_t cap,
                         uint32_t n_pad, float *__restrict__ grad)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
    constexpr int NT = kOut / 8;
    float c[NT][4];
#pragma unroll
    for (int j = 0; j < NT; j++) c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.f;
    const uint32_t k_begin = blockIdx.x * kDwChunk;
    const uint32_t k_end = min(n_pad, k_begin + kDwChunk);
    const __nv_bfloat16 *arow0 = A + (size_t)(warp * 16 + g) * cap, *arow1 = A + (size_t)(warp * 16 + g + 8) * cap;
    for (uint32_t k0 = k_begin; k0 < k_end; k0 += 16) {
        uint32_t a[4];
        a[0] = ld_u32(arow0 + k0 + 2 * tig);
        a[1] = ld_u32(arow1 + k0 + 2 * tig);
        a[2] = ld_u32(arow0 + k0 + 2 * tig + 8);
        a[3] = ld_u32(arow1 + k0 + 2 * tig + 8);
#pragma unroll
        for (int j = 0; j < NT; j++) {
            const __nv_bfloat16 *brow = B + (size_t)(8 * j + g) * cap + k0 + 2 * tig;
            mma16816(c[j], a, ld_u32(brow), ld_u32(brow + 8));
        }
    }
#pragma unroll
    for (int j = 0; j < NT; j++) {
        const int col = 8 * j + 2 * tig;
        const int r = warp * 16 + g;
        atomicAdd(&grad[(size_t)r * kOut + col], c[j][0]);
        atomicAdd(&grad[(size_t)r * kOut + col + 1], c[j][1]);
        atomicAdd(&grad[(size_t)(r + 8) * kOut + col], c[j][2]);
        atomicAdd(&grad[(size_t)(r + 8) * kOut + col + 1], c[j][3]);
    }
}

__device__ __forceinline__ int layer_of(int i)
{
    int l = 0;
#pragma unroll
    for (int k = 1; k < kMlpLayers; k++)
        if (i >= mlp_off(k)) l = k;
    return l;
}

__device__ __forceinline__ void write_copies(const MlpDev &M, int i, float w)
{
    const int l = layer_of(i);
    const int local = i - mlp_off(l);
    const int in = local / mlp_out(l), o = local % mlp_out(l);
    const __nv_bfloat16 b = __float2bfloat16_rn(w);
    M.wf[fwd_off(l) + o * fwd_stride(l) + in] = b;
    if (l >= 1) M.wb[bwd_off(l) + in * bwd_stride(l) + o] = b;
    if (M.wu) {
        // element (n = o, k = in) of the K-major core-matrix layout
        const int kc = mlp_in(l) / 8;
        M.wu[umma_off(l) + (o / 8) * kc * 64 + (in / 8) * 64 + (o % 8) * 8 + (in % 8)] = b;
    }
    if (M.wv && l >= 1) {
        // element (n = in, k = o) of the backward copy
        const int kc = umma_bk(l) / 8;
        M.wv[umma_boff(l) + (in / 8) * kc * 64 + (o / 8) * 64 + (in % 8) * 8 + (o % 8)] = b;
    }
}

__device__ __forceinline__ float hash_uniform(uint32_t seed, uint32_t i)
{
    uint32_t x = i * 0x9E3779B9u ^ (seed * 0x85EBCA6Bu + 0x7F4A7C15u);
    x ^= x >> 16; x *= 0x7FEB352Du; x ^= x >> 15; x *= 0x846CA68Bu; x ^= x >> 16;
    return (x >> 8) * 0x1p-24f;
}

__global__ void k_mlp_init(MlpDev M, uint32_t seed)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpParams) return;
    const int l = layer_of(i);
    const int local = i - mlp_off(l);
    const int o = local % mlp_out(l);
    const float bound = sqrtf(6.f / (float)(mlp_in(l) + (l == kMlpLayers - 1 ? 3 : mlp_out(l))));
    float w = (2.f * hash_uniform(seed, (uint32_t)i) - 1.f) * bound;
    if (l == kMlpLayers - 1 && o >= 3) w = 0.f;  // unused output columns stay zero
    M.w[i] = w;
    M.m[i] = 0.f;
    M.v[i] = 0.f;
    write_copies(M, i, w);
}

__global__ void k_mlp_copies(MlpDev M)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpParams) return;
    write_copies(M, i, M.w[i]);
}

__global__ void k_mlp_adam(MlpDev M, float lr, float bc1, float bc2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpParams) return;
    const int l = layer_of(i);
    if (l == kMlpLayers - 1 && ((i - mlp_off(l)) % mlp_out(l)) >= 3) return;
    const float b1 = 0.9f, b2 = 0.99f, eps = 1e-15f;
    const float gr = M.grad[i];
    const float m = b1 * M.m[i] + (1.f - b1) * gr;
    const float v = b2 * M.v[i] + (1.f - b2) * gr * gr;
    M.m[i] = m;
    M.v[i] = v;
    const float w = M.w[i] - lr * (m / bc1) / (sqrtf(v / bc2) + eps);
    M.w[i] = w;
    write_copies(M, i, w);
}

__global__ void k_grid_init(MlpDev M, uint32_t seed)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kGridParams) return;
    M.grid[i] = (2.f * hash_uniform(seed ^ 0xA5A5A5A5u, i) - 1.f) * 1e-4f;
    M.grid_m[i] = 0.f;
    M.grid_v[i] = 0.f;
}

// Gradient of the loss with respect to the grid features: per row, dX of the
// 32 grid columns = dZ0 W0^T (W0 as the forward used it, in BF16), then
// scattered to the eight corners of every level with the trilinear weights.
constexpr int kGridBwdThreads = 256;

// One thread per (row, level), as k_grid_encode: the sixteen levels of a row
// run in parallel (a batch of 16,384 rows is 262,144 threads, where one
// thread per row left the SMs a few warps each). The row's dZ0 loads are
// shared by the 16 lanes of a half-warp (one address per load); W0's rows are
// padded to 65 floats so that the 16 levels of a half-warp read 16 banks.
__global__ void __launch_bounds__(kGridBwdThreads) k_grid_bwd(MlpDev M, const float *__restrict__ raw, uint32_t n)
{
    __shared__ float w0[2 * kGridLevels][kMlpHid + 1];
    for (int i = threadIdx.x; i < 2 * kGridLevels * kMlpHid; i += blockDim.x)
        w0[i / kMlpHid][i % kMlpHid] = __bfloat162float(__float2bfloat16_rn(M.w[mlp_off(0) + i]));
    __syncthreads();
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = (uint32_t)(i / kGridLevels), l = (uint32_t)(i % kGridLevels);
    if (r >= n) return;
    float d0 = 0.f, d1 = 0.f;
#pragma unroll 16
    for (int j = 0; j < kMlpHid; j++) {
        const float dz = __bfloat162float(M.dzcm[(size_t)j * M.cap + r]);
        d0 = fmaf(dz, w0[2 * l][j], d0);
        d1 = fmaf(dz, w0[2 * l + 1][j], d1);
    }
    if (d0 == 0.f && d1 == 0.f) return;
    const float x = raw[(size_t)r * kMlpRaw], y = raw[(size_t)r * kMlpRaw + 1], z = raw[(size_t)r * kMlpRaw + 2];
    const uint32_t res = M.grid_res[l];
    uint32_t ix, iy, iz;
    float fx, fy, fz;
    grid_cell(x, res, ix, fx);
    grid_cell(y, res, iy, fy);
    grid_cell(z, res, iz, fz);
    float2 *gg = reinterpret_cast<float2 *>(M.grid_grad) + (size_t)l * kGridSize;
#pragma unroll
    for (int c = 0; c < 8; c++) {
        const float wx = (c & 1) ? fx : __fsub_rn(1.f, fx);
        const float wy = (c & 2) ? fy : __fsub_rn(1.f, fy);
        const float wz = (c & 4) ? fz : __fsub_rn(1.f, fz);
        const float w = __fmul_rn(__fmul_rn(wx, wy), wz);
        // both features of the corner in one vector atomic (sm_90 and later)
        atomicAdd(gg + grid_index(res, ix + (c & 1), iy + ((c >> 1) & 1), iz + (c >> 2)), make_float2(w * d0, w * d1));
    }
}

inline unsigned grid_bwd_blocks(uint32_t n)
{
    return (unsigned)(((uint64_t)n * kGridLevels + kGridBwdThreads - 1) / kGridBwdThreads);
}

__global__ void k_grid_adam(MlpDev M, float lr, float bc1, float bc2)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kGridParams) return;
    const float b1 = 0.9f, b2 = 0.99f, eps = 1e-15f;
    const float gr = M.grid_grad[i];
    const float m = b1 * M.grid_m[i] + (1.f - b1) * gr;
    const float v = b2 * M.grid_v[i] + (1.f - b2) * gr * gr;
    M.grid_m[i] = m;
    M.grid_v[i] = v;
    M.grid[i] -= lr * (m / bc1) / (sqrtf(v / bc2) + eps);
}

inline uint32_t grid_for(uint32_t n_rows, int sms)
{
    const uint32_t tiles = (n_rows + 15) / 16;
    uint32_t blocks = (tiles + 3) / 4;
    const uint32_t cap = (uint32_t)sms * 8;
    return blocks < 1 ? 1 : (blocks > cap ? cap : blocks);
}

int num_sms() { return current_sm_count(); }

}  // namespace

void grid_resolution(uint32_t (&res)[kGridLevels])
{
    for (int l = 0; l < kGridLevels; l++) res[l] = (uint32_t)std::floor(16.0 * std::pow(2.0, 7.0 * l / 15.0));
}

cudaError_t mlp_init(const MlpDev &M, uint32_t seed, cudaStream_t st)
{
    k_grid_init<<<(kGridParams + 255) / 256, 256, 0, st>>>(M, seed);
    cudaError_t e;
    if ((e = cudaMemsetAsync(M.wf, 0, kFwdElems * sizeof(__nv_bfloat16), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(M.wb, 0, kBwdElems * sizeof(__nv_bfloat16), st)) != cudaSuccess) return e;
    if (M.wu && (e = cudaMemsetAsync(M.wu, 0, kUmmaElems * sizeof(__nv_bfloat16), st)) != cudaSuccess) return e;
    if (M.wv && (e = cudaMemsetAsync(M.wv, 0, kUmmaBwdElems * sizeof(__nv_bfloat16), st)) != cudaSuccess) return e;
    k_mlp_init<<<(kMlpParams + 255) / 256, 256, 0, st>>>(M, seed);
    return cudaGetLastError();
}

cudaError_t mlp_refresh_copies(const MlpDev &M, cudaStream_t st)
{
    k_mlp_copies<<<(kMlpParams + 255) / 256, 256, 0, st>>>(M);
    return cudaGetLastError();
}

cudaError_t mlp_infer(const MlpDev &M, const float *raw, uint32_t n, float *out, cudaStream_t st,
                      const uint32_t *n_dev)
{
    return mlp_infer_tc(M, raw, n, out, st, n_dev, M.err);
}

cudaError_t mlp_infer_warp(const MlpDev &M, const float *raw, uint32_t n, float *out, cudaStream_t st,
                           const uint32_t *n_dev)
{
    if (n == 0) return cudaSuccess;
    const size_t smem = kFwdElems * sizeof(__nv_bfloat16);
    cudaError_t e = ensure_dynamic_smem((const void *)k_mlp_fwd<false>, (int)smem);
    if (e != cudaSuccess) return e;
    k_mlp_fwd<false><<<grid_for(n, num_sms()), 128, smem, st>>>(M, raw, n, out, n_dev);
    return cudaGetLastError();
}

cudaError_t mlp_grads(const MlpDev &M, const float *raw, const float *target, uint32_t n, cudaStream_t st,
                      bool warp_mma)
{
    if (n == 0 || n > M.cap) return cudaErrorInvalidValue;
    cudaError_t e;
    const uint32_t n_pad = (n + 15) / 16 * 16;
    if (!warp_mma && M.wv) {
        if ((e = cudaMemsetAsync(M.grad, 0, kMlpParams * sizeof(float), st)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(M.loss, 0, sizeof(float), st)) != cudaSuccess) return e;
        const bool has_grid = M.encoding == kEncHashGrid;
        if (has_grid && (e = cudaMemsetAsync(M.grid_grad, 0, kGridParams * sizeof(float), st)) != cudaSuccess)
            return e;
        if ((e = mlp_train_tc(M, raw, target, n, st)) != cudaSuccess) return e;
        if (has_grid)
            k_grid_bwd<<<grid_bwd_blocks(n), kGridBwdThreads, 0, st>>>(M, raw, n);
        if ((e = mlp_dw_tc(M, n_pad, st)) != cudaSuccess) return e;
        return cudaGetLastError();
    }
    // rows n..n_pad of the column-major scratch must be zero; the kernels
    // write exact zeros for them, but clear once so stale rows never leak
    if ((e = cudaMemsetAsync(M.grad, 0, kMlpParams * sizeof(float), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(M.loss, 0, sizeof(float), st)) != cudaSuccess) return e;
    const bool has_grid = M.encoding == kEncHashGrid;
    if (has_grid && (e = cudaMemsetAsync(M.grid_grad, 0, kGridParams * sizeof(float), st)) != cudaSuccess) return e;
    const size_t smem_f = kFwdElems * sizeof(__nv_bfloat16);
    const size_t smem_b = (kFwdElems + kBwdElems) * sizeof(__nv_bfloat16);
    if ((e = ensure_dynamic_smem((const void *)k_mlp_fwd<true>, (int)smem_f)) != cudaSuccess) return e;
    if ((e = ensure_dynamic_smem((const void *)k_mlp_bwd, (int)smem_b)) != cudaSuccess) return e;
    const uint32_t grid = grid_for(n, num_sms());
    k_mlp_fwd<true><<<grid, 128, smem_f, st>>>(M, raw, n, nullptr, nullptr);
    k_mlp_bwd<<<grid, 128, smem_b, st>>>(M, raw, target, n);
    if (has_grid) k_grid_bwd<<<grid_bwd_blocks(n), kGridBwdThreads, 0, st>>>(M, raw, n);
    const uint32_t chunks = (n_pad + kDwChunk - 1) / kDwChunk;
    for (int l = 0; l < kMlpLayers; l++) {
        const __nv_bfloat16 *A = l == 0 ? M.xcm : M.hcm + (size_t)(l - 1) * kMlpHid * M.cap;
        const __nv_bfloat16 *B = M.dzcm + (size_t)l * kMlpHid * M.cap;
        float *gl = M.grad + mlp_off(l);
        const int warps = mlp_in(l) / 16;
        if (l == kMlpLayers - 1)
            k_mlp_dw<kMlpOutP><<<chunks, 32 * warps, 0, st>>>(A, B, M.cap, n_pad, gl);
        else
            k_mlp_dw<kMlpHid><<<chunks, 32 * warps, 0, st>>>(A, B, M.cap, n_pad, gl);
    }
    return cudaGetLastError();
}

cudaError_t mlp_adam(const MlpDev &M, uint32_t step, float lr, cudaStream_t st)
{
    const float bc1 = 1.f - powf(0.9f, (float)step), bc2 = 1.f - powf(0.99f, (float)step);
    k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(M, lr, bc1, bc2);
    if (M.encoding == kEncHashGrid) k_grid_adam<<<(kGridParams + 255) / 256, 256, 0, st>>>(M, lr, bc1, bc2);
    return cudaGetLastError();
}

}  // namespace ilg
