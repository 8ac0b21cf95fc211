// Radiance-cache training on the 5th-generation tensor cores.
//
// k_mlp_train_tc: one CTA of 128 threads per SM takes 128-row tiles of the
// batch (one row per thread, the TMEM lane of the row's accumulator) through
//   * the forward pass: the encoded input X and the hidden activations
//     H_0..H_4 (ReLU, rounded to BF16) stay in shared memory as K-major
//     A tiles, every layer one tcgen05.mma group (M = 128, K = 96 or 64,
//     N = 64 or 16) against the forward weight copy, accumulated in TMEM;
//   * the loss: the relative L2 loss of the three outputs (y held constant
//     in the denominator) and dL/dy, rounded to BF16 as dZ_5;
//   * the backward pass: dH_{l-1} = dZ_l W_l^T as one MMA group per layer
//     against the backward weight copy (W_l as N = in x K = out), masked by
//     H_{l-1} > 0 and rounded to BF16 as dZ_{l-1}, written over the A tile
//     it came from;
// storing X, H_l and dZ_l column-major (rows contiguous per feature) for the
// weight gradients.
//
// k_mlp_dw_tc: dW_l = H_{l-1}^T dZ_l for every layer l, split over the
// batch: a CTA owns 512 rows of one layer and accumulates, 64 rows at a
// time, M = 128 features (the layer's 96 or 64, the rest zero) x N = 64 (16
// for the output layer) in TMEM, both operands loaded from the column-major
// activations, which are K-major for this product; the partial sums are
// added atomically to the FP32 gradient.
//
// The arithmetic is the warp-level kernels' (mlp.cu): BF16 operands at the
// same points, FP32 accumulation. Every mbarrier wait is bounded and raises
// an error bit instead of hanging; TMEM is allocated once per CTA and freed
// on exit.
#include "devinfo.cuh"
#include "mlp.cuh"
#include "umma.cuh"

namespace ilg {

namespace {

using namespace umma;

constexpr int kTrRows = 128;
constexpr uint32_t kTrTmemCols = 64;
constexpr size_t kTrWf = ((kUmmaElems * 2 + 1023) / 1024) * 1024;     // forward weights
constexpr size_t kTrWb = ((kUmmaBwdElems * 2 + 1023) / 1024) * 1024;  // backward weights
constexpr size_t kTrX = (size_t)kTrRows * kMlpIn * 2;                 // X tile, then the dZ tiles
constexpr size_t kTrH = (size_t)kTrRows * kMlpHid * 2;                // one hidden tile
constexpr size_t kTrSmem = kTrWf + kTrWb + kTrX + 5 * kTrH;
static_assert(kTrSmem <= 227 * 1024, "shared memory of the training kernel");
static_assert(kTrX % 1024 == 0 && kTrH % 1024 == 0, "tile alignment");

// One layer's MMAs, D (TMEM, 128 x N) = A (128 x K) B^T (B: N x K), both
// K-major tiles of 8-row x 16-byte core matrices; issued by one thread and
// committed to `bar`.
__device__ __forceinline__ void issue_layer(uint32_t tmem, uint32_t a_addr, uint32_t b_addr, int K, int N, uint32_t bar)
{
    const uint32_t idesc = umma_idesc(kTrRows, N);
    for (int s = 0; s < K / 16; s++) {
        const uint64_t da = umma_desc(a_addr + s * 256, 128, (K / 8) * 128);
        const uint64_t db = umma_desc(b_addr + s * 256, 128, (K / 8) * 128);
        mma_bf16(tmem, da, db, idesc, s > 0 ? 1u : 0u);
    }
    mma_commit(bar);
}

// Every thread's smem writes visible to the tensor core, then the issue.
__device__ __forceinline__ void cta_sync_for_mma()
{
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
}

__global__ void __launch_bounds__(kTrRows, 1) k_mlp_train_tc(const MlpDev M, const float *__restrict__ raw,
                                                             const float *__restrict__ target, uint32_t n,
                                                             uint32_t n_pad)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *wf_s = smem, *wb_s = smem + kTrWf, *xz_s = wb_s + kTrWb, *h_s = xz_s + kTrX;
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base_s;

    const int tid = threadIdx.x, warp = tid >> 5;
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(M.wu);
        uint4 *dst = reinterpret_cast<uint4 *>(wf_s);
        for (int i = tid; i < kUmmaElems / 8; i += kTrRows) dst[i] = src[i];
        src = reinterpret_cast<const uint4 *>(M.wv);
        dst = reinterpret_cast<uint4 *>(wb_s);
        for (int i = tid; i < kUmmaBwdElems / 8; i += kTrRows) dst[i] = src[i];
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                     "r"(kTrTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    cta_sync_for_mma();
    const uint32_t tmem = tmem_base_s;
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t bar_a = smem_u32(&bar);
    const uint32_t wf_a = smem_u32(wf_s), wb_a = smem_u32(wb_s), xz_a = smem_u32(xz_s), h_a = smem_u32(h_s);
    const size_t cap = M.cap;
    const float inv_count = 1.f / (3.f * (float)n);
    uint32_t phase = 0;
    bool ok = true;
    float loss = 0.f;

    // waits for the layer's MMAs; false (and the error bit) if the wait ran out
    auto wait_layer = [&]() {
        const bool waited = mbar_wait(bar_a, phase);
        if (!waited) atomicOr(M.err, kErrWait);
        ok = __syncthreads_and(waited) != 0;
        phase ^= 1u;
        fence_after_sync();
        return ok;
    };

    const uint32_t n_tiles = (n + kTrRows - 1) / kTrRows;
    for (uint32_t tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
        const uint32_t row = tile * kTrRows + tid;
        const bool live = row < n, keep = row < n_pad;
        // the encoded input: A tile of layer 0, and X column-major for dW_0
        {
            float f[kMlpRaw];
            const float4 *src = reinterpret_cast<const float4 *>(raw + (size_t)row * kMlpRaw);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const float4 q = live ? src[k] : make_float4(0.f, 0.f, 0.f, 0.f);
                f[4 * k] = q.x;
                f[4 * k + 1] = q.y;
                f[4 * k + 2] = q.z;
                f[4 * k + 3] = q.w;
            }
#pragma unroll 1
            for (int c = 0; c < kMlpIn / 8; c++) {
                float v[8];
#pragma unroll
                for (int e = 0; e < 8; e += 2) {
                    const float2 p = encode_pair(f, 8 * c + e, M);
                    v[e] = live ? p.x : 0.f;
                    v[e + 1] = live ? p.y : 0.f;
                }
                put_chunk(xz_s, tid, c, kMlpIn, v);
                if (keep) {
#pragma unroll
                    for (int e = 0; e < 8; e++) M.xcm[(size_t)(8 * c + e) * cap + row] = __float2bfloat16_rn(v[e]);
                }
            }
        }
        // forward
#pragma unroll 1
        for (int l = 0; l < kMlpLayers && ok; l++) {
            cta_sync_for_mma();
            if (tid == 0)
                issue_layer(tmem, l == 0 ? xz_a : h_a + (uint32_t)((l - 1) * kTrH), wf_a + umma_off(l) * 2, mlp_in(l),
                            umma_n(l), bar_a);
            if (!wait_layer()) break;
            if (l < kMlpLayers - 1) {
                unsigned char *ht = h_s + (size_t)l * kTrH;
                __nv_bfloat16 *hg = M.hcm + (size_t)l * kMlpHid * cap;
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    float v[16];
                    tmem_ld16(taddr + q * 16, v);
                    tmem_wait_ld();
#pragma unroll
                    for (int e = 0; e < 16; e++) v[e] = fmaxf(v[e], 0.f);
                    put_chunk(ht, tid, 2 * q, kMlpHid, v);
                    put_chunk(ht, tid, 2 * q + 1, kMlpHid, v + 8);
                    if (keep) {
#pragma unroll
                        for (int e = 0; e < 16; e++) hg[(size_t)(16 * q + e) * cap + row] = __float2bfloat16_rn(v[e]);
                    }
                }
            } else {
                // loss and dL/dy (mean over rows and RGB of (y - t)^2 / (y^2 + 0.01))
                float y[16];
                tmem_ld16(taddr, y);
                tmem_wait_ld();
                float d[16];
#pragma unroll
                for (int e = 0; e < 16; e++) d[e] = 0.f;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    if (live) {
                        const float t = target[(size_t)row * 3 + c];
                        const float den = y[c] * y[c] + 0.01f;
                        const float diff = y[c] - t;
                        loss += diff * diff / den;
                        d[c] = 2.f * diff / den * inv_count;
                    }
                }
                // dZ_5 as the A tile of the first backward layer (K = 16)
                put_chunk(xz_s, tid, 0, 16, d);
                put_chunk(xz_s, tid, 1, 16, d + 8);
                if (keep) {
                    __nv_bfloat16 *dz5 = M.dzcm + (size_t)(kMlpLayers - 1) * kMlpHid * cap;
#pragma unroll
                    for (int c = 0; c < kMlpOutP; c++) dz5[(size_t)c * cap + row] = __float2bfloat16_rn(d[c]);
                }
            }
        }
        if (!ok) break;
        // backward: dZ_{l-1} = (dZ_l W_l^T) * (H_{l-1} > 0)
#pragma unroll 1
        for (int l = kMlpLayers - 1; l >= 1; l--) {
            cta_sync_for_mma();
            if (tid == 0) issue_layer(tmem, xz_a, wb_a + umma_boff(l) * 2, umma_bk(l), mlp_in(l), bar_a);
            if (!wait_layer()) break;
            const unsigned char *ht = h_s + (size_t)(l - 1) * kTrH;
            __nv_bfloat16 *dzg = M.dzcm + (size_t)(l - 1) * kMlpHid * cap;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                float v[16];
                tmem_ld16(taddr + q * 16, v);
                tmem_wait_ld();
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    // this row's 8 activations of chunk 2q + h (the K-major tile's 16-byte row piece)
                    const int c = 2 * q + h;
                    const uint4 hv = *reinterpret_cast<const uint4 *>(ht + (size_t)(tid / 8) * (kMlpHid / 8) * 128 +
                                                                      (size_t)c * 128 + (tid % 8) * 16);
                    const uint32_t w4[4] = {hv.x, hv.y, hv.z, hv.w};
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        if (!((w4[e] & 0x7fffu) != 0u && !(w4[e] & 0x8000u))) v[8 * h + 2 * e] = 0.f;
                        if (!((w4[e] >> 16 & 0x7fffu) != 0u && !(w4[e] & 0x80000000u))) v[8 * h + 2 * e + 1] = 0.f;
                    }
                }
                put_chunk(xz_s, tid, 2 * q, kMlpHid, v);
                put_chunk(xz_s, tid, 2 * q + 1, kMlpHid, v + 8);
                if (keep) {
#pragma unroll
                    for (int e = 0; e < 16; e++) dzg[(size_t)(16 * q + e) * cap + row] = __float2bfloat16_rn(v[e]);
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if ((tid & 31) == 0 && loss != 0.f) atomicAdd(M.loss, loss / (3.f * (float)n));
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTrTmemCols) : "memory");
}

// the batch rows (K) one CTA sums; measured on a B200 (16,384-row step):
// 1024 rows 12 % slower, 256 rows 2 % slower
constexpr uint32_t kDwTcRowsPerCta = 512;
constexpr int kDwTcK = 64;                  // rows per MMA group

__global__ void __launch_bounds__(128) k_mlp_dw_tc(const MlpDev M, uint32_t n_pad)
{
    __shared__ __align__(1024) unsigned char a_s[128 * kDwTcK * 2];  // M = 128 features x K = 64 rows
    __shared__ __align__(1024) unsigned char b_s[64 * kDwTcK * 2];   // N (<= 64) features x K = 64 rows
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base_s;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int l = blockIdx.y;
    const int in = mlp_in(l), out = mlp_out(l), N = umma_n(l);
    const size_t cap = M.cap;
    const __nv_bfloat16 *A = l == 0 ? M.xcm : M.hcm + (size_t)(l - 1) * kMlpHid * cap;
    const __nv_bfloat16 *B = M.dzcm + (size_t)l * kMlpHid * cap;
    // features past the layer's own stay zero in both tiles
    for (int i = tid; i < (int)(sizeof(a_s) / 16); i += 128) reinterpret_cast<uint4 *>(a_s)[i] = make_uint4(0u, 0u, 0u, 0u);
    for (int i = tid; i < (int)(sizeof(b_s) / 16); i += 128) reinterpret_cast<uint4 *>(b_s)[i] = make_uint4(0u, 0u, 0u, 0u);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                     "r"(kTrTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_base_s;
    const uint32_t bar_a = smem_u32(&bar), a_a = smem_u32(a_s), b_a = smem_u32(b_s);
    uint32_t phase = 0;
    bool ok = true, any = false;
    const uint32_t k_begin = blockIdx.x * kDwTcRowsPerCta;
    const uint32_t k_end = min(n_pad, k_begin + kDwTcRowsPerCta);
    for (uint32_t k0 = k_begin; k0 < k_end && ok; k0 += kDwTcK) {
        // 16-byte pieces: (feature f, 8-row group g) -> core matrix (f / 8, g), row f % 8
        for (int u = tid; u < in * (kDwTcK / 8); u += 128) {
            const int f = u / (kDwTcK / 8), g = u % (kDwTcK / 8);
            const uint32_t r = k0 + 8u * g;
            const uint4 v = r < k_end ? *reinterpret_cast<const uint4 *>(A + (size_t)f * cap + r) : make_uint4(0u, 0u, 0u, 0u);
            *reinterpret_cast<uint4 *>(a_s + (size_t)(f / 8) * (kDwTcK / 8) * 128 + g * 128 + (f % 8) * 16) = v;
        }
        for (int u = tid; u < out * (kDwTcK / 8); u += 128) {
            const int f = u / (kDwTcK / 8), g = u % (kDwTcK / 8);
            const uint32_t r = k0 + 8u * g;
            const uint4 v = r < k_end ? *reinterpret_cast<const uint4 *>(B + (size_t)f * cap + r) : make_uint4(0u, 0u, 0u, 0u);
            *reinterpret_cast<uint4 *>(b_s + (size_t)(f / 8) * (kDwTcK / 8) * 128 + g * 128 + (f % 8) * 16) = v;
        }
        cta_sync_for_mma();
        if (tid == 0) {
            const uint32_t idesc = umma_idesc(128, N);
            for (int s = 0; s < kDwTcK / 16; s++) {
                const uint64_t da = umma_desc(a_a + s * 256, 128, (kDwTcK / 8) * 128);
                const uint64_t db = umma_desc(b_a + s * 256, 128, (kDwTcK / 8) * 128);
                mma_bf16(tmem, da, db, idesc, (any || s > 0) ? 1u : 0u);
            }
            mma_commit(bar_a);
        }
        const bool waited = mbar_wait(bar_a, phase);
        if (!waited) atomicOr(M.err, kErrWait);
        ok = __syncthreads_and(waited) != 0;
        phase ^= 1u;
        fence_after_sync();
        any = true;
    }
    if (ok && any) {
        // row `tid` of dW_l: feature tid, the N accumulator columns
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
        float *g = M.grad + mlp_off(l);
        for (int q = 0; q < N / 16; q++) {
            float v[16];
            tmem_ld16(taddr + q * 16, v);
            tmem_wait_ld();
            if (tid < in) {
#pragma unroll
                for (int e = 0; e < 16; e++) {
                    const int o = 16 * q + e;
                    if (o < out) atomicAdd(g + (size_t)tid * out + o, v[e]);
                }
            }
        }
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTrTmemCols) : "memory");
}

}  // namespace

cudaError_t mlp_train_tc(const MlpDev &M, const float *raw, const float *target, uint32_t n, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    if ((uintptr_t)raw & 15u) return cudaErrorMisalignedAddress;  // rows are read as 16-byte vectors
    const uint32_t n_pad = (n + 15) / 16 * 16;
    if (n_pad > M.cap) return cudaErrorInvalidValue;
    cudaError_t e = ensure_dynamic_smem((const void *)k_mlp_train_tc, (int)kTrSmem);
    if (e != cudaSuccess) return e;
    const uint32_t tiles = (n + kTrRows - 1) / kTrRows;
    const uint32_t sms = (uint32_t)current_sm_count();
    k_mlp_train_tc<<<tiles < sms ? tiles : sms, kTrRows, kTrSmem, st>>>(M, raw, target, n, n_pad);
    return cudaGetLastError();
}

cudaError_t mlp_dw_tc(const MlpDev &M, uint32_t n_pad, cudaStream_t st)
{
    if (n_pad == 0) return cudaSuccess;
    if (n_pad > M.cap || (n_pad & 15u) || (M.cap & 15u)) return cudaErrorInvalidValue;
    const dim3 grid((n_pad + kDwTcRowsPerCta - 1) / kDwTcRowsPerCta, kMlpLayers);
    // 6 KB of unused dynamic shared memory keep at most 7 CTAs on an SM, so
    // their 64-column TMEM allocations always fit the SM's 512 columns
    k_mlp_dw_tc<<<grid, 128, 6 * 1024, st>>>(M, n_pad);
    return cudaGetLastError();
}

}  // namespace ilg
