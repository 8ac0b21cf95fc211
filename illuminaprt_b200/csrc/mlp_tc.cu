// Radiance-cache inference on the 5th-generation tensor cores.
//
// A CTA runs kTcGroups independent pipelines of 128 threads. Each group owns
// one 128-row tile of queries at a time (one row per thread, which is the
// TMEM lane the row's accumulator lives in) and takes it through all six
// layers without leaving the CTA:
//   * the weights (all layers, 46 KiB of BF16) sit in shared memory once per
//     CTA, as W^T in the UMMA K-major no-swizzle layout: 8-row x 16-byte core
//     matrices, the two K halves of one instruction 128 bytes apart (LBO),
//     consecutive 8-row groups K/8 x 128 bytes apart (SBO);
//   * each thread writes its row's activations (the encoded input, then each
//     hidden layer after ReLU and rounding to BF16) into its group's
//     shared-memory A tile in the same layout;
//   * one elected thread per group issues the layer's K/16 tcgen05.mma
//     instructions (M = 128, N = 64 or 16, K = 16, BF16 x BF16 -> FP32 into
//     the group's 64 TMEM columns) and commits them to the group's mbarrier;
//   * the group's threads wait on it (bounded), read their rows back from
//     TMEM with tcgen05.ld, apply ReLU and write the next A tile.
// The groups synchronise on their own named barriers, so while one group
// drains its accumulator and writes activations, the tensor core runs the
// other groups' layers: kTcGroups tiles are in flight per SM (the A tiles
// share one copy of the weights, so shared memory holds six). TMEM is
// allocated once per CTA and freed on exit; every wait has an iteration
// limit that raises an error bit instead of hanging.
#include "devinfo.cuh"
#include "mlp.cuh"
#include "umma.cuh"

namespace ilg {

namespace {

using namespace umma;

constexpr int kTcRows = 128;
constexpr int kTcGroups = 6;         // tile pipelines per CTA
constexpr uint32_t kTmemCols = 512;  // power of two >= 64 per group
constexpr size_t kWBytes = ((kUmmaElems * 2 + 1023) / 1024) * 1024;
constexpr size_t kATileBytes = (size_t)kTcRows * kMlpIn * 2;
static_assert(64 * kTcGroups <= (int)kTmemCols, "TMEM columns for every group");
static_assert(kWBytes + kTcGroups * kATileBytes <= 227 * 1024, "shared memory per CTA");

// Barrier of one group's 128 threads (named barrier 1 + group).
__device__ __forceinline__ void group_sync(int id)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(kTcRows) : "memory");
}

// Barrier of one group's threads that also ANDs a predicate over them.
__device__ __forceinline__ bool group_and(int id, bool v)
{
    uint32_t r;
    asm volatile(
        "{\n\t"
        ".reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t"
        "}\n"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id), "r"(kTcRows)
        : "memory");
    return r != 0;
}

// The grid columns of every query, one thread per (row, level): the gathers
// of all levels of all rows in flight at once, at full occupancy, instead of
// one thread walking its row's sixteen levels in turn inside the tensor-core
// kernel (whose shared memory allows three CTAs per SM).
__global__ void __launch_bounds__(256) k_grid_encode(const MlpDev M, const float *__restrict__ raw, uint32_t n,
                                                     const uint32_t *__restrict__ n_dev)
{
    if (n_dev) n = min(n, *n_dev);
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t row = (uint32_t)(i / kGridLevels), l = (uint32_t)(i % kGridLevels);
    if (row >= n) return;
    const float *f = raw + (size_t)row * kMlpRaw;
    const float2 g = grid_features(M, (int)l, f[0], f[1], f[2]);
    M.enc[i] = pack2(g.x, g.y);
}

__global__ void __launch_bounds__(kTcRows * kTcGroups, 1)
    k_mlp_infer_tc(const MlpDev M, const float *__restrict__ raw, uint32_t n, const uint32_t *__restrict__ n_dev,
                   float *__restrict__ out, uint32_t *__restrict__ err)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *w_s = smem;  // kUmmaElems bf16
    __shared__ __align__(8) uint64_t bar[kTcGroups];
    __shared__ uint32_t tmem_base_s;

    if (n_dev) n = min(n, *n_dev);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int grp = tid / kTcRows, lt = tid % kTcRows;
    const int bar_id = 1 + grp;
    unsigned char *a_s = smem + kWBytes + (size_t)grp * kATileBytes;  // this group's 128 x 96 bf16 tile
    // weights -> shared memory (16-byte vectors)
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(M.wu);
        uint4 *dst = reinterpret_cast<uint4 *>(w_s);
        for (int i = tid; i < kUmmaElems / 8; i += blockDim.x) dst[i] = src[i];
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid < kTcGroups) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[tid])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    // this group's 64 accumulator columns; this warp's 32 TMEM lanes
    const uint32_t tmem = tmem_base_s + (uint32_t)(64 * grp);
    const uint32_t taddr = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    const uint32_t bar_a = smem_u32(&bar[grp]);
    const uint32_t w_a = smem_u32(w_s), a_a = smem_u32(a_s);
    uint32_t phase = 0;
    bool ok = true;

    const uint32_t n_tiles = (n + kTcRows - 1) / kTcRows;
    // the row's 16 raw features as four 16-byte loads, issued one tile ahead
    float4 fv[4];
    auto load_row = [&](uint32_t tile) {
        const uint32_t row = tile * kTcRows + lt;
        const float4 *src = reinterpret_cast<const float4 *>(raw + (size_t)row * kMlpRaw);
#pragma unroll
        for (int k = 0; k < 4; k++) fv[k] = (tile < n_tiles && row < n) ? src[k] : make_float4(0.f, 0.f, 0.f, 0.f);
    };
    load_row(blockIdx.x * kTcGroups + grp);
    for (uint32_t tile = blockIdx.x * kTcGroups + grp; tile < n_tiles && ok; tile += gridDim.x * kTcGroups) {
        const uint32_t row = tile * kTcRows + lt;
        // encoded input row -> A tile (K = 96)
        {
            float f[kMlpRaw];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                f[4 * k] = fv[k].x;
                f[4 * k + 1] = fv[k].y;
                f[4 * k + 2] = fv[k].z;
                f[4 * k + 3] = fv[k].w;
            }
            load_row(tile + gridDim.x * kTcGroups);
            if (M.encoding == kEncFreq12) {
                // per axis: the anchors of bands 0, 4, 8 and three doublings
                // each (the values freq_band gives), one chunk per anchor
#pragma unroll
                for (int a = 0; a < 3; a++) {
#pragma unroll
                    for (int j = 0; j < 3; j++) {
                        float v[8], sn, cs;
                        sincospif(ldexpf(f[a], 4 * j), &sn, &cs);
#pragma unroll
                        for (int k = 0; k < 4; k++) {
                            if (k) freq_double(sn, cs);
                            v[2 * k] = row < n ? sn : 0.f;
                            v[2 * k + 1] = row < n ? cs : 0.f;
                        }
                        put_chunk(a_s, lt, 3 * a + j, kMlpIn, v);
                    }
                }
#pragma unroll
                for (int c = 9; c < kMlpIn / 8; c++) {
                    float v[8];
#pragma unroll
                    for (int e = 0; e < 8; e += 2) {
                        const float2 p = encode_pair_freq(f, 8 * c + e);
                        v[e] = row < n ? p.x : 0.f;
                        v[e + 1] = row < n ? p.y : 0.f;
                    }
                    put_chunk(a_s, lt, c, kMlpIn, v);
                }
            } else
#pragma unroll
            for (int c = 0; c < kMlpIn / 8; c++) {
                float v[8];
                if (M.enc && c < 2 * kGridLevels / 8) {
                    // grid columns precomputed by k_grid_encode (BF16, exact here)
                    const uint4 q = row < n ? *reinterpret_cast<const uint4 *>(M.enc + (size_t)row * kGridLevels + 4 * c)
                                            : make_uint4(0u, 0u, 0u, 0u);
                    const uint32_t w4[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        v[2 * e] = __uint_as_float(w4[e] << 16);
                        v[2 * e + 1] = __uint_as_float(w4[e] & 0xffff0000u);
                    }
                    put_chunk(a_s, lt, c, kMlpIn, v);
                    continue;
                }
#pragma unroll
                for (int e = 0; e < 8; e += 2) {
                    const float2 p = encode_pair(f, 8 * c + e, M);
                    v[e] = row < n ? p.x : 0.f;
                    v[e + 1] = row < n ? p.y : 0.f;
                }
                put_chunk(a_s, lt, c, kMlpIn, v);
            }
        }
#pragma unroll 1
        for (int l = 0; l < kMlpLayers; l++) {
            const int K = mlp_in(l), N = umma_n(l);
            fence_async_smem();
            fence_before_sync();
            group_sync(bar_id);
            fence_after_sync();
            if (lt == 0) {
                const uint32_t idesc = umma_idesc(kTcRows, N);
                for (int s = 0; s < K / 16; s++) {
                    // K step s covers core-matrix chunks 2s, 2s+1
                    const uint64_t da = umma_desc(a_a + s * 256, 128, (K / 8) * 128);
                    const uint64_t db = umma_desc(w_a + umma_off(l) * 2 + s * 256, 128, (K / 8) * 128);
                    mma_bf16(tmem, da, db, idesc, s > 0 ? 1u : 0u);
                }
                mma_commit(bar_a);
            }
            const bool waited = mbar_wait(bar_a, phase);
            if (!waited) atomicOr(err, kErrWait);
            ok = group_and(bar_id, waited);  // the group's threads leave together
            if (!ok) break;
            phase ^= 1u;
            fence_after_sync();
            if (l < kMlpLayers - 1) {
                // 64 columns in four 16-column loads; ReLU and the BF16
                // rounding in one cvt per pair
#pragma unroll
                for (int h = 0; h < 4; h++) {
                    uint32_t r[16];
                    tmem_ld16(taddr + h * 16, r);
                    tmem_wait_ld();
#pragma unroll
                    for (int c = 0; c < 2; c++)
                        put_chunk_bits(a_s, lt, 2 * h + c, kMlpHid,
                                       make_uint4(pack2_relu(r[8 * c], r[8 * c + 1]), pack2_relu(r[8 * c + 2], r[8 * c + 3]),
                                                  pack2_relu(r[8 * c + 4], r[8 * c + 5]),
                                                  pack2_relu(r[8 * c + 6], r[8 * c + 7])));
                }
            } else {
                float v[16];
                tmem_ld16(taddr, v);
                tmem_wait_ld();
                if (row < n) {
                    out[(size_t)row * 3] = v[0];
                    out[(size_t)row * 3 + 1] = v[1];
                    out[(size_t)row * 3 + 2] = v[2];
                }
            }
        }
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base_s), "r"(kTmemCols)
                     : "memory");
}

}  // namespace

cudaError_t mlp_infer_tc(const MlpDev &M, const float *raw, uint32_t n, float *out, cudaStream_t st,
                         const uint32_t *n_dev, uint32_t *err)
{
    if (n == 0) return cudaSuccess;
    if ((uintptr_t)raw & 15u) return cudaErrorMisalignedAddress;  // rows are read as 16-byte vectors
    const size_t smem = kWBytes + kTcGroups * kATileBytes;
    cudaError_t e = ensure_dynamic_smem((const void *)k_mlp_infer_tc, (int)smem);
    if (e != cudaSuccess) return e;
    const int sms = current_sm_count();
    const uint32_t tiles = (n + kTcRows - 1) / kTcRows;
    const uint32_t ctas = (tiles + kTcGroups - 1) / kTcGroups;
    const uint32_t grid = ctas < (uint32_t)sms ? ctas : (uint32_t)sms;  // one CTA per SM (shared memory)
    MlpDev Mi = M;
    if (M.enc && n <= M.enc_cap) {
        k_grid_encode<<<(unsigned)(((uint64_t)n * kGridLevels + 255) / 256), 256, 0, st>>>(M, raw, n, n_dev);
    } else {
        Mi.enc = nullptr;
    }
    k_mlp_infer_tc<<<grid, kTcRows * kTcGroups, smem, st>>>(Mi, raw, n, n_dev, out, err);
    return cudaGetLastError();
}

}  // namespace ilg
