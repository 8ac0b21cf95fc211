// Progressive accumulation and tone mapping of rendered images on the device:
// the post-processes the reference applies to its RadianceBuffer after each
// frame (Core/Postproc/*.h), done where the frame already is, so a
// progressive renderer copies only the displayed image back to the host.
//
//   k_accumulate     AccumulationBuffer::Apply (AccumulationBuffer.h:59-87):
//                    acc = in + acc; out = acc * (1 / frames)
//   k_tone_global    GlobalTone::Apply (GlobalTone.h:39-57): c / (c + 1)
//   k_minmax_*       per-channel minimum (from FLT_MAX) and maximum (from 0)
//                    over the image, as AutoTone and DragoTone scan it
//   k_tone_auto      AutoTone::Apply (AutoTone.h:37-75): (c - low) / (high - low),
//                    clamped to [0, 1]
//   k_tone_drago     DragoTone::Apply (DragoTone.h:37-81) with its fixed bias
//                    0.8 and scale 0.95: each logarithm and power evaluated in
//                    double and rounded to float, as the reference's
//                    Maths::Log / LogBase / Pow do (Maths.h:63-122)
//
// Every float operation is the reference's, rounded separately, so the
// accumulation, GlobalTone and AutoTone are bit for bit the reference's.
#include <cfloat>
#include <cuda_runtime.h>

#include "postproc.cuh"

namespace ilg {

namespace {

__global__ void k_accumulate(const float *__restrict__ in, float *__restrict__ acc, float *__restrict__ out,
                             uint32_t n3, float count_inv)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    const float a = __fadd_rn(in[i], acc[i]);
    acc[i] = a;
    out[i] = __fmul_rn(a, count_inv);
}

__global__ void k_tone_global(const float *__restrict__ in, float *__restrict__ out, uint32_t n3)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    const float c = in[i];
    out[i] = __fdiv_rn(c, __fadd_rn(c, 1.f));
}

constexpr int kReduceThreads = 256;

// Per-block minimum and maximum of each channel: part[6 * block + k] = min of
// channel k, part[6 * block + 3 + k] = max of channel k (max starts at 0, as
// the reference's scans do).
__global__ void __launch_bounds__(kReduceThreads) k_minmax_part(const float *__restrict__ in, uint32_t n,
                                                                float *__restrict__ part)
{
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {0.f, 0.f, 0.f};
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float c = in[3ull * p + k];
            lo[k] = fminf(lo[k], c);
            hi[k] = fmaxf(hi[k], c);
        }
    }
    __shared__ float s[6][kReduceThreads];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        s[k][threadIdx.x] = lo[k];
        s[3 + k][threadIdx.x] = hi[k];
    }
    __syncthreads();
    for (int w = kReduceThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
#pragma unroll
            for (int k = 0; k < 3; k++) {
                s[k][threadIdx.x] = fminf(s[k][threadIdx.x], s[k][threadIdx.x + w]);
                s[3 + k][threadIdx.x] = fmaxf(s[3 + k][threadIdx.x], s[3 + k][threadIdx.x + w]);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x < 6) part[6 * blockIdx.x + threadIdx.x] = s[threadIdx.x][0];
}

// Reduces the per-block results to part[0..5] (one block).
__global__ void __launch_bounds__(kReduceThreads) k_minmax_final(float *__restrict__ part, uint32_t blocks)
{
    __shared__ float s[6][kReduceThreads];
    float v[6] = {FLT_MAX, FLT_MAX, FLT_MAX, 0.f, 0.f, 0.f};
    for (uint32_t b = threadIdx.x; b < blocks; b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            v[k] = fminf(v[k], part[6 * b + k]);
            v[3 + k] = fmaxf(v[3 + k], part[6 * b + 3 + k]);
        }
    }
#pragma unroll
    for (int k = 0; k < 6; k++) s[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int w = kReduceThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
#pragma unroll
            for (int k = 0; k < 3; k++) {
                s[k][threadIdx.x] = fminf(s[k][threadIdx.x], s[k][threadIdx.x + w]);
                s[3 + k][threadIdx.x] = fmaxf(s[3 + k][threadIdx.x], s[3 + k][threadIdx.x + w]);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x < 6) part[threadIdx.x] = s[threadIdx.x][0];
}

__device__ __forceinline__ float clamp01(float v) { return v < 0.f ? 0.f : (v > 1.f ? 1.f : v); }

__global__ void k_tone_auto(const float *__restrict__ in, float *__restrict__ out, uint32_t n3,
                            const float *__restrict__ mm)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    const int k = i % 3;
    const float low = mm[k], range = __fsub_rn(mm[3 + k], low);
    out[i] = clamp01(__fdiv_rn(__fsub_rn(in[i], low), range));
}

// Maths::Log (log10 in double, to float), Maths::LogBase, Maths::Pow
__device__ __forceinline__ float ref_log10(float v) { return (float)log10((double)v); }
__device__ __forceinline__ float ref_log_base(float v, float b) { return (float)(log((double)v) / log((double)b)); }
__device__ __forceinline__ float ref_pow(float b, float e) { return (float)pow((double)b, (double)e); }

__global__ void k_tone_drago(const float *__restrict__ in, float *__restrict__ out, uint32_t n3,
                             const float *__restrict__ mm)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    const int k = i % 3;
    const float lwmax = mm[3 + k];
    const float scale = __fmul_rn(95.f, 0.01f);
    const float bias = __fdiv_rn(ref_log10(0.8f), ref_log10(0.5f));
    const float c = in[i];
    const float a = __fdiv_rn(scale, ref_log_base(__fadd_rn(lwmax, 1.f), 10.f));
    const float num = ref_log10(__fadd_rn(c, 1.f));
    const float den = ref_log10(__fadd_rn(2.f, __fmul_rn(ref_pow(__fdiv_rn(c, lwmax), bias), 8.f)));
    out[i] = clamp01(__fdiv_rn(__fmul_rn(a, num), den));
}

inline uint32_t blocks_of(uint64_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

}  // namespace

cudaError_t post_accumulate(const float *in, float *acc, float *out, uint32_t n_pixels, uint32_t frames,
                            cudaStream_t st)
{
    if (n_pixels == 0) return cudaSuccess;
    const uint32_t n3 = 3u * n_pixels;
    const float count_inv = 1.0f / (float)frames;
    k_accumulate<<<blocks_of(n3, 256), 256, 0, st>>>(in, acc, out, n3, count_inv);
    return cudaGetLastError();
}

uint32_t post_scratch_floats(uint32_t n_pixels)
{
    const uint32_t blocks = std::min<uint32_t>(1024u, blocks_of(n_pixels, kReduceThreads));
    return 6u * (blocks < 1u ? 1u : blocks);
}

cudaError_t post_tonemap(const float *in, float *out, uint32_t n_pixels, uint32_t op, float *scratch,
                         cudaStream_t st)
{
    if (n_pixels == 0) return cudaSuccess;
    const uint32_t n3 = 3u * n_pixels;
    if (op == 0u) {
        k_tone_global<<<blocks_of(n3, 256), 256, 0, st>>>(in, out, n3);
        return cudaGetLastError();
    }
    const uint32_t blocks = post_scratch_floats(n_pixels) / 6u;
    k_minmax_part<<<blocks, kReduceThreads, 0, st>>>(in, n_pixels, scratch);
    k_minmax_final<<<1, kReduceThreads, 0, st>>>(scratch, blocks);
    if (op == 1u) k_tone_auto<<<blocks_of(n3, 256), 256, 0, st>>>(in, out, n3, scratch);
    else k_tone_drago<<<blocks_of(n3, 256), 256, 0, st>>>(in, out, n3, scratch);
    return cudaGetLastError();
}

}  // namespace ilg
