// Device post-processing of rendered images (postproc.cu).
#pragma once

#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

namespace ilg {

// acc += in; out = acc * (1 / frames)   (rgb floats, n_pixels x 3)
cudaError_t post_accumulate(const float *in, float *acc, float *out, uint32_t n_pixels, uint32_t frames,
                            cudaStream_t st);
// op 0 GlobalTone, 1 AutoTone, 2 DragoTone; scratch holds post_scratch_floats(n_pixels) floats
cudaError_t post_tonemap(const float *in, float *out, uint32_t n_pixels, uint32_t op, float *scratch,
                         cudaStream_t st);
uint32_t post_scratch_floats(uint32_t n_pixels);

}  // namespace ilg
