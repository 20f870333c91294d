// Film denoiser (denoise.cu).
#pragma once

#include <cuda_runtime.h>

namespace sdb {

struct DenoiseParams {
  int passes = 4;               // a-trous passes (holes 1, 2, 4, ...)
  float sigmaLuminance = 4.0f;  // luminance tolerance in local standard deviations
  float sigmaNormal = 0.2f;     // normal-AOV tolerance
  float sigmaAlbedo = 0.05f;    // albedo-AOV tolerance
};
DenoiseParams denoiseDefaults();

// Denoised copy of a w x h float4 film (device) into out (device), guided by
// the first-hit albedo and camera-space normal AOVs; waits for the stream.
void denoiseFilm(const float4* film, const float4* albedo, const float4* normal, int w, int h,
                 const DenoiseParams& p, float4* out, cudaStream_t st);

}  // namespace sdb
