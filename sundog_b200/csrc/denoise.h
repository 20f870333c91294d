// Film denoiser (denoise.cu).
#pragma once

#include <cuda_runtime.h>

namespace sdb {

struct DenoiseParams {
  int passes = 5;            // a-trous passes (holes 1, 2, 4, ...)
  float sigmaColor = 0.4f;   // tone-compressed colour tolerance of the first pass
  float sigmaNormal = 0.3f;  // normal-AOV tolerance
  float sigmaAlbedo = 0.1f;  // albedo-AOV tolerance
};
DenoiseParams denoiseDefaults();

// Denoised copy of a w x h float4 film (device) into out (device), guided by
// the first-hit albedo and camera-space normal AOVs; waits for the stream.
void denoiseFilm(const float4* film, const float4* albedo, const float4* normal, int w, int h,
                 const DenoiseParams& p, float4* out, cudaStream_t st);

}  // namespace sdb
