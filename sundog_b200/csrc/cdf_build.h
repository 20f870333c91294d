// Device builds of the sampling tables (cdf_build.cu).
#pragma once

#include <cuda_runtime.h>

#include "scene_model.h"
#include "sd_types.h"

namespace sdb {

// Environment CDFs of a w x h float4 texel grid already on the device:
// marg (h + 1 floats) and cond (h * (w + 1) floats), device memory; waits for
// the stream. degenerate: the map has no luminance (uniform ramps stored).
void buildEnvCdfDevice(const float4* texels, int w, int h, float* marg, float* cond,
                       bool& degenerate, cudaStream_t st);

// Search guides (sd_types.h kCdfGuide) of `rows` CDFs of n entries each,
// row r at cdf + r * stride (device); guide receives rows x (kCdfGuide + 1)
// ints (device). Does not wait for the stream.
void buildCdfGuideDevice(const float* cdf, int n, size_t stride, int rows, int* guide,
                         cudaStream_t st);

// World-space vertices (worldPos, numVerts) and area CDF (cdf, numTris + 1
// floats) of a mesh instance whose object-space vertices and indices are on
// the device; returns the total area (FP64). Waits for the stream.
double buildMeshLightCdfDevice(const float3* pos, int numVerts, const uint3* idx, int numTris,
                               const Xform& xf, float3* worldPos, float* cdf, cudaStream_t st);

}  // namespace sdb
