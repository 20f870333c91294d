// Host entry points of the CUDA translation units (launch wrappers).
#pragma once

#include <cuda_runtime.h>

#include "sd_types.h"

namespace sdb {

constexpr int kRenderBlock = 128;

// Path tracer (pt_kernel.cu).
cudaError_t setLaunch(const SdLaunch& lp, cudaStream_t st);
int renderGridSize();
cudaError_t launchRender(cudaStream_t st, int grid);
cudaError_t launchFold(int npix, cudaStream_t st);
struct TraceCount;  // sd_trace.cuh: four u64 counters
// Same kernel with traversal visit counters (node box tests, triangle and
// quadric tests, BLAS entries) summed into counts; for the roofline only.
cudaError_t launchRenderCounting(cudaStream_t st, int grid, TraceCount* counts);

}  // namespace sdb
