// Host entry points of the CUDA translation units (launch wrappers).
#pragma once

#include <cuda_runtime.h>

#include "sd_types.h"

namespace sdb {

#ifndef SDB_RENDER_BLOCK
#define SDB_RENDER_BLOCK 128
#endif
// Resident 128-thread blocks per SM the path kernels are compiled for: 16
// (2048 threads, the SM's limit) caps them at 32 registers. The kernel is
// latency-bound, so occupancy beats the spills it costs: measured 653, 709,
// 776 and 829 Mrays/s at 6, 8, 12 and 16 blocks on the instancing frame.
#ifndef SDB_MIN_BLOCKS
#define SDB_MIN_BLOCKS 16
#endif
constexpr int kRenderBlock = SDB_RENDER_BLOCK;

// Path tracer (pt_kernel.cu).
cudaError_t setLaunch(const SdLaunch& lp, cudaStream_t st);
// BVH layout the kernels were compiled for: 2 (BvhNode) or 8 (CwNode).
int bvhWidth();
int renderGridSize();
// guide: 0 plain; kGuideSample / kGuideRecord bits select the guided variants.
cudaError_t launchRender(cudaStream_t st, int grid, int guide = 0);
cudaError_t launchFold(int npix, cudaStream_t st);
// Same kernel with traversal visit counters (node box tests, triangle and
// quadric tests, BLAS entries) summed into counts; for the roofline only.
cudaError_t launchRenderCounting(cudaStream_t st, int grid, TraceCount* counts);

}  // namespace sdb
