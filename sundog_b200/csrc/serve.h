// Shared between the serving kernels (serve.cu) and the server (serve_host.cpp).
#pragma once

#include <cuda_runtime.h>

#include "sd_types.h"

namespace sdb {

constexpr int kMaxServeJobs = 32;

// One tile-pass: samples [sampleBegin, sampleBegin + sampleCount) of the
// w x h pixel rectangle at (x0, y0) of the job in slot `job`.
struct ServeItem {
  int job;
  int x0, y0, w, h;
  int bw;                        // 8x8 blocks across the rectangle
  int npad;                      // pixels rounded up to whole 8x8 blocks
  int sampleBegin, sampleCount;
  int pad0;
  unsigned long long pathBegin;  // first path id of the item in the batch
};

struct ServeBatch {
  const ServeItem* items;        // device array, sorted by pathBegin
  int numItems;
  unsigned long long numPaths;
  unsigned long long* pathCounter;
  unsigned long long* rayCounter;
  float4* sampleL;               // radiance per path id
};

// Writes a job's launch block into slot `slot` of the device job table
// (ordered on st before later launches).
// The whole job table (kMaxServeJobs launch blocks, host memory; unused slots
// zero) into the megakernel server's constant memory.
cudaError_t serveSetJobs(const SdLaunch* table, cudaStream_t st);
int serveGridSize();
// The batch's persistent render launch followed by its fold launch.
cudaError_t serveLaunch(const ServeBatch& batch, int grid, cudaStream_t st);
// The fold launch alone, for a batch rendered by the wavefront engine.
cudaError_t serveFold(const ServeBatch& batch, cudaStream_t st);

}  // namespace sdb
