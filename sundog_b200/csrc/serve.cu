// Serving kernels: one persistent launch renders tile-passes of many jobs.
//
// A batch is a list of tile-passes (job slot, pixel rectangle, sample
// range). Path ids run over the batch: item i owns ids [pathBegin_i,
// pathBegin_i + npad_i * sampleCount_i), with the item's pixels in 8x8 blocks
// (npad_i = the rectangle rounded up to whole blocks) so a warp starts on an
// 8x4 patch of neighbouring camera rays. The kernel keeps the path tracer's
// lane refill (ptPersistent): a lane whose path ends takes the next id,
// whatever job it belongs to, so jobs share warps and the launch stays full
// until the batch runs dry. A lane reads its job's launch block from the
// constant-memory job table.
//
// ptServeFold folds each item's samples into its job's film in sample order
// with the running mean of device/programs.cu:560-563, so a job's film is
// bit-identical to a plain render of it.
#include "pt_path.cuh"
#include "serve.h"

namespace sdb {

__constant__ SdLaunch c_jobs[kMaxServeJobs];
__constant__ ServeBatch c_batch;

static_assert(sizeof(SdLaunch) * kMaxServeJobs <= 48 * 1024, "job table exceeds constant memory");

// Path id -> camera sample; false for block padding.
__device__ __forceinline__ bool serveStart(unsigned long long id, Path& p, int& job) {
  const ServeBatch& b = c_batch;
  int lo = 0, hi = b.numItems - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (b.items[mid].pathBegin <= id) lo = mid;
    else hi = mid - 1;
  }
  const ServeItem& it = b.items[lo];
  unsigned long long local = id - it.pathBegin;
  int sLocal = (int)(local / (unsigned long long)it.npad);
  int rem = (int)(local - (unsigned long long)sLocal * it.npad);
  int blk = rem >> 6, within = rem & 63;
  int lx = (blk % it.bw) * 8 + (within & 7), ly = (blk / it.bw) * 8 + (within >> 3);
  if (lx >= it.w || ly >= it.h) return false;
  job = it.job;
  startPathAt(c_jobs[job], it.x0 + lx, it.y0 + ly, it.sampleBegin + sLocal, p);
  p.slot = 0;
  return true;
}

__global__ void __launch_bounds__(kRenderBlock, SDB_MIN_BLOCKS) ptServe() {
  const ServeBatch& b = c_batch;
  const unsigned full = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31;
  const unsigned ltMask = (1u << lane) - 1u;
  unsigned long long rays = 0;
  bool active = false;
  bool exhausted = false;  // warp-uniform
  unsigned long long myId = 0;
  int job = 0;
  Path p;
  p.slot = 0;
  while (true) {
    if (!exhausted) {
      unsigned need = __ballot_sync(full, !active);
      if (need) {
        int leader = __ffs(need) - 1;
        unsigned long long base = 0;
        if (lane == leader) base = atomicAdd(b.pathCounter, (unsigned long long)__popc(need));
        base = __shfl_sync(full, base, leader);
        if (base + __popc(need) >= b.numPaths) exhausted = true;
        if (!active) {
          unsigned long long id = base + __popc(need & ltMask);
          if (id < b.numPaths) {
            active = serveStart(id, p, job);
            myId = id;
          }
        }
      }
    }
    if (!__any_sync(full, active)) {
      if (exhausted) break;
      continue;
    }
    if (active) {
      if (!bounce<false>(c_jobs[job], p, rays, nullptr)) {
        float3 L = sanitize3(p.L);
        b.sampleL[myId] = make_float4(L.x, L.y, L.z, 1.0f);
        active = false;
      }
    }
  }
  for (int off = 16; off > 0; off >>= 1) rays += __shfl_down_sync(full, rays, off);
  if (lane == 0 && rays) atomicAdd(b.rayCounter, rays);
}

// One block per item: running mean of the item's samples into its job's film.
__global__ void ptServeFold() {
  const ServeBatch& b = c_batch;
  const ServeItem& it = b.items[blockIdx.x];
  const SdLaunch& lp = c_jobs[it.job];
  if (!lp.accum) return;  // an empty table slot: nothing to fold into
  const int npt = it.w * it.h;
  for (int q = threadIdx.x; q < npt; q += blockDim.x) {
    int lx = q % it.w, ly = q / it.w;
    int rem = ((ly >> 3) * it.bw + (lx >> 3)) * 64 + (ly & 7) * 8 + (lx & 7);
    size_t pix = (size_t)(it.y0 + ly) * lp.width + it.x0 + lx;
    float4 acc = lp.accum[pix];
    for (int k = 0; k < it.sampleCount; k++) {
      float4 x = b.sampleL[it.pathBegin + (unsigned long long)k * it.npad + rem];
      int s1 = it.sampleBegin + k + 1;
      acc = make_float4(acc.x + (x.x - acc.x) / s1, acc.y + (x.y - acc.y) / s1,
                        acc.z + (x.z - acc.z) / s1, 1.0f);
    }
    lp.accum[pix] = acc;
  }
}

cudaError_t serveSetJobs(const SdLaunch* table, cudaStream_t st) {
  return cudaMemcpyToSymbolAsync(c_jobs, table, kMaxServeJobs * sizeof(SdLaunch), 0,
                                 cudaMemcpyHostToDevice, st);
}

int serveGridSize() {
  int dev = 0, sms = 0, perSm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, ptServe, kRenderBlock, 0);
  if (perSm < 1) perSm = 1;
  return sms * perSm;
}

cudaError_t serveLaunch(const ServeBatch& batch, int grid, cudaStream_t st) {
  cudaError_t e = cudaMemcpyToSymbolAsync(c_batch, &batch, sizeof batch, 0,
                                          cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  ptServe<<<grid, kRenderBlock, 0, st>>>();
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  ptServeFold<<<batch.numItems, 256, 0, st>>>();
  return cudaGetLastError();
}

cudaError_t serveFold(const ServeBatch& batch, cudaStream_t st) {
  cudaError_t e = cudaMemcpyToSymbolAsync(c_batch, &batch, sizeof batch, 0,
                                          cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  ptServeFold<<<batch.numItems, 256, 0, st>>>();
  return cudaGetLastError();
}

}  // namespace sdb
