// Path-tracing kernels for sm_100a.
//
// ptPersistent: a persistent megakernel. Each warp keeps 32 paths in flight;
// a lane whose path ends writes that sample's radiance to the per-sample
// buffer and immediately takes the next path index (one warp-aggregated
// atomicAdd per refill), so lanes stay busy while long paths finish. A path
// index maps to (sample, pixel) with the sample outermost and pixels in 8x8
// tiles, so a warp starts on an 8x4 block of neighbouring camera rays.
//
// ptFold: folds the per-sample values into the film in sample order with the
// reference's running mean acc += (x - acc) / (s + 1) (device/programs.cu:
// 560-563), which keeps the film bit-identical to a one-thread-per-pixel
// sequential loop regardless of which thread traced which sample.
//
// Guided variants (GUIDE != 0, sd_guide.cuh) draw directions by MIS with the
// learned guide and/or record training samples; GUIDE = 0 is the plain
// reference sampler with no guiding code compiled in.
//
// The path segment (bounce, pt_path.cuh) follows device/programs.cu:311-572.
#include "pt_path.cuh"

namespace sdb {

__constant__ SdLaunch c_lp;

template <bool COUNT, int GUIDE>
__global__ void __launch_bounds__(kRenderBlock, SDB_MIN_BLOCKS) ptPersistent(TraceCount* counts) {
  const SdLaunch& lp = c_lp;
  // Counting build: [0] radiance traversals and the path loop, [1] shadow
  // traversals.
  TraceCount cnt[2] = {{0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0}};
  const unsigned full = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31;
  const unsigned ltMask = (1u << lane) - 1u;
  unsigned long long rays = 0;
  bool active = false;
  bool exhausted = false;  // warp-uniform
  Path p;
  p.slot = 0;
  GuideTrail trail;
  trail.n = 0;

  while (true) {
    if (!exhausted) {
      unsigned need = __ballot_sync(full, !active);
      if (need) {
        int leader = __ffs(need) - 1;
        unsigned long long base = 0;
        if (lane == leader) base = atomicAdd(lp.pathCounter, (unsigned long long)__popc(need));
        base = __shfl_sync(full, base, leader);
        if (base + __popc(need) >= lp.numPaths) exhausted = true;
        if (!active) {
          unsigned long long id = base + __popc(need & ltMask);
          // Tile padding and indices past the end simply draw again next
          // round (padding) or leave the lane idle (past the end).
          if (id < lp.numPaths) active = startPath(lp, id, p);
          if (GUIDE & kGuideRecord) trail.n = 0;
        }
      }
    }
    if (!__any_sync(full, active)) {
      if (exhausted) break;
      continue;
    }
    if (active) {
      if (COUNT) countWarp(&cnt[0], cnt[0].loopIters, cnt[0].loopLanes);
      if (!bounce<COUNT, GUIDE>(lp, p, rays, cnt, &trail)) {
        float3 L = sanitize3(p.L);
        if (GUIDE & kGuideRecord) guideFlush(lp, trail, L);
        lp.sampleL[p.slot] = make_float4(L.x, L.y, L.z, 1.0f);
        active = false;
      }
    }
  }
  // One ray-counter update per warp.
  for (int off = 16; off > 0; off >>= 1) rays += __shfl_down_sync(full, rays, off);
  if (lane == 0 && rays) atomicAdd(lp.rayCounter, rays);
  if (COUNT) {
    for (int k = 0; k < 2; k++) {
      atomicAdd(&counts[k].boxTests, cnt[k].boxTests);
      atomicAdd(&counts[k].triTests, cnt[k].triTests);
      atomicAdd(&counts[k].quadTests, cnt[k].quadTests);
      atomicAdd(&counts[k].blasEntries, cnt[k].blasEntries);
      atomicAdd(&counts[k].travIters, cnt[k].travIters);
      atomicAdd(&counts[k].travLanes, cnt[k].travLanes);
      atomicAdd(&counts[k].loopIters, cnt[k].loopIters);
      atomicAdd(&counts[k].loopLanes, cnt[k].loopLanes);
      atomicAdd(&counts[k].traces, cnt[k].traces);
    }
  }
}

// Running mean of this launch's samples into the film, in sample order.
__global__ void ptFold() {
  const SdLaunch& lp = c_lp;
  int npix = lp.width * lp.height;
  int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= npix) return;
  if (lp.shardCount > 1) {  // another shard's pixel: no samples here
    int px = pix % lp.width, py = pix / lp.width;
    if (((py >> 6) * lp.shardTilesX + (px >> 6)) % lp.shardCount != lp.shardIndex) return;
  }
  float4 acc = lp.accum[pix];
  for (int i = 0; i < lp.sppThisLaunch; i++) {
    float4 x = lp.sampleL[(size_t)i * npix + pix];
    int s1 = lp.sampleOffset + i + 1;
    acc = make_float4(acc.x + (x.x - acc.x) / s1, acc.y + (x.y - acc.y) / s1,
                      acc.z + (x.z - acc.z) / s1, 1.0f);
  }
  lp.accum[pix] = acc;
  if (!lp.aovOn) return;
  float4 al = lp.aovAlbedo[pix], nm = lp.aovNormal[pix];
  for (int i = 0; i < lp.sppThisLaunch; i++) {
    size_t k = (size_t)i * npix + pix;
    float4 a = lp.sampleAlb[k], n = lp.sampleNrm[k];
    int s1 = lp.sampleOffset + i + 1;
    al = make_float4(al.x + (a.x - al.x) / s1, al.y + (a.y - al.y) / s1, al.z + (a.z - al.z) / s1, 1.0f);
    nm = make_float4(nm.x + (n.x - nm.x) / s1, nm.y + (n.y - nm.y) / s1, nm.z + (n.z - nm.z) / s1, 1.0f);
  }
  lp.aovAlbedo[pix] = al;
  lp.aovNormal[pix] = nm;
}

// ---- host-side launch wrappers ------------------------------------------------

cudaError_t setLaunch(const SdLaunch& lp, cudaStream_t st) {
  return cudaMemcpyToSymbolAsync(c_lp, &lp, sizeof(SdLaunch), 0, cudaMemcpyHostToDevice, st);
}

int bvhWidth() { return SDB_WIDE_BVH ? 8 : 2; }

// Persistent grid of a path kernel: every SM filled with resident blocks.
template <typename K>
static int persistentGrid(K kernel) {
  int dev = 0, sms = 0, perSm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, kRenderBlock, 0);
  if (perSm < 1) perSm = 1;
  return sms * perSm;
}

int renderGridSize() { return persistentGrid(ptPersistent<false, 0>); }

// grid: the plain kernel's persistent grid; the record variants size their
// own (their trail of guided vertices may change their occupancy).
cudaError_t launchRender(cudaStream_t st, int grid, int guide) {
  switch (guide) {
    case 0: ptPersistent<false, 0><<<grid, kRenderBlock, 0, st>>>(nullptr); break;
    case kGuideSample: ptPersistent<false, kGuideSample><<<grid, kRenderBlock, 0, st>>>(nullptr); break;
    case kGuideRecord: {
      static const int g = persistentGrid(ptPersistent<false, kGuideRecord>);
      ptPersistent<false, kGuideRecord><<<g, kRenderBlock, 0, st>>>(nullptr);
      break;
    }
    case kGuideSample | kGuideRecord: {
      static const int g = persistentGrid(ptPersistent<false, kGuideSample | kGuideRecord>);
      ptPersistent<false, kGuideSample | kGuideRecord><<<g, kRenderBlock, 0, st>>>(nullptr);
      break;
    }
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launchRenderCounting(cudaStream_t st, int grid, TraceCount* counts) {
  ptPersistent<true, 0><<<grid, kRenderBlock, 0, st>>>(counts);
  return cudaGetLastError();
}

cudaError_t launchFold(int npix, cudaStream_t st) {
  ptFold<<<(npix + 255) / 256, 256, 0, st>>>();
  return cudaGetLastError();
}

}  // namespace sdb
