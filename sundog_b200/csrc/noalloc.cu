// Allocation-free tile render.
//
// Some callers cannot allocate device memory at the point where they want a
// render: a worker process whose device memory is owned by another
// allocator (a framework's caching allocator or a fixed memory budget that
// any cudaMalloc outside it would break), or code running where allocating
// would synchronise the device. For them sundog_session_render_tile_noalloc
// renders a rectangle of a resident session's image into a device film the
// caller already owns, and allocates nothing: the scratch the path kernel
// needs (a per-sample radiance buffer, two counters and the launch block)
// lives in the file-scope device variables below, which every GPU that loads
// this library holds until the process exits.
//
// Limits and sharing:
//  * at most kTileSlots (1,048,576) pixel-samples per call, e.g. a 64 x 64
//    tile at 256 spp; larger requests are rejected with an error;
//  * all calls share the one scratch array (per device) and it keeps the
//    last call's contents; every call clears the counters and rewrites every
//    radiance slot it reads. Calls that overlap on the GPU (two streams, or
//    two host threads) race on the array and on the launch block: serialise
//    them;
//  * the launch block and tile description reach the device as kernel
//    arguments of a one-thread set-up kernel, which copies them into the
//    scratch; no host memory is read after the call returns;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before starting any stream capture.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <stdexcept>

#include "../../include/sundog_api.h"
#include "abi_util.h"
#include "pt_path.cuh"
#include "render_session.h"

namespace sdb {

constexpr size_t kTileSlots = size_t(1) << 20;            // float4 radiance slots
constexpr size_t kTileCounterBytes = 256;                  // path + ray counters
constexpr size_t kTileScratchBytes = kTileCounterBytes + kTileSlots * sizeof(float4);

static __device__ __align__(256) unsigned char g_tileScratch[kTileScratchBytes];

struct TileSpec {
  int x0, y0, w, h;
  int sampleBegin, sampleCount;
  float4* film;  // caller's w*h running means
};

// The call's launch block and tile, written by ptTileSetup on the call's
// stream; part of the library's static scratch.
static __device__ SdLaunch g_tileLp;
static __device__ TileSpec g_tile;

// Copies the call's launch block and tile (kernel arguments) into the
// scratch and clears the two counters.
__global__ void ptTileSetup(SdLaunch lp, TileSpec t) {
  g_tileLp = lp;
  g_tile = t;
  lp.pathCounter[0] = 0ull;
  lp.rayCounter[0] = 0ull;
}

// Full-frame path index of tile pixel (px, py), sample sLocal: the same
// 8x8-tiled numbering the full render uses, so startPath() derives the
// identical camera ray and random stream.
__device__ __forceinline__ unsigned long long fullFrameId(const SdLaunch& lp, int px, int py,
                                                          int sLocal) {
  int tile = (py >> 3) * lp.tilesX + (px >> 3);
  int rem = tile * 64 + (py & 7) * 8 + (px & 7);
  return (unsigned long long)sLocal * lp.npixPad + rem;
}

__global__ void __launch_bounds__(kRenderBlock) ptTileNoAlloc() {
  const SdLaunch& lp = g_tileLp;
  const TileSpec& t = g_tile;
  const unsigned full = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31;
  unsigned long long rays = 0;
  const int npt = t.w * t.h;
  const long long total = (long long)npt * t.sampleCount;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    int sLocal = (int)(i / npt);
    int rem = (int)(i - (long long)sLocal * npt);
    int px = t.x0 + rem % t.w, py = t.y0 + rem / t.w;
    Path p;
    if (!startPath(lp, fullFrameId(lp, px, py, sLocal), p)) continue;
    p.slot = (int)i;
    while (bounce<false>(lp, p, rays, nullptr)) {
    }
    float3 L = sanitize3(p.L);
    lp.sampleL[i] = make_float4(L.x, L.y, L.z, 1.0f);
  }
  for (int off = 16; off > 0; off >>= 1) rays += __shfl_down_sync(full, rays, off);
  if (lane == 0 && rays) atomicAdd(lp.rayCounter, rays);
}

// Running mean of the call's samples into the caller's film, in sample order.
__global__ void ptTileFold() {
  const SdLaunch& lp = g_tileLp;
  const TileSpec& t = g_tile;
  int npt = t.w * t.h;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npt) return;
  float4 acc = t.film[i];
  for (int k = 0; k < t.sampleCount; k++) {
    float4 x = lp.sampleL[(size_t)k * npt + i];
    int s1 = t.sampleBegin + k + 1;
    acc = make_float4(acc.x + (x.x - acc.x) / s1, acc.y + (x.y - acc.y) / s1,
                      acc.z + (x.z - acc.z) / s1, 1.0f);
  }
  t.film[i] = acc;
}

// Device address of the scratch array, looked up once per device.
static void* scratchAddress() {
  static std::mutex mu;
  static void* addr[64] = {nullptr};
  int dev = 0;
  cudaCheck(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= 64) throw std::runtime_error("noalloc: device index out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_tileScratch);
    if (e != cudaSuccess)
      throw std::runtime_error(std::string("noalloc: cudaGetSymbolAddress failed: ") +
                               cudaGetErrorString(e));
    addr[dev] = p;
  }
  return addr[dev];
}

}  // namespace sdb

using namespace sdb;

// Renders samples [sample_begin, sample_begin + sample_count) of the pixel
// rectangle (x0, y0, w, h) of a resident session's image and folds them, in
// sample order, into film_device: w*h float4 running means in the caller's
// device memory (row-major, row 0 = image row y0), holding the means of the
// samples before sample_begin (zeros when sample_begin is 0). Sample indices
// count from the session's first sample (its sample_offset), as in a full
// render of the session, so the result is identical to the same pixels of a
// full render of it. Sessions with learned guiding enabled are rejected: this
// entry point traces plain samples only. Allocates nothing. rays_out (host,
// may be NULL) receives the radiance + shadow traces; when it is non-NULL
// the call waits for the render to finish, otherwise the work is left queued
// on cuda_stream (NULL = legacy default stream). Returns 0, or 1 with
// sundog_last_error() set.
extern "C" int sundog_session_render_tile_noalloc(sundog_session* sh, int x0, int y0, int w, int h,
                                                  int sample_begin, int sample_count,
                                                  float* film_device, uint64_t* rays_out,
                                                  void* cuda_stream) {
  SDB_TRY
  if (!sh) throw std::runtime_error("noalloc: null session");
  if (!film_device) throw std::runtime_error("noalloc: null film");
  const RenderSession& s = *reinterpret_cast<const RenderSession*>(sh);
  if (s.guide)
    throw std::runtime_error("noalloc: the session has learned guiding enabled; this entry point "
                             "renders plain samples only (disable guiding or use "
                             "sundog_session_render)");
  if (w <= 0 || h <= 0 || x0 < 0 || y0 < 0 || x0 + w > s.lp.width || y0 + h > s.lp.height)
    throw std::runtime_error("noalloc: tile outside the image");
  if (sample_count <= 0 || sample_begin < 0) throw std::runtime_error("noalloc: bad sample range");
  if ((unsigned long long)w * h * sample_count > kTileSlots)
    throw std::runtime_error("noalloc: tile pixels x samples exceeds the 1048576-slot scratch "
                             "(for example 64x64 at 256 spp); split the call");
  if ((long long)s.sampleBase + sample_begin + sample_count > 0x7FFFFFFFll)
    throw std::runtime_error("noalloc: sample index overflows");
  cudaStream_t st = (cudaStream_t)cuda_stream;
  unsigned char* base = (unsigned char*)scratchAddress();

  const int first = s.sampleBase + sample_begin;
  SdLaunch lp = s.lp;
  lp.shardCount = 0;  // ids below use the whole-frame numbering
  lp.aovOn = 0;
  lp.sampleOffset = first;
  lp.sppThisLaunch = sample_count;
  lp.pathCounter = (unsigned long long*)base;
  lp.rayCounter = (unsigned long long*)(base + 8);
  lp.sampleL = (float4*)(base + kTileCounterBytes);
  lp.sampleAlb = nullptr;
  lp.sampleNrm = nullptr;
  lp.accum = nullptr;
  TileSpec t = {x0, y0, w, h, first, sample_count, (float4*)film_device};

  ptTileSetup<<<1, 1, 0, st>>>(lp, t);
  cudaCheck(cudaGetLastError(), "noalloc set-up launch");
  long long total = (long long)w * h * sample_count;
  int grid = (int)((total + kRenderBlock - 1) / kRenderBlock);
  ptTileNoAlloc<<<grid, kRenderBlock, 0, st>>>();
  cudaCheck(cudaGetLastError(), "noalloc render launch");
  ptTileFold<<<(w * h + 255) / 256, 256, 0, st>>>();
  cudaCheck(cudaGetLastError(), "noalloc fold launch");
  if (rays_out) {
    unsigned long long r = 0;
    cudaCheck(cudaMemcpyAsync(&r, lp.rayCounter, sizeof r, cudaMemcpyDeviceToHost, st),
              "noalloc ray count");
    cudaCheck(cudaStreamSynchronize(st), "noalloc render");
    *rays_out = r;
  }
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}
