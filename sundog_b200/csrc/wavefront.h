// Wavefront path tracer (wavefront.cu): pool buffers and the host driver.
#pragma once

#include <cuda_runtime.h>

#include <memory>

#include "render_session.h"
#include "sd_types.h"

namespace sdb {

struct Path;
struct Vertex;
struct TraceHit;
struct GuideTrail;

// A pool entry: the per-path record at a 16-byte boundary, so the stages
// move it with 128-bit loads and stores (instancing frame: 1,213 Mrays/s
// against 1,133 at the records' natural 8-byte alignment, 1,158 at 32
// bytes). The records themselves keep their natural layout, so the
// megakernel's register and local-memory frames do not grow.
template <typename T>
struct __align__(16) PoolSlot {
  T v;
};

// Device view of the slot pool (one path per slot).
struct WfPool {
  PoolSlot<Path>* paths;
  PoolSlot<Vertex>* verts;
  PoolSlot<TraceHit>* hits;
  float4* trs;             // shadow-ray transmittance of the slot's vertex
  unsigned char* pending;  // 1: the slot's second half is due this iteration
  int* lists[2];           // live slot lists, ping-pong between iterations
  int* shadowList;
  unsigned* counts;        // [0], [1]: list lengths; [2]: shadow-list length;
                           // [3]: rays the trace stage has fetched
  PoolSlot<GuideTrail>* trails;  // guided vertices awaiting their path's end (record passes)
  unsigned char* jobs;     // serving batches: the job slot of each slot's path
  int cap;
  int refillOpen;          // 0: every path of the launch fits the pool at once (no refills)
};

// Host-owned pool storage, grown on demand.
struct WfBuffers {
  // One device allocation holds every per-slot array (carved at 256-byte
  // boundaries), so a pool costs one cudaMalloc and one cudaFree.
  DevBuf slab, counts;
  void *paths = nullptr, *verts = nullptr, *hits = nullptr, *trs = nullptr, *pending = nullptr,
       *list0 = nullptr, *list1 = nullptr, *shadow = nullptr, *jobs = nullptr;
  DevBuf trails;  // allocated by the first training-record pass
  unsigned* hostCount = nullptr;   // pinned: the four list counters (from a process-wide free list)
  cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // stage timing
  int cap = 0;
  int trailCap = 0;
  int gridStart = 0, gridTrace = 0, gridShadeA = 0, gridShadow = 0, gridShadeB = 0;
  WfBuffers() = default;
  WfBuffers(const WfBuffers&) = delete;
  WfBuffers& operator=(const WfBuffers&) = delete;
  ~WfBuffers();
  void ensure(int slots);
  void ensureTrails();  // one GuideTrail per slot
};

// Device bytes per pool slot.
size_t wfSlotBytes();
// A pool for the current device: the idle one kept from an earlier session,
// or a new empty one. wfRelease keeps a finished session's pool for reuse.
std::unique_ptr<WfBuffers> wfAcquire();
void wfRelease(std::unique_ptr<WfBuffers> b);
// Frees the idle pools of every device.
void wfReleaseIdle();
// Whether finished sessions keep their device buffers for the next one
// (sundog_set_device_memory_cache; render.cpp).
bool keepDeviceMemory();
// Renders lp.numPaths camera paths (counters cleared by the caller) into
// lp.sampleL; returns the number of kernels launched. Synchronises st once per
// iteration to read the live-path count. guide: 0, or a combination of
// kGuideSample (draw directions by MIS with the learned guide of lp) and
// kGuideRecord (keep each path's guided vertices in its slot's trail and turn
// them into training records when the path ends).
// times: when non-null, per-stage event times and ray counts are added to it.
int wfRender(const SdLaunch& lp, WfBuffers& b, cudaStream_t st, int guide = 0,
             WfStageTimes* times = nullptr);

// Serving batches (serve.h): the engine's whole job table (kMaxServeJobs
// launch blocks, host memory), and one batch of tile-passes rendered through
// the pool into batch.sampleL at each path's id (the caller folds them).
// Returns the kernels launched.
// maxInstances: the largest instance count among the batch's scenes (picks
// the shadow-ray kernel, as a render does by its own scene's count).
struct ServeBatch;
cudaError_t wfSetJobs(const SdLaunch* table, cudaStream_t st);
int wfRenderBatch(const ServeBatch& batch, WfBuffers& b, cudaStream_t st, int maxInstances = 0);

// Scenes with at least this many instances trace their shadow rays with
// dynamic fetch (wfShadowFetch), smaller ones one ray per thread (wfShadow).
#ifndef SDB_SHADOW_FETCH_INSTANCES
#define SDB_SHADOW_FETCH_INSTANCES 64
#endif
constexpr int kShadowFetchInstances = SDB_SHADOW_FETCH_INSTANCES;

}  // namespace sdb
