// A scene uploaded to the device and ready to render repeatedly.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/sundog_api.h"
#include "assets.h"
#include "scene_model.h"

namespace sdb {

void cudaCheck(cudaError_t e, const char* what);
// Adds to the device-to-host byte count sundog_transfer_bytes reports.
void countDownload(size_t bytes);

// Per-stage device time of wavefront renders, accumulated while a session
// has stage timing on: CUDA events on the render stream around each stage
// launch, read at the per-iteration synchronisation the engine makes anyway.
struct WfStageTimes {
  double startMs = 0, traceMs = 0, shadeAMs = 0, shadowMs = 0, shadeBMs = 0;
  unsigned long long iterations = 0, radianceRays = 0, shadowRays = 0, launches = 0;
};


// Four pinned host words for a counter read-back, from a process-wide free
// list (a pinned allocation costs more than the render of a small frame);
// returned words are kept for the next caller, never freed.
unsigned* pinnedWords();
void returnPinnedWords(unsigned* p);

struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), bytes(o.bytes) {
    o.ptr = nullptr;
    o.bytes = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      ptr = o.ptr;
      bytes = o.bytes;
      o.ptr = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(size_t n);
  void upload(const void* src, size_t n);
  void release();
};

struct MeshBufs {
  DevBuf pos, idx, nrm, uv;
};

void quadricBoundsHost(int kind, float3& lo, float3& hi);
// Whether binary BVHs are built on the device (sundog_set_bvh_builder).
bool deviceBvhBuilds();
// The current device's launch lock (render.cpp): held from writing the
// constant-memory launch blocks until the kernels reading them are done.
std::mutex& deviceLaunchLock();

struct GuideState;  // guide.h
struct WfBuffers;   // wavefront.h

// A scene's data on the device (textures, meshes, light CDFs, environment
// CDFs, BVH, materials). Independent of resolution, spp and seed: several
// films can render from one copy.
struct DeviceScene {
  SceneDesc scene;
  SdEnv env{};
  int numLights = 0, numObjects = 0;
  bool wideNodes = false;
  size_t meshTriangles = 0, numNodes = 0, numTris = 0, deviceBytes = 0;
  int tlasDepth = 0, blasDepth = 0;
  double loadMs = 0, buildMs = 0;
  DevBuf envTex, envMarg, envCond, envGuide;  // envGuide: marginal, then each row's
  std::vector<DevBuf> texImages;
  std::vector<MeshBufs> meshBufs;
  std::vector<DevBuf> lightBufs;
  DevBuf dNodes, dTris, dInst, dMeshes, dTex, dMat, dLights, dFlames;
  DevBuf dNodes4;  // the 4-wide layout (SDB_BVH4), collapsed from dNodes
  std::vector<SdLight> lights;  // host copy of the device light list

  void build(const SceneDesc& desc);
  // The binary BVH of every mesh and the TLAS built on the device into
  // dNodes / dTris (tlasOrder: TLAS leaf order -> object).
  void buildAccelOnDevice(const std::vector<HostMesh>& meshes, std::vector<SdMesh>& meshDescs,
                          std::vector<int>& tlasOrder);
  // Copies sampling table `which` (0 env marginal CDF, 1 env conditional
  // CDFs, 2 + k the area CDF of light k; empty when the scene has none) to
  // out (cap floats); returns its length.
  size_t table(int which, float* out, size_t cap) const;
  void fillLaunch(SdLaunch& l) const;  // scene pointers and counts
};

// sundog_render's option overrides applied to a scene's render settings.
void applyRenderOverrides(SceneDesc& scene, const sundog_render_options* opt);

// Render settings and camera of one film of the given size.
void fillRenderLaunch(SdLaunch& l, const SceneDesc& scene, const RenderCfg& rs);

struct RenderSession {
  SceneDesc scene;
  SdLaunch lp{};
  bool quiet = false;
  bool aov = false;
  int chunk = 1;
  int sampleBase = 0;  // first sample index of a render
  unsigned long long shardPixels = 0;  // film pixels this session renders
  int grid = 0;
  size_t freeBefore = 0, deviceBytes = 0;
  size_t meshTriangles = 0, numNodes = 0, numTris = 0;
  int tlasDepth = 0, blasDepth = 0;
  double loadMs = 0, buildMs = 0, setupMs = 0;
  unsigned long long lastRays = 0;
  double lastRenderMs = 0, lastKernelMs = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t kev[2] = {nullptr, nullptr};  // around each path-kernel launch

  std::shared_ptr<const DeviceScene> dev;
  DevBuf accum, aovAlb, aovNrm, sampleL, sampleAlb, sampleNrm, counters;
  std::unique_ptr<GuideState> guide;  // learned path guiding, when enabled
  std::unique_ptr<WfBuffers> wf;      // wavefront slot pool, when used
  int engine = 0;                     // sundog_render_ext.engine
  bool stageTiming = false;           // sundog_session_set_stage_timing
  WfStageTimes stages;                // per-stage times of the last render

  ~RenderSession();
  void build(const sundog_scene* h, const sundog_render_options* opt, const sundog_render_ext* ext);
  void render(cudaStream_t st, bool reset, sundog_render_result* res);
  void read(float* film, float* alb, float* nrm);
  // Counting render: traversal visit counts of both ray kinds in *out, or,
  // with `shadow`, radiance rays in *out and shadow rays in *shadow.
  void countTraversal(sundog_trace_counts* out, sundog_trace_counts* shadow = nullptr);
  void setGuiding(bool enable, const sundog_guiding_config* cfg);
};

}  // namespace sdb
