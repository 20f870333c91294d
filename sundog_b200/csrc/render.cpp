// Render orchestration: sundog_probe, sundog_render (drop-in) and the
// additive session API that keeps a scene resident on the device.
//
// A session does the reference's load-time steps once (src/capi_render.cpp:
// 74-221): render overrides, OBJ / HDR / image loading, mesh-light CDFs in
// FP64 (126-172), environment CDFs in FP64 (src/env_light.cpp:27-56), BVH
// build (host SAH, replacing the OptiX GAS/IAS builds at 175-185) and the
// uploads. Each session_render then runs the sample loop on the device:
// per chunk one persistent path-tracing launch plus one film fold.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/sundog_api.h"
#include "abi_util.h"
#include "assets.h"
#include "bvh_build.h"
#include "bvh_device.h"
#include "guide.h"
#include "kernels.h"
#include "cdf_build.h"
#include "render_session.h"
#include "wavefront.h"
#include "scene_model.h"

using namespace sdb;
using Clock = std::chrono::steady_clock;

namespace sdb {

static double msSince(Clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

void cudaCheck(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

static std::mutex g_pinnedMu;
static std::vector<unsigned*> g_pinnedFree;

unsigned* pinnedWords() {
  {
    std::lock_guard<std::mutex> lock(g_pinnedMu);
    if (!g_pinnedFree.empty()) {
      unsigned* p = g_pinnedFree.back();
      g_pinnedFree.pop_back();
      return p;
    }
  }
  unsigned* p = nullptr;
  cudaCheck(cudaMallocHost((void**)&p, 4 * sizeof(unsigned)), "pinned words");
  return p;
}

void returnPinnedWords(unsigned* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lock(g_pinnedMu);
  g_pinnedFree.push_back(p);
}

void DevBuf::alloc(size_t n) {
  release();
  if (n == 0) return;
  cudaCheck(cudaMalloc(&ptr, n), "cudaMalloc");
  bytes = n;
}
std::atomic<unsigned long long> g_h2dBytes{0}, g_d2hBytes{0};
void countDownload(size_t bytes) { g_d2hBytes += bytes; }

void DevBuf::upload(const void* src, size_t n) {
  alloc(n);
  if (n) cudaCheck(cudaMemcpy(ptr, src, n, cudaMemcpyHostToDevice), "upload");
  g_h2dBytes += n;
}
void DevBuf::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

static std::string resolvePath(const SceneDesc& s, const std::string& p) {
  if (!p.empty() && p[0] != '/') return s.baseDir + "/" + p;
  return p;
}

// Inverse of a 3x4 affine map, computed in double and rounded once.
static void invertAffine(const Xform& x, float4 out[3]) {
  const float* m = x.m;
  double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
  double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
  double det = a * A + b * B + c * C;
  if (det == 0.0) throw std::runtime_error("scene: object transform is singular");
  double inv[9] = {A / det,
                   -(b * i - c * h) / det,
                   (b * f - c * e) / det,
                   B / det,
                   (a * i - c * g) / det,
                   -(a * f - c * d) / det,
                   C / det,
                   -(a * h - b * g) / det,
                   (a * e - b * d) / det};
  double t[3] = {m[3], m[7], m[11]};
  for (int r = 0; r < 3; r++) {
    double tr = -(inv[r * 3] * t[0] + inv[r * 3 + 1] * t[1] + inv[r * 3 + 2] * t[2]);
    out[r] = make_float4((float)inv[r * 3], (float)inv[r * 3 + 1], (float)inv[r * 3 + 2], (float)tr);
  }
}

static int strataFor(int spp) {  // device/programs.cu:317-319
  int n = (int)floorf(sqrtf((float)spp) + 0.5f);
  if (n * n > spp) n--;
  if (n < 1) n = 1;
  return n;
}

// Device-memory cache between calls (sundog_set_device_memory_cache): off by
// default, so a one-shot render (sundog_render, sundog_render_ex) frees all
// it allocated before it returns, as the reference's render does
// (src/capi_render.cpp:65, 303-304). On, the largest per-sample radiance
// buffer and the wavefront pool of a finished session stay allocated for the
// next one on the same device (a one-shot render then skips allocating and
// freeing about 1 GiB + the pool per call; the free alone measured 5-60 ms),
// until sundog_release_device_memory or the cache is switched off.
static std::atomic<int> g_keepMemory{0};
static std::mutex g_samplesMu;
static DevBuf g_idleSamples[64];

bool keepDeviceMemory() { return g_keepMemory.load() != 0; }

static void acquireSamples(DevBuf& b, size_t bytes) {
  int dev = 0;
  cudaCheck(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev >= 0 && dev < 64) {
    std::lock_guard<std::mutex> lock(g_samplesMu);
    if (g_idleSamples[dev].ptr && g_idleSamples[dev].bytes >= bytes) {
      b = std::move(g_idleSamples[dev]);
      return;
    }
  }
  b.alloc(bytes);
}

static void releaseSamples(DevBuf& b) {
  int dev = 0;
  if (!b.ptr || cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  if (!keepDeviceMemory()) {
    b.release();
    return;
  }
  std::lock_guard<std::mutex> lock(g_samplesMu);
  if (g_idleSamples[dev].bytes < b.bytes) g_idleSamples[dev] = std::move(b);
}

// Frees the idle buffers of every device (the current device stays current).
static void releaseIdleSamples() {
  int cur = 0;
  if (cudaGetDevice(&cur) != cudaSuccess) return;
  std::lock_guard<std::mutex> lock(g_samplesMu);
  for (int d = 0; d < 64; d++) {
    if (!g_idleSamples[d].ptr) continue;
    if (cudaSetDevice(d) == cudaSuccess) g_idleSamples[d].release();
  }
  cudaSetDevice(cur);
}

RenderSession::~RenderSession() {
  releaseSamples(sampleL);
  wfRelease(std::move(wf));
  if (stream) cudaStreamDestroy(stream);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (kev[0]) cudaEventDestroy(kev[0]);
  if (kev[1]) cudaEventDestroy(kev[1]);
}

// Scene data on the device: assets, CDFs, BVH and uploads (the reference's
// load-time steps, src/capi_render.cpp:84-221). Independent of the render
// settings, so one copy serves every render of the scene.
void DeviceScene::build(const SceneDesc& desc) {
  scene = desc;
  size_t freeB = 0, totB = 0, freeBefore = 0;
  cudaCheck(cudaMemGetInfo(&freeBefore, &totB), "cudaMemGetInfo");
  // ---- assets ----
  auto tLoad = Clock::now();
  std::vector<HostMesh> meshes;
  meshTriangles = 0;
  for (const MeshCfg& mc : scene.meshes) {
    meshes.push_back(loadObj(resolvePath(scene, mc.file), mc.smooth, mc.usemtl));
    meshTriangles += meshes.back().idx.size();
  }
  std::vector<SdTexture> texDescs;
  for (const TextureCfg& tc : scene.textures) {
    SdTexture d = tc.desc;
    if (d.kind == TX_IMAGE) {
      int w = 0, hh = 0;
      std::vector<unsigned char> px;
      std::string err;
      std::string p = resolvePath(scene, tc.file);
      if (!loadImageRgba8(p, w, hh, px, err))
        throw std::runtime_error("cannot load texture " + p + ": " + err);
      texImages.emplace_back();
      texImages.back().upload(px.data(), px.size());
      d.img = (const uchar4*)texImages.back().ptr;
      d.imgW = w;
      d.imgH = hh;
      d.srgb = tc.srgb ? 1 : 0;
    }
    texDescs.push_back(d);
  }
  env = SdEnv{};
  std::vector<float> envRgba;
  int envW = 0, envH = 0;
  if (scene.bgKind == BG_ENVMAP) {
    std::string p = resolvePath(scene, scene.env.file);
    std::string err;
    if (!loadHdr(p, envW, envH, envRgba, err))
      throw std::runtime_error("cannot load envmap '" + p + "' (" + err + ")");
  }
  loadMs = msSince(tLoad);

  // ---- CDFs + BVH (the reference's "gas_build" segment) ----
  auto tBuild = Clock::now();
  if (scene.bgKind == BG_ENVMAP) {
    // Texels up, then the CDFs built from them on the device (cdf_build.cu).
    envTex.upload(envRgba.data(), envRgba.size() * sizeof(float));
    envMarg.alloc((size_t)(envH + 1) * sizeof(float));
    envCond.alloc((size_t)envH * (envW + 1) * sizeof(float));
    bool degenerate = false;
    buildEnvCdfDevice((const float4*)envTex.ptr, envW, envH, (float*)envMarg.ptr,
                      (float*)envCond.ptr, degenerate, 0);
    if (degenerate && scene.env.importance)
      std::fprintf(stderr, "envmap: %s has zero luminance, falling back to uniform sampling\n",
                   scene.env.file.c_str());
    // Search guides: the marginal's, then each row's conditional's.
    envGuide.alloc((size_t)(envH + 1) * (kCdfGuide + 1) * sizeof(int));
    int* guide = (int*)envGuide.ptr;
    buildCdfGuideDevice((const float*)envMarg.ptr, envH + 1, 0, 1, guide, 0);
    buildCdfGuideDevice((const float*)envCond.ptr, envW + 1, (size_t)envW + 1, envH,
                        guide + (kCdfGuide + 1), 0);
    env.texels = (const float4*)envTex.ptr;
    env.margCdf = (const float*)envMarg.ptr;
    env.condCdf = (const float*)envCond.ptr;
    env.margGuide = guide;
    env.condGuide = guide + (kCdfGuide + 1);
    env.width = envW;
    env.height = envH;
    env.rotate = scene.env.rotateDeg * kPi / 180.0f;
    env.intensity = scene.env.intensity;
    env.importance = (scene.env.importance && !degenerate) ? 1 : 0;
  }

  // Mesh data on the device.
  std::vector<SdMesh> meshDescs(meshes.size());
  meshBufs.resize(meshes.size());
  for (size_t i = 0; i < meshes.size(); i++) {
    const HostMesh& m = meshes[i];
    MeshBufs& mb = meshBufs[i];
    mb.pos.upload(m.pos.data(), m.pos.size() * sizeof(float3));
    mb.idx.upload(m.idx.data(), m.idx.size() * sizeof(uint3));
    if (!m.nrm.empty()) mb.nrm.upload(m.nrm.data(), m.nrm.size() * sizeof(float3));
    if (!m.uv.empty()) mb.uv.upload(m.uv.data(), m.uv.size() * sizeof(float2));
    meshDescs[i].pos = (const float3*)mb.pos.ptr;
    meshDescs[i].idx = (const uint3*)mb.idx.ptr;
    meshDescs[i].nrm = (const float3*)mb.nrm.ptr;
    meshDescs[i].uv = (const float2*)mb.uv.ptr;
    meshDescs[i].numTris = (int)m.idx.size();
  }

  // Mesh lights: render-local copy of the light list with world geometry;
  // world vertices and area CDF built on the device (cdf_build.cu).
  lights = scene.lights;
  for (const ObjectCfg& o : scene.objects) {
    if (o.kind != GK_MESH || o.lightId < 0) continue;
    const HostMesh& m = meshes[o.mesh];
    lightBufs.emplace_back();
    lightBufs.back().alloc(m.pos.size() * sizeof(float3));
    float3* dpos = (float3*)lightBufs.back().ptr;
    lightBufs.emplace_back();
    lightBufs.back().alloc((m.idx.size() + 1) * sizeof(float));
    double total = buildMeshLightCdfDevice(meshDescs[o.mesh].pos, (int)m.pos.size(),
                                           meshDescs[o.mesh].idx, (int)m.idx.size(), o.xform, dpos,
                                           (float*)lightBufs.back().ptr, 0);
    if (!(total > 0.0))
      throw std::runtime_error("mesh NEE light has zero surface area: " + scene.meshes[o.mesh].file);
    SdLight& ld = lights[o.lightId];
    ld.mPos = dpos;
    ld.mCdf = (const float*)lightBufs.back().ptr;
    ld.mIdx = meshDescs[o.mesh].idx;
    ld.mUv = meshDescs[o.mesh].uv;
    ld.mNumTris = (int)m.idx.size();
    ld.area = (float)total;
    ld.mNgSign = orientSign(o.xform.vec(v3(1, 0, 0)), o.xform.vec(v3(0, 1, 0)),
                            o.xform.vec(v3(0, 0, 1)));
  }

  // BLAS per mesh, TLAS over objects, in one node array (TLAS first);
  // triangles stored in leaf order. The binary layout is built on the device
  // (bvh_device.cu) unless the host builder is selected
  // (sundog_set_bvh_builder); the 8-wide layout is built on the host.
  int nObj = (int)scene.objects.size();
  const bool wide = bvhWidth() == 8;
  std::vector<int> tlasOrder;
  bool builtOnDevice = false;
  if (!wide && nObj > 0 && deviceBvhBuilds()) {
    buildAccelOnDevice(meshes, meshDescs, tlasOrder);
    builtOnDevice = true;
  }
  std::vector<float4> allTris;
  std::vector<CwNode> cwNodes;
  std::vector<BvhNode> binNodes;
  if (!builtOnDevice) {
    std::vector<Box3> instBoxes(nObj);
    for (int i = 0; i < nObj; i++) {
      const ObjectCfg& o = scene.objects[i];
      Box3 b = boxEmpty();
      if (o.kind == GK_MESH) {
        for (const float3& p : meshes[o.mesh].pos) boxGrow(b, o.xform.point(p));
      } else {
        float3 lo, hi;
        quadricBoundsHost(o.kind, lo, hi);
        for (int c = 0; c < 8; c++)
          boxGrow(b, o.xform.point(v3(c & 1 ? hi.x : lo.x, c & 2 ? hi.y : lo.y, c & 4 ? hi.z : lo.z)));
      }
      // World boxes come from rounded corner transforms: pad by a few ulps.
      float3 pad = (vmax(vmax(b.hi, -b.hi), vmax(b.lo, -b.lo)) + v3(1.0f)) * 1e-6f;
      b.lo = b.lo - pad;
      b.hi = b.hi + pad;
      instBoxes[i] = b;
    }
    if (wide) {
      CwBuild tlas = buildCw(instBoxes, 1, 0, 0);
      cwNodes = tlas.nodes;
      tlasOrder = tlas.order;
      tlasDepth = tlas.maxDepth;
    } else {
      BvhBuild tlas = buildBvh(instBoxes, 1, 0, 0);
      binNodes = tlas.nodes;
      tlasOrder = tlas.order;
      tlasDepth = tlas.maxDepth;
    }
    blasDepth = 0;
    for (size_t i = 0; i < meshes.size(); i++) {
      const HostMesh& m = meshes[i];
      std::vector<Box3> tb(m.idx.size());
      for (size_t t = 0; t < m.idx.size(); t++) {
        Box3 b = boxEmpty();
        boxGrow(b, m.pos[m.idx[t].x]);
        boxGrow(b, m.pos[m.idx[t].y]);
        boxGrow(b, m.pos[m.idx[t].z]);
        tb[t] = b;
      }
      int primBase = (int)(allTris.size() / 3);
      std::vector<int> order;
      if (wide) {
        int nodeBase = (int)cwNodes.size();
        CwBuild bl = buildCw(tb, kCwLeafMax, nodeBase, primBase);
        blasDepth = std::max(blasDepth, bl.maxDepth);
        meshDescs[i].root = nodeBase;
        cwNodes.insert(cwNodes.end(), bl.nodes.begin(), bl.nodes.end());
        order = bl.order;
      } else {
        int nodeBase = (int)binNodes.size();
        BvhBuild bl = buildBvh(tb, 4, nodeBase, primBase);
        blasDepth = std::max(blasDepth, bl.maxDepth);
        meshDescs[i].root = nodeBase;
        binNodes.insert(binNodes.end(), bl.nodes.begin(), bl.nodes.end());
        order = bl.order;
      }
      for (int k : order) {
        const uint3& t = m.idx[k];
        float3 a = m.pos[t.x], b = m.pos[t.y], c = m.pos[t.z];
        int ki = k;
        float kf;
        std::memcpy(&kf, &ki, sizeof kf);
        allTris.push_back(make_float4(a.x, a.y, a.z, kf));
        allTris.push_back(make_float4(b.x, b.y, b.z, 0.0f));
        allTris.push_back(make_float4(c.x, c.y, c.z, 0.0f));
      }
    }
  }
  // A traversal keeps at most one stack entry per tree level (plus its
  // BLAS-entry entries), so trees this deep could fill the stack; reject them
  // rather than let a ray skip part of the scene.
  if (SDB_BVH4 && !wide) {
    // Three entries per 4-wide level (two binary levels) plus the marker.
    const int need = 3 * ((tlasDepth + 2) / 2 + (blasDepth + 2) / 2) + 1;
    if (need > kTraversal4Stack)
      throw std::runtime_error("scene: BVH too deep for the 4-wide traversal stack (TLAS depth " +
                               std::to_string(tlasDepth) + ", BLAS depth " +
                               std::to_string(blasDepth) + ")");
  }
  const int depthRoom = wide ? kCwTraversalStack - 4 : kTraversalStack - 2;
  if (!(SDB_BVH4 && !wide) && tlasDepth + blasDepth > depthRoom)
    throw std::runtime_error("scene: BVH too deep for the traversal stack (TLAS depth " +
                             std::to_string(tlasDepth) + " + BLAS depth " +
                             std::to_string(blasDepth) + " > " + std::to_string(depthRoom) + ")");
  // Instances in TLAS leaf order (leaf primitive index = position here).
  std::vector<SdInstance> inst(nObj);
  for (int k = 0; k < nObj; k++) {
    const ObjectCfg& o = scene.objects[tlasOrder[k]];
    SdInstance& in = inst[k];
    std::memset(&in, 0, sizeof in);
    invertAffine(o.xform, in.w2o);
    in.kind = o.kind;
    in.mesh = o.mesh;
    in.mats = (uint32_t)o.matFront | ((uint32_t)o.matBack << 16);
    in.lightId = o.lightId;
    in.cutoutTex = o.cutoutTex;
    bool masked = o.matFront == kMatNone || o.matBack == kMatNone || o.cutoutTex >= 0;
    bool trans = matTransmissive(scene, o.matFront) || matTransmissive(scene, o.matBack);
    in.flags = (masked ? kInstMasked : 0) | (trans ? kInstTransmissive : 0);
  }
  if (!builtOnDevice) {
    numNodes = wide ? cwNodes.size() : binNodes.size();
    numTris = allTris.size() / 3;
    if (wide)
      dNodes.upload(cwNodes.data(), cwNodes.size() * sizeof(CwNode));
    else
      dNodes.upload(binNodes.data(), binNodes.size() * sizeof(BvhNode));
    dTris.upload(allTris.data(), allTris.size() * sizeof(float4));
  }
  if (SDB_BVH4 && !wide && numNodes > 0) {
    // The 4-wide layout, collapsed on the device from the binary nodes; the
    // TLAS root stays node 0 and each BLAS root moves to its 4-wide node.
    std::vector<int> roots(1 + meshDescs.size()), roots4(roots.size());
    roots[0] = 0;
    for (size_t i = 0; i < meshDescs.size(); i++) roots[1 + i] = meshDescs[i].root;
    dNodes4.alloc(numNodes * sizeof(Bvh4Node));
    collapseBvh4Device((const BvhNode*)dNodes.ptr, (int)numNodes, roots.data(), (int)roots.size(),
                       (Bvh4Node*)dNodes4.ptr, roots4.data(), 0);
    for (size_t i = 0; i < meshDescs.size(); i++) meshDescs[i].root = roots4[1 + i];
  }
  dInst.upload(inst.data(), inst.size() * sizeof(SdInstance));
  dMeshes.upload(meshDescs.data(), meshDescs.size() * sizeof(SdMesh));
  dTex.upload(texDescs.data(), texDescs.size() * sizeof(SdTexture));
  dMat.upload(scene.materials.data(), scene.materials.size() * sizeof(SdMaterial));
  dLights.upload(lights.data(), lights.size() * sizeof(SdLight));
  dFlames.upload(scene.flames.data(), scene.flames.size() * sizeof(SdFlame));
  buildMs = msSince(tBuild);
  numLights = (int)lights.size();
  numObjects = nObj;
  wideNodes = wide;
  cudaCheck(cudaDeviceSynchronize(), "scene upload");
  cudaCheck(cudaMemGetInfo(&freeB, &totB), "cudaMemGetInfo");
  deviceBytes = freeBefore > freeB ? freeBefore - freeB : 0;
}

// One lock per device over the launch blocks kept in constant memory (the
// render and server kernels read their scene, film and job tables from
// there): whoever writes them holds the lock until the kernels that read
// them have finished, so sessions and servers in different host threads can
// share a device.
static std::mutex g_launchLocks[64];
std::mutex& deviceLaunchLock() {
  int dev = 0;
  cudaCheck(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= 64) throw std::runtime_error("device index out of range");
  return g_launchLocks[dev];
}

// Which builder makes the binary BVH (sundog_set_bvh_builder): 1 = on the
// device (default), 0 = the host binned-SAH builder.
static std::atomic<int> g_deviceBvh{1};
bool deviceBvhBuilds() { return g_deviceBvh.load() != 0; }

namespace {
// One node whose first child is a leaf holding all n primitives and whose
// second is an empty box far away (never entered): the root of a tree too
// small to split, as the host builder makes it.
BvhNode singleLeafRoot(const Box3& b, int link) {
  BvhNode nd;
  nd.xy0 = make_float4(b.lo.x, b.hi.x, b.lo.y, b.hi.y);
  nd.xy1 = make_float4(3e30f, 3e30f, 3e30f, 3e30f);
  nd.zz = make_float4(b.lo.z, b.hi.z, 3e30f, 3e30f);
  nd.link = make_int4(link, link, 0, 0);
  return nd;
}
}  // namespace

void DeviceScene::buildAccelOnDevice(const std::vector<HostMesh>& meshes,
                                     std::vector<SdMesh>& meshDescs,
                                     std::vector<int>& tlasOrder) {
  const int nObj = (int)scene.objects.size();
  cudaStream_t st = 0;
  // Node capacity: at most n - 1 inner nodes per tree of n > 1 primitives.
  size_t cap = (size_t)std::max(nObj - 1, 1);
  size_t totalTris = 0;
  for (const HostMesh& m : meshes) {
    cap += (size_t)std::max((int)m.idx.size() - 1, 1);
    totalTris += m.idx.size();
  }
  dNodes.alloc(cap * sizeof(BvhNode));
  dTris.alloc(std::max<size_t>(totalTris, 1) * 3 * sizeof(float4));
  BvhNode* nodes = (BvhNode*)dNodes.ptr;
  float4* tris = (float4*)dTris.ptr;

  // TLAS over the instances' world boxes.
  std::vector<DevInstanceSrc> src(nObj);
  for (int i = 0; i < nObj; i++) {
    const ObjectCfg& o = scene.objects[i];
    DevInstanceSrc& d = src[i];
    std::memset(&d, 0, sizeof d);
    std::memcpy(d.xf, o.xform.m, sizeof d.xf);
    if (o.kind == GK_MESH) {
      d.pos = meshDescs[o.mesh].pos;
      d.numVerts = (int)meshes[o.mesh].pos.size();
    } else {
      quadricBoundsHost(o.kind, d.qlo, d.qhi);
    }
  }
  DevBuf dSrc, boxLo, boxHi, cent, order;
  dSrc.upload(src.data(), src.size() * sizeof(DevInstanceSrc));
  size_t maxPrims = std::max<size_t>((size_t)nObj, 1);
  for (const HostMesh& m : meshes) maxPrims = std::max(maxPrims, m.idx.size());
  boxLo.alloc(maxPrims * sizeof(float4));
  boxHi.alloc(maxPrims * sizeof(float4));
  cent.alloc(maxPrims * sizeof(float4));
  order.alloc(maxPrims * sizeof(int));
  instanceBoxesDevice((const DevInstanceSrc*)dSrc.ptr, nObj, (float4*)boxLo.ptr,
                      (float4*)boxHi.ptr, (float4*)cent.ptr, st);
  int cursor = 0;
  tlasOrder.assign(nObj, 0);
  if (nObj > 1) {
    DevBvhStats t = buildBvhDevice((const float4*)boxLo.ptr, (const float4*)boxHi.ptr,
                                   (const float4*)cent.ptr, nObj, 1, 0, 0, nodes, nObj - 1,
                                   (int*)order.ptr, st);
    cudaCheck(cudaMemcpy(tlasOrder.data(), order.ptr, nObj * sizeof(int), cudaMemcpyDeviceToHost),
              "TLAS order");
    tlasDepth = t.maxDepth;
    cursor = t.nodes;
  } else {
    float4 l, h;
    cudaCheck(cudaMemcpy(&l, boxLo.ptr, sizeof l, cudaMemcpyDeviceToHost), "instance box");
    cudaCheck(cudaMemcpy(&h, boxHi.ptr, sizeof h, cudaMemcpyDeviceToHost), "instance box");
    BvhNode root = singleLeafRoot({v3(l.x, l.y, l.z), v3(h.x, h.y, h.z)}, ~0);
    cudaCheck(cudaMemcpy(nodes, &root, sizeof root, cudaMemcpyHostToDevice), "TLAS root");
    tlasDepth = 0;
    cursor = 1;
  }

  // One BLAS per mesh (leaves of up to 4 triangles), triangles gathered into
  // leaf order after each build.
  blasDepth = 0;
  int triCursor = 0;
  for (size_t i = 0; i < meshes.size(); i++) {
    const HostMesh& m = meshes[i];
    const int nt = (int)m.idx.size();
    meshDescs[i].root = cursor;
    if (nt > 4) {
      meshBoxesDevice(meshDescs[i].pos, meshDescs[i].idx, nt, (float4*)boxLo.ptr,
                      (float4*)boxHi.ptr, (float4*)cent.ptr, st);
      DevBvhStats b = buildBvhDevice((const float4*)boxLo.ptr, (const float4*)boxHi.ptr,
                                     (const float4*)cent.ptr, nt, 4, cursor, triCursor,
                                     nodes + cursor, nt - 1, (int*)order.ptr, st);
      blasDepth = std::max(blasDepth, b.maxDepth);
      gatherTrisDevice(meshDescs[i].pos, meshDescs[i].idx, (const int*)order.ptr, nt,
                       tris + 3 * (size_t)triCursor, st);
      cursor += b.nodes;
    } else {
      // Too small to split: one leaf under a single root node.
      Box3 b = boxEmpty();
      std::vector<int> ident(std::max(nt, 1));
      for (int t = 0; t < nt; t++) {
        ident[t] = t;
        boxGrow(b, m.pos[m.idx[t].x]);
        boxGrow(b, m.pos[m.idx[t].y]);
        boxGrow(b, m.pos[m.idx[t].z]);
      }
      int link = nt > 0 ? ~((triCursor << 3) | (nt - 1)) : ~0;
      BvhNode root = nt > 0 ? singleLeafRoot(b, link)
                            : singleLeafRoot({v3(3e30f), v3(3e30f)}, ~0);
      cudaCheck(cudaMemcpy(nodes + cursor, &root, sizeof root, cudaMemcpyHostToDevice), "BLAS root");
      if (nt > 0) {
        cudaCheck(cudaMemcpy(order.ptr, ident.data(), nt * sizeof(int), cudaMemcpyHostToDevice),
                  "BLAS order");
        gatherTrisDevice(meshDescs[i].pos, meshDescs[i].idx, (const int*)order.ptr, nt,
                         tris + 3 * (size_t)triCursor, st);
      }
      cursor += 1;
    }
    triCursor += nt;
  }
  cudaCheck(cudaStreamSynchronize(st), "device BVH build");
  numNodes = (size_t)cursor;
  numTris = (size_t)triCursor;
}

size_t DeviceScene::table(int which, float* out, size_t cap) const {
  const float* src = nullptr;
  size_t n = 0;
  if (which == 0 && env.margCdf) {
    src = env.margCdf;
    n = (size_t)env.height + 1;
  } else if (which == 1 && env.condCdf) {
    src = env.condCdf;
    n = (size_t)env.height * (env.width + 1);
  } else if (which >= 2 && which - 2 < (int)lights.size() && lights[which - 2].mCdf) {
    src = lights[which - 2].mCdf;
    n = (size_t)lights[which - 2].mNumTris + 1;
  } else if (which < 0) {
    throw std::runtime_error("table: bad index");
  }
  if (out && src) cudaCheck(cudaMemcpy(out, src, std::min(n, cap) * sizeof(float),
                                       cudaMemcpyDeviceToHost), "table download");
  return n;
}

void DeviceScene::fillLaunch(SdLaunch& l) const {
  l.bgKind = scene.bgKind;
  l.bgA = scene.bgA;
  l.bgB = scene.bgB;
  l.env = env;
  l.textures = (const SdTexture*)dTex.ptr;
  l.materials = (const SdMaterial*)dMat.ptr;
  l.lights = (const SdLight*)dLights.ptr;
  l.numLights = numLights;
  l.flames = (const SdFlame*)dFlames.ptr;
  l.numFlames = (int)scene.flames.size();
  l.nodes = wideNodes ? nullptr : (const BvhNode*)dNodes.ptr;
  l.nodes4 = (const Bvh4Node*)dNodes4.ptr;
  l.cw = wideNodes ? (const CwNode*)dNodes.ptr : nullptr;
  l.tris = (const float4*)dTris.ptr;
  l.inst = (const SdInstance*)dInst.ptr;
  l.meshes = (const SdMesh*)dMeshes.ptr;
  l.tlasRoot = 0;
  l.numInstances = numObjects;
}

// Paths per sample of a launch: the padded film, or the owned tiles of a
// tile shard.
static int pathsPerSample(const SdLaunch& l) { return l.shardCount > 1 ? l.shardPad : l.npixPad; }

// Render settings and camera of one film (rs: settings after overrides).
void fillRenderLaunch(SdLaunch& l, const SceneDesc& scene, const RenderCfg& rs) {
  l.width = rs.width;
  l.height = rs.height;
  l.sppTotal = rs.spp;
  l.maxDepth = rs.maxDepth;
  l.nStrata = strataFor(rs.spp);
  l.clampVal = rs.clampVal;
  l.seed = rs.seed;
  l.transparentShadows = rs.transparentShadows ? 1 : 0;
  l.tilesX = (rs.width + 7) / 8;
  l.npixPad = l.tilesX * ((rs.height + 7) / 8) * 64;
  l.cam = buildCamera(scene.camera, rs.width, rs.height);
}


// Option overrides of sundog_render (src/capi_render.cpp:74-83).
void applyRenderOverrides(SceneDesc& scene, const sundog_render_options* opt) {
  RenderCfg& rs = scene.render;
  if (opt) {
    if (opt->spp > 0) rs.spp = opt->spp;
    if (opt->width > 0) rs.width = opt->width;
    if (opt->height > 0) rs.height = opt->height;
    if (opt->seed >= 0) rs.seed = (unsigned)opt->seed;
    if (opt->denoise >= 0) rs.denoise = opt->denoise == 1;
    if (opt->transparent_shadows >= 0) rs.transparentShadows = opt->transparent_shadows == 1;
    if (!std::isnan(opt->clamp) && opt->clamp >= 0.0) rs.clampVal = (float)opt->clamp;
    float pt = std::isnan(opt->physics_time) ? -1.0f : (float)opt->physics_time;
    if (pt >= 0.0f && !scene.physics.enabled)
      throw std::runtime_error("--physics-time: scene has no physics block");
  }
  if (rs.width <= 0 || rs.height <= 0 || rs.spp <= 0) throw std::runtime_error("render: bad size");
}

void RenderSession::build(const sundog_scene* h, const sundog_render_options* opt,
                          const sundog_render_ext* ext) {
  auto tTotal = Clock::now();
  scene = h->scene;
  quiet = opt && opt->quiet != 0;
  // ---- overrides (src/capi_render.cpp:74-83) ----
  RenderCfg& rs = scene.render;
  applyRenderOverrides(scene, opt);
  if (scene.physics.enabled && !quiet)
    std::fprintf(stderr,
                 "sundog: physics settling is not part of this renderer; rendering authored "
                 "poses\n");
  // AOVs when asked for, and as the denoiser's guides when it runs.
  aov = (opt && (opt->aov_albedo_path || opt->aov_normal_path)) ||
        (ext && (ext->aov_albedo || ext->aov_normal)) || rs.denoise;
  int devId = 0;
  cudaCheck(cudaGetDevice(&devId), "cudaGetDevice");
  cudaCheck(cudaFree(nullptr), "CUDA context");
  size_t freeB = 0, totB = 0;
  cudaCheck(cudaMemGetInfo(&freeB, &totB), "cudaMemGetInfo");
  freeBefore = freeB;
  cudaCheck(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
  cudaCheck(cudaEventCreate(&ev0), "event");
  cudaCheck(cudaEventCreate(&ev1), "event");
  cudaCheck(cudaEventCreate(&kev[0]), "event");
  cudaCheck(cudaEventCreate(&kev[1]), "event");

  // ---- scene data (assets, CDFs, BVH, uploads) ----
  {
    std::shared_ptr<DeviceScene> ds(new DeviceScene());
    ds->build(scene);
    dev = ds;
  }
  loadMs = dev->loadMs;
  buildMs = dev->buildMs;
  meshTriangles = dev->meshTriangles;
  numNodes = dev->numNodes;
  numTris = dev->numTris;
  tlasDepth = dev->tlasDepth;
  blasDepth = dev->blasDepth;

  // ---- film and per-sample buffers ----
  size_t npix = (size_t)rs.width * rs.height;
  accum.alloc(npix * sizeof(float4));
  if (aov) {
    aovAlb.alloc(npix * sizeof(float4));
    aovNrm.alloc(npix * sizeof(float4));
  }
  chunk = ext && ext->chunk_spp > 0 ? ext->chunk_spp : 0;
  if (chunk <= 0) {
    // Keep the per-sample buffers near 1 GiB.
    size_t perSample = npix * sizeof(float4) * (aov ? 3 : 1);
    size_t cap = (size_t)1 << 30;
    chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)rs.spp, cap / perSample));
  }
  chunk = std::min(chunk, rs.spp);
  sampleBase = ext && ext->sample_offset > 0 ? ext->sample_offset : 0;
  acquireSamples(sampleL, npix * chunk * sizeof(float4));
  if (aov) {
    sampleAlb.alloc(npix * chunk * sizeof(float4));
    sampleNrm.alloc(npix * chunk * sizeof(float4));
  }
  counters.alloc(2 * sizeof(unsigned long long));

  SdLaunch& l = lp;
  std::memset(&l, 0, sizeof l);
  fillRenderLaunch(l, scene, rs);
  if (ext && ext->frame_spp > 0) l.nStrata = strataFor(ext->frame_spp);
  shardPixels = npix;
  if (ext && ext->shard_count > 1) {
    const int n = ext->shard_count, r = ext->shard_index;
    if (r < 0 || r >= n) throw std::runtime_error("render: shard_index must be in [0, shard_count)");
    l.shardCount = n;
    l.shardIndex = r;
    l.shardTilesX = (rs.width + 63) / 64;
    const int tiles = l.shardTilesX * ((rs.height + 63) / 64);
    const int owned = r < tiles ? (tiles - r + n - 1) / n : 0;
    l.shardPad = owned * 4096;
    shardPixels = 0;
    for (int t = r; t < tiles; t += n) {
      int x0 = (t % l.shardTilesX) * 64, y0 = (t / l.shardTilesX) * 64;
      shardPixels += (unsigned long long)std::min(64, rs.width - x0) * std::min(64, rs.height - y0);
    }
  }
  engine = ext ? ext->engine : 0;
  if (engine < 0 || engine > 2) throw std::runtime_error("render: engine must be 0, 1 or 2");
  dev->fillLaunch(l);
  l.aovOn = aov ? 1 : 0;
  l.pathCounter = (unsigned long long*)counters.ptr;
  l.rayCounter = (unsigned long long*)counters.ptr + 1;
  l.sampleL = (float4*)sampleL.ptr;
  l.sampleAlb = (float4*)sampleAlb.ptr;
  l.sampleNrm = (float4*)sampleNrm.ptr;
  l.accum = (float4*)accum.ptr;
  l.aovAlbedo = (float4*)aovAlb.ptr;
  l.aovNormal = (float4*)aovNrm.ptr;
  grid = renderGridSize();
  if (ext && ext->guiding) setGuiding(true, nullptr);
  cudaCheck(cudaMemGetInfo(&freeB, &totB), "cudaMemGetInfo");
  deviceBytes = freeBefore > freeB ? freeBefore - freeB : 0;
  setupMs = msSince(tTotal);
}

// Wavefront pool size (slots, 285 B each; WfBuffers::ensure also caps it at
// half the free device memory): up to 64 M, so a 32-spp chunk of a 1080p
// frame (66 M paths) is almost all in flight at once and runs in about as
// many iterations as its longest path has bounces. Measured on the instancing
// frame: 894 / 981 / 1,049 / 1,092 / 1,115 Mrays/s at 4 / 8 / 16 / 32 / 64 M
// slots (fewer iterations: fewer host round trips and stage-launch tails).
#ifndef SDB_WF_SLOTS_LOG2
#define SDB_WF_SLOTS_LOG2 26
#endif
static constexpr unsigned long long kWavefrontSlots = 1ull << SDB_WF_SLOTS_LOG2;

void RenderSession::setGuiding(bool enable, const sundog_guiding_config* cfg) {
  if (!enable) {
    guide.reset();
    return;
  }
  std::unique_ptr<GuideState> g(new GuideState());
  g->configure(cfg ? *cfg : guideDefaults());
  guide = std::move(g);
}

void RenderSession::render(cudaStream_t st, bool reset, sundog_render_result* res) {
  if (!st) st = stream;
  size_t npix = (size_t)lp.width * lp.height;
  if (guide && reset) guide->reset();
  if (reset) {
    cudaCheck(cudaMemsetAsync(accum.ptr, 0, accum.bytes, st), "film reset");
    if (aov) {
      cudaCheck(cudaMemsetAsync(aovAlb.ptr, 0, aovAlb.bytes, st), "film reset");
      cudaCheck(cudaMemsetAsync(aovNrm.ptr, 0, aovNrm.bytes, st), "film reset");
    }
  }
  cudaCheck(cudaMemsetAsync(lp.rayCounter, 0, sizeof(unsigned long long), st), "counter reset");
  cudaCheck(cudaStreamSynchronize(st), "sync");
  stages = WfStageTimes();
  auto t0 = Clock::now();
  cudaCheck(cudaEventRecord(ev0, st), "event");
  uint64_t launches = 0;
  int done = 0;
  float kms = 0.0f;
  while (done < lp.sppTotal) {
    int n = std::min(chunk, lp.sppTotal - done);
    int mode = guide ? guide->kernelMode() : 0;
    if (mode & kGuideRecord) {
      n = std::min(n, std::min(guide->cfg.pass_spp, guide->cfg.train_spp - guide->trainedSpp));
      guide->beginPass(lp, st);
    }
    lp.sampleOffset = sampleBase + done;
    lp.sppThisLaunch = n;
    lp.numPaths = (unsigned long long)pathsPerSample(lp) * n;
    cudaCheck(cudaMemsetAsync(lp.pathCounter, 0, sizeof(unsigned long long), st), "counter reset");
    {
      // The launch blocks live in per-device constant memory: hold the
      // device's launch lock from writing them until the chunk's last kernel
      // that reads them (the fold) has finished.
      std::lock_guard<std::mutex> launchLock(deviceLaunchLock());
      cudaCheck(setLaunch(lp, st), "launch params");
      cudaCheck(cudaEventRecord(kev[0], st), "event");
      const bool wavefront = engine != 1;
      if (lp.numPaths == 0) {
        // A tile shard that owns no tile: nothing to trace.
      } else if (wavefront) {
        if (!wf) wf = wfAcquire();
        wf->ensure((int)std::min<unsigned long long>(lp.numPaths, kWavefrontSlots));
        launches += wfRender(lp, *wf, st, mode, stageTiming ? &stages : nullptr);
      } else {
        cudaCheck(launchRender(st, grid, mode), "path kernel launch");
        launches += 1;
      }
      cudaCheck(cudaEventRecord(kev[1], st), "event");
      cudaCheck(cudaEventSynchronize(kev[1]), "path kernel");
      float one = 0.0f;
      cudaCheck(cudaEventElapsedTime(&one, kev[0], kev[1]), "event time");
      kms += one;
      cudaCheck(launchFold((int)npix, st), "fold launch");
      cudaCheck(cudaStreamSynchronize(st), "fold");
    }
    launches += 1;
    done += n;
    if (mode & kGuideRecord) {
      guide->trainAndBake(lp, st, n);
      launches += 2 + 2 * guide->cfg.steps_per_pass;
    }
  }
  cudaCheck(cudaEventRecord(ev1, st), "event");
  cudaCheck(cudaStreamSynchronize(st), "path kernels");
  double wall = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
  float evMs = 0.0f;
  cudaCheck(cudaEventElapsedTime(&evMs, ev0, ev1), "event time");
  unsigned long long rays = 0;
  cudaCheck(cudaMemcpy(&rays, lp.rayCounter, sizeof rays, cudaMemcpyDeviceToHost), "ray count");
  lastRays = rays;
  lastRenderMs = wall;
  lastKernelMs = evMs;
  if (res) {
    res->rays_traced = rays;
    res->paths = (uint64_t)shardPixels * lp.sppTotal;
    res->render_ms = wall;
    res->build_ms = buildMs;
    res->load_ms = loadMs;
    res->mrays_per_sec = wall > 0 ? rays / wall / 1000.0 : 0.0;
    res->samples_per_sec = wall > 0 ? (double)shardPixels * lp.sppTotal / (wall / 1000.0) : 0.0;
    res->kernel_launches = launches;
    res->kernel_ms = kms;
  }
}

void RenderSession::countTraversal(sundog_trace_counts* out, sundog_trace_counts* shadow) {
  DevBuf dc;
  dc.alloc(2 * sizeof(TraceCount));
  cudaCheck(cudaMemset(dc.ptr, 0, dc.bytes), "counter reset");
  cudaCheck(cudaMemsetAsync(accum.ptr, 0, accum.bytes, stream), "film reset");
  cudaCheck(cudaMemsetAsync(lp.rayCounter, 0, sizeof(unsigned long long), stream), "counter reset");
  int done = 0;
  size_t npix = (size_t)lp.width * lp.height;
  while (done < lp.sppTotal) {
    int n = std::min(chunk, lp.sppTotal - done);
    lp.sampleOffset = sampleBase + done;
    lp.sppThisLaunch = n;
    lp.numPaths = (unsigned long long)pathsPerSample(lp) * n;
    cudaCheck(cudaMemsetAsync(lp.pathCounter, 0, sizeof(unsigned long long), stream), "counter reset");
    std::lock_guard<std::mutex> launchLock(deviceLaunchLock());
    cudaCheck(setLaunch(lp, stream), "launch params");
    cudaCheck(launchRenderCounting(stream, grid, (TraceCount*)dc.ptr), "counting launch");
    cudaCheck(launchFold((int)npix, stream), "fold launch");
    cudaCheck(cudaStreamSynchronize(stream), "counting chunk");
    done += n;
  }
  cudaCheck(cudaStreamSynchronize(stream), "counting render");
  TraceCount c[2];
  unsigned long long rays = 0;
  cudaCheck(cudaMemcpy(c, dc.ptr, sizeof c, cudaMemcpyDeviceToHost), "counts");
  cudaCheck(cudaMemcpy(&rays, lp.rayCounter, sizeof rays, cudaMemcpyDeviceToHost), "ray count");
  auto put = [](sundog_trace_counts* o, const TraceCount& a, const TraceCount* b,
                unsigned long long r) {
    o->rays = r;
    o->box_tests = a.boxTests + (b ? b->boxTests : 0);
    o->tri_tests = a.triTests + (b ? b->triTests : 0);
    o->quadric_tests = a.quadTests + (b ? b->quadTests : 0);
    o->blas_entries = a.blasEntries + (b ? b->blasEntries : 0);
    o->trav_iters = a.travIters + (b ? b->travIters : 0);
    o->trav_lanes = a.travLanes + (b ? b->travLanes : 0);
    o->loop_iters = a.loopIters;
    o->loop_lanes = a.loopLanes;
  };
  if (!shadow) {
    put(out, c[0], &c[1], rays);  // both ray kinds together
  } else {
    put(out, c[0], nullptr, c[0].traces);
    put(shadow, c[1], nullptr, c[1].traces);
    shadow->loop_iters = shadow->loop_lanes = 0;
  }
}

void RenderSession::read(float* film, float* alb, float* nrm) {
  size_t n = (size_t)lp.width * lp.height * sizeof(float4);
  if (film) cudaCheck(cudaMemcpy(film, accum.ptr, n, cudaMemcpyDeviceToHost), "film download");
  g_d2hBytes += (film ? n : 0) + (alb ? n : 0) + (nrm ? n : 0);
  if (alb) {
    if (!aov) throw std::runtime_error("session: AOVs were not requested");
    cudaCheck(cudaMemcpy(alb, aovAlb.ptr, n, cudaMemcpyDeviceToHost), "aov download");
  }
  if (nrm) {
    if (!aov) throw std::runtime_error("session: AOVs were not requested");
    cudaCheck(cudaMemcpy(nrm, aovNrm.ptr, n, cudaMemcpyDeviceToHost), "aov download");
  }
}

void quadricBoundsHost(int kind, float3& lo, float3& hi) {
  const float e = 1e-4f;
  if (kind == GK_RECT || kind == GK_DISK) {
    lo = v3(-1.0f, -e, -1.0f);
    hi = v3(1.0f, e, 1.0f);
  } else if (kind == GK_PARABOLA) {
    lo = v3(-1.0f, -e, -1.0f);
    hi = v3(1.0f, 0.5f + e, 1.0f);
  } else {
    lo = v3(-1.0f);
    hi = v3(1.0f);
  }
}

}  // namespace sdb

// ---- ABI ---------------------------------------------------------------------

// src/capi_render.cpp:55-77 — device identity; no OptiX in this build.
extern "C" int sundog_probe(sundog_device_info* out) {
  SDB_TRY
  if (!out) throw std::runtime_error("probe: null output");
  int dev = 0;
  cudaCheck(cudaGetDevice(&dev), "cudaGetDevice");
  cudaDeviceProp p;
  cudaCheck(cudaGetDeviceProperties(&p, dev), "cudaGetDeviceProperties");
  std::memset(out, 0, sizeof *out);
  std::snprintf(out->name, sizeof(out->name), "%s", p.name);
  out->cc_major = p.major;
  out->cc_minor = p.minor;
  int dv = 0, rv = 0;
  cudaDriverGetVersion(&dv);
  cudaRuntimeGetVersion(&rv);
  out->driver_version = dv;
  out->runtime_version = rv;
  out->total_mem_mb = (uint64_t)(p.totalGlobalMem >> 20);
  out->optix_header_version = 0;
  out->rtcore_version = 0;
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" sundog_session* sundog_session_create(sundog_scene* h, const sundog_render_options* opt,
                                                 const sundog_render_ext* ext) {
  SDB_TRY
  if (!h) throw std::runtime_error("render: null scene");
  if (sundog_scene_validate(h) != SUNDOG_OK) throw std::runtime_error(sundog_last_error());
  std::unique_ptr<RenderSession> s(new RenderSession());
  s->build(h, opt, ext);
  return reinterpret_cast<sundog_session*>(s.release());
  SDB_CATCH(nullptr)
}

extern "C" int sundog_session_render(sundog_session* sh, void* stream, int reset,
                                     sundog_render_result* res) {
  SDB_TRY
  if (!sh) throw std::runtime_error("session: null handle");
  reinterpret_cast<RenderSession*>(sh)->render((cudaStream_t)stream, reset != 0, res);
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_session_read(sundog_session* sh, float* film, float* alb, float* nrm) {
  SDB_TRY
  if (!sh) throw std::runtime_error("session: null handle");
  reinterpret_cast<RenderSession*>(sh)->read(film, alb, nrm);
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_session_copy_film(sundog_session* sh, void* film_device, void* stream) {
  SDB_TRY
  if (!sh || !film_device) throw std::runtime_error("session: null argument");
  RenderSession* s = reinterpret_cast<RenderSession*>(sh);
  cudaCheck(cudaMemcpyAsync(film_device, s->accum.ptr, s->accum.bytes, cudaMemcpyDeviceToDevice,
                            (cudaStream_t)stream),
            "film copy");
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_session_info(sundog_session* sh, sundog_session_stats* st) {
  SDB_TRY
  if (!sh || !st) throw std::runtime_error("session: null argument");
  const RenderSession* s = reinterpret_cast<RenderSession*>(sh);
  st->width = s->lp.width;
  st->height = s->lp.height;
  st->spp = s->lp.sppTotal;
  st->chunk_spp = s->chunk;
  st->grid = s->grid;
  st->block = kRenderBlock;
  st->device_bytes = s->deviceBytes;
  st->bvh_nodes = s->numNodes;
  st->triangles = s->numTris;
  st->instances = (uint64_t)s->lp.numInstances;
  st->tlas_depth = s->tlasDepth;
  st->blas_depth = s->blasDepth;
  st->load_ms = s->loadMs;
  st->build_ms = s->buildMs;
  st->setup_ms = s->setupMs;
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_session_trace_counts(sundog_session* sh, sundog_trace_counts* out) {
  SDB_TRY
  if (!sh || !out) throw std::runtime_error("session: null argument");
  reinterpret_cast<RenderSession*>(sh)->countTraversal(out);
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_set_bvh_builder(int device) {
  SDB_TRY
  g_deviceBvh.store(device ? 1 : 0);
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_set_device_memory_cache(int keep) {
  SDB_TRY
  g_keepMemory.store(keep ? 1 : 0);
  if (!keep) {
    releaseIdleSamples();
    wfReleaseIdle();
  }
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_release_device_memory(void) {
  SDB_TRY
  releaseIdleSamples();
  wfReleaseIdle();
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_session_table(sundog_session* sh, int which, float* out, size_t cap,
                                    size_t* count) {
  SDB_TRY
  if (!sh) throw std::runtime_error("table: null session");
  size_t n = reinterpret_cast<RenderSession*>(sh)->dev->table(which, out, cap);
  if (count) *count = n;
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_session_set_stage_timing(sundog_session* sh, int enable) {
  SDB_TRY
  if (!sh) throw std::runtime_error("stage timing: null session");
  reinterpret_cast<RenderSession*>(sh)->stageTiming = enable != 0;
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_session_stage_times(sundog_session* sh, sundog_stage_times* out) {
  SDB_TRY
  if (!sh || !out) throw std::runtime_error("stage times: null argument");
  const WfStageTimes& t = reinterpret_cast<RenderSession*>(sh)->stages;
  out->start_ms = t.startMs;
  out->trace_ms = t.traceMs;
  out->shade_a_ms = t.shadeAMs;
  out->shadow_ms = t.shadowMs;
  out->shade_b_ms = t.shadeBMs;
  out->iterations = t.iterations;
  out->radiance_rays = t.radianceRays;
  out->shadow_rays = t.shadowRays;
  out->launches = t.launches;
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_session_trace_counts_split(sundog_session* sh, sundog_trace_counts* radiance,
                                                 sundog_trace_counts* shadow) {
  SDB_TRY
  if (!sh || !radiance || !shadow) throw std::runtime_error("trace counts: null argument");
  reinterpret_cast<RenderSession*>(sh)->countTraversal(radiance, shadow);
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" void sundog_guiding_defaults(sundog_guiding_config* c) {
  if (c) *c = guideDefaults();
}

extern "C" int sundog_session_set_guiding(sundog_session* sh, int enable,
                                          const sundog_guiding_config* cfg) {
  SDB_TRY
  if (!sh) throw std::runtime_error("session: null handle");
  reinterpret_cast<RenderSession*>(sh)->setGuiding(enable != 0, cfg);
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_session_guiding_stats(sundog_session* sh, sundog_guiding_stats* out) {
  SDB_TRY
  if (!sh || !out) throw std::runtime_error("session: null argument");
  const RenderSession* s = reinterpret_cast<RenderSession*>(sh);
  if (!s->guide) throw std::runtime_error("session: guiding is not enabled");
  *out = s->guide->stats;
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" void sundog_transfer_bytes(uint64_t* h2d, uint64_t* d2h) {
  if (h2d) *h2d = g_h2dBytes.load();
  if (d2h) *d2h = g_d2hBytes.load();
}

extern "C" void sundog_session_destroy(sundog_session* sh) {
  delete reinterpret_cast<RenderSession*>(sh);
}
