// Wavefront path tracer: the plain path kernel's per-path computation split
// into stages over a pool of path slots held in global memory.
//
//   wfStart        fill every slot with a camera path
//   per iteration, over the slots in the live list:
//   wfTraceFetch   trace the radiance ray (traversal only)
//   wfShadeA       shadeVertex: media, flames, escape, shading, emission, the
//                  NEE light draw; queues the slot's shadow ray
//   wfShadow       trace the queued shadow rays (transparent shadows)
//   wfShadeB       finishVertex: NEE contribution, BSDF sample, roulette
//
// A slot whose path ends writes that sample and takes the next camera path at
// once (warp-aggregated counter), so the pool stays full until the frame's
// paths run out. Each stage's code is small next to the megakernel's and
// keeps its state in registers instead of a 1 KB spilled frame, so at full
// occupancy the instruction and local-memory traffic of the megakernel
// disappear; the price is the path state's round trip through global memory
// between stages (a few hundred bytes per path segment).
//
// The stages call the megakernel's own shadeVertex / finishVertex /
// traverse in the same order with the same random draws, so every sample is
// the same sample as in ptPersistent, and the film fold is unchanged.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstddef>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <vector>

#include "pt_path.cuh"
#include "serve.h"
#include "wavefront.h"

namespace sdb {

namespace cg = cooperative_groups;

__constant__ SdLaunch c_wlp;
__constant__ WfPool c_pool;

// Serving batches (GUIDE & kWfServe): tile-passes of many jobs in one pool.
// Each slot's path reads its job's launch block from this table (pool.jobs
// holds the job slot); path ids map to tile-passes as in ptServe (serve.cu),
// and finished samples go to the batch's sample buffer at their path id.
constexpr int kWfServe = 4;
__constant__ SdLaunch c_wjobs[kMaxServeJobs];
__constant__ ServeBatch c_wbatch;

// Launch block of the path in `slot`.
template <int GUIDE>
__device__ __forceinline__ const SdLaunch& slotLaunch(int slot) {
  if (GUIDE & kWfServe) return c_wjobs[c_pool.jobs[slot]];
  return c_wlp;
}

#ifndef SDB_WF_TRACE_BLOCKS
#define SDB_WF_TRACE_BLOCKS 8
#endif
// Resident blocks per SM the stage kernels are compiled for: traversal 8 ->
// 64 registers, shading 5 -> 102 registers. Shading at 6 blocks (80
// registers) gains on config 1 and 2 (1,716 / 2,558 against 1,697 / 2,507
// Mrays/s) and loses on config 0 and the gallery scenes, whose shading
// spills more at 80 registers (01-marble-run 4,476 against 4,709,
// 02-cornell-lume 3,673 against 3,819); 4 blocks lose on all (1,648 /
// 2,402 on configs 1 / 2).
#ifndef SDB_WF_SHADE_BLOCKS
#define SDB_WF_SHADE_BLOCKS 5
#endif
// The second shading stage alone at 6 blocks (80 registers): config 1
// 1,718 -> 1,729 Mrays/s, config 0 2,756 -> 2,779, config 2 and the gallery
// scenes within 0.2%.
#ifndef SDB_WF_SHADEB_BLOCKS
#define SDB_WF_SHADEB_BLOCKS 6
#endif

// Slot index for an append to a list by the calling lanes together.
__device__ __forceinline__ unsigned appendSlot(unsigned* count) {
  cg::coalesced_group g = cg::coalesced_threads();
  unsigned base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(count, g.size());
  return g.shfl(base, 0) + g.thread_rank();
}

template <int GUIDE>
__device__ __forceinline__ unsigned long long nextPathId() {
  cg::coalesced_group g = cg::coalesced_threads();
  unsigned long long* counter = (GUIDE & kWfServe) ? c_wbatch.pathCounter : c_wlp.pathCounter;
  unsigned long long base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(counter, (unsigned long long)g.size());
  return g.shfl(base, 0) + g.thread_rank();
}

// Serving: path id -> its tile-pass's camera sample (false for block
// padding), as serveStart in serve.cu.
__device__ __forceinline__ bool serveStartW(unsigned long long id, Path& p, int& job) {
  const ServeBatch& b = c_wbatch;
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
  startPathAt(c_wjobs[job], it.x0 + lx, it.y0 + ly, it.sampleBegin + sLocal, p);
  p.slot = (int)id;
  return true;
}

// Puts the next camera path in `slot` and lists it in list `out`; leaves the
// slot empty when the frame's paths are used up. Record passes (GUIDE &
// kGuideRecord) start the slot's trail empty.
template <int GUIDE>
__device__ __forceinline__ void refill(int slot, int out, bool start = false) {
  const WfPool& pool = c_pool;
  // When the start stage placed every path, a slot whose path ends has no id
  // left to take: skip the atomic on the path counter that would say so.
  if (!start && !pool.refillOpen) return;
  const unsigned long long numPaths = (GUIDE & kWfServe) ? c_wbatch.numPaths : c_wlp.numPaths;
  while (true) {
    unsigned long long id = nextPathId<GUIDE>();
    if (id >= numPaths) return;
    Path p;
    int job = 0;
    if ((GUIDE & kWfServe) ? serveStartW(id, p, job) : startPath(c_wlp, id, p)) {
      pool.paths[slot].v = p;
      if (GUIDE & kWfServe) pool.jobs[slot] = (unsigned char)job;
      if (GUIDE & kGuideRecord) pool.trails[slot].v.n = 0;
      pool.lists[out][appendSlot(&pool.counts[out])] = slot;
      return;
    }
  }
}

// The finished path's sample; record passes also turn its trail of guided
// vertices into training records.
template <int GUIDE>
__device__ __forceinline__ void finishPath(const Path& p, int slot) {
  float3 L = sanitize3(p.L);
  if (GUIDE & kGuideRecord) guideFlush(c_wlp, c_pool.trails[slot].v, L);
  float4* sampleL = (GUIDE & kWfServe) ? c_wbatch.sampleL : c_wlp.sampleL;
  sampleL[p.slot] = make_float4(L.x, L.y, L.z, 1.0f);
}

template <int GUIDE = 0>
__device__ __forceinline__ void addRays(unsigned long long rays) {
  for (int off = 16; off > 0; off >>= 1) rays += __shfl_down_sync(0xFFFFFFFFu, rays, off);
  unsigned long long* counter = (GUIDE & kWfServe) ? c_wbatch.rayCounter : c_wlp.rayCounter;
  if ((threadIdx.x & 31) == 0 && rays) atomicAdd(counter, rays);
}

template <int GUIDE>
__global__ void __launch_bounds__(kRenderBlock) wfStart() {
  const WfPool& pool = c_pool;
  for (int slot = blockIdx.x * blockDim.x + threadIdx.x; slot < pool.cap;
       slot += gridDim.x * blockDim.x)
    refill<GUIDE>(slot, 0, true);
}

// Camera paths into the pool without atomics, for frames whose 8x8 pixel
// tiles cover the image exactly (every path id is a pixel sample, so
// refill's id counter and list appends would only number the slots in
// order): slot i takes path i, the live list is the identity, and the list
// length and path counter continue from n = min(pool, paths). The same
// paths in the same slots as wfStart.
template <int GUIDE>
__global__ void __launch_bounds__(kRenderBlock) wfStartDirect(unsigned n) {
  const WfPool& pool = c_pool;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    pool.counts[0] = n;
    *c_wlp.pathCounter = n;
  }
  for (unsigned slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n;
       slot += gridDim.x * blockDim.x) {
    Path p;
    startPath(c_wlp, slot, p);
    pool.paths[slot].v = p;
    if (GUIDE & kGuideRecord) pool.trails[slot].v.n = 0;
    pool.lists[0][slot] = (int)slot;
  }
}

// Stores a closest-hit candidate straight into the slot's hit record (three
// 16-byte stores), so the trace loop keeps no hit fields in registers: each
// closer hit overwrites the record, and a ray that hits nothing leaves the
// miss marker (inst = -1) written when it was fetched.
__device__ __forceinline__ void putHit(PoolSlot<TraceHit>& s, float t, int inst, int prim, float u,
                                       float v, float3 nq, bool front) {
  static_assert(offsetof(TraceHit, nq) == 20 && offsetof(TraceHit, front) == 32 &&
                    sizeof(PoolSlot<TraceHit>) == 48,
                "TraceHit layout assumed by the vector stores");
  float4* p = reinterpret_cast<float4*>(&s);
  p[0] = make_float4(t, __int_as_float(inst), __int_as_float(prim), u);
  p[1] = make_float4(v, nq.x, nq.y, nq.z);
  p[2] = make_float4(__int_as_float(front ? 1 : 0), 0.0f, 0.0f, 0.0f);
}

// Steps a lane may take in a row inside one round of the fetch loop, and
// the fewest lanes still descending that keep the warp in the run (config 1
// / config 0, Mrays/s; while any lane descends: 1 step 1,351 / 2,648; 4:
// 1,459 / 2,697; 8: 1,497 / 2,723; 16: 1,512 / 2,726; 64: 1,499 / 2,709;
// letting leaves continue the run too, 16 steps: 1,405 / 2,692; 16 steps
// while at least 2 / 4 / 8 / 12 lanes descend: 1,555 / 2,713, 1,568 /
// 2,718, 1,559 / 2,655, 1,525 / 2,680).
#ifndef SDB_WF_INNER
#define SDB_WF_INNER 16
#endif
#ifndef SDB_WF_INNER_MIN
#define SDB_WF_INNER_MIN 4
#endif
// Idle lanes a warp gathers before it fetches new rays (on the instancing
// frame with the one-action loop: 894 Mrays/s at 24, 869 with a grid-stride
// loop, 752 when every idle lane fetches at once: fresh rays at the TLAS
// root diverge from the warp's deep BLAS walks; with the 4-wide walk and
// descent runs, config 1 / config 0: 1,717 / 2,798 at 20, 1,706 / 2,801 at
// 24, 1,678 / 2,799 at 28).
#ifndef SDB_WF_FETCH_IDLE
#define SDB_WF_FETCH_IDLE 20
#endif

// Radiance rays with dynamic ray fetch (Aila and Laine, "Understanding the
// Efficiency of Ray Traversal on GPUs", 2009): the traversal loop runs per
// warp, and a lane whose ray is done writes its hit and, once
// SDB_WF_FETCH_IDLE lanes of the warp are idle, takes the next ray of the
// live list (one warp-aggregated atomicAdd on counts[3]), so a warp no longer
// waits for its longest ray. Each ray visits the nodes of traverse<false>
// (sd_trace.cuh) in the same order with the same tests: the same closest
// accepted hit. (Shadow rays, shorter, gained nothing from it.) SERVE: a
// serving batch, each lane tracing in its own job's scene.
#if SDB_WIDE_BVH
// The same stage over the compressed 8-wide BVH (CwNode, sd_trace.cuh): each
// loop iteration a lane either tests one primitive of its current leaf group
// (a triangle, or a TLAS instance: quadric roots or entry into its BLAS),
// tests the 8 child boxes of the nearest remaining child node, or pops a
// group. The visit order and tests are those of traverse<false> in the
// 8-wide build: the same closest accepted hit.
template <bool SERVE>
__global__ void __launch_bounds__(kRenderBlock, SDB_WF_TRACE_BLOCKS) wfTraceFetch(int in) {
  const WfPool& pool = c_pool;
  const unsigned n = pool.counts[in];
  const unsigned full = 0xFFFFFFFFu;
  const unsigned ltMask = (1u << (threadIdx.x & 31)) - 1u;
  int job = 0;  // SERVE: the lane's job slot
  const float tmin = 0.0f;
  unsigned long long rays = 0;
  int slot = -1;
  bool exhausted = false;  // warp-uniform
  float3 O = v3(0.0f), D = v3(0.0f);
  RayCtx ray;
  rayInit(ray, O, v3(1.0f), false);
  float tmax = 0.0f;
  TraceHit hit;
  bool found = false, inBlas = false;
  int curInst = -1, sp = 0;
  uint32_t gBase = 0, gHits = 0, gImask = 0, tBase = 0, tBits = 0;
  uint2 stack[kCwStack];
  while (true) {
    const unsigned idle = __ballot_sync(full, slot < 0);
    if (!exhausted && (idle == full || __popc(idle) >= SDB_WF_FETCH_IDLE)) {
      const int leader = __ffs(idle) - 1;
      unsigned base = 0;
      if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(&pool.counts[3], (unsigned)__popc(idle));
      base = __shfl_sync(full, base, leader);
      if (base + __popc(idle) >= n) exhausted = true;
      if (slot < 0) {
        unsigned i = base + __popc(idle & ltMask);
        if (i < n) {
          slot = pool.lists[in][i];
          if (SERVE) job = pool.jobs[slot];
          const SdLaunch& jl = SERVE ? c_wjobs[job] : c_wlp;
          O = pool.paths[slot].v.o;
          D = pool.paths[slot].v.d;
          rayInit(ray, O, D, false);
          tmax = 1e16f;
          found = false;
          inBlas = false;
          curInst = -1;
          sp = 0;
          gBase = (uint32_t)jl.tlasRoot;
          gHits = jl.numInstances > 0 ? 1u << (0u ^ ray.rayOct) : 0u;
          gImask = 1u;
          tBits = 0;
        }
      }
    }
    if (__ballot_sync(full, slot >= 0) == 0) {
      if (exhausted) break;
      continue;
    }
    if (slot < 0) continue;
    const SdLaunch& lp = SERVE ? c_wjobs[job] : c_wlp;
    if (tBits) {
      const int j = __ffs(tBits) - 1;
      tBits &= tBits - 1u;
      const int prim = (int)tBase + j;
      if (!inBlas) {
        const SdInstance& inst = lp.inst[prim];
        float3 o2 = xfPoint(inst.w2o, O), d2 = xfVec(inst.w2o, D);
        if (inst.kind == GK_MESH) {
          // Suspend this level (the scene build keeps TLAS + BLAS depth
          // within the stack) and walk the BLAS in object space.
          if (sp + 3 > kCwStack) continue;
          if (gHits) stack[sp++] = make_uint2(gBase, gHits | (gImask << 8));
          if (tBits) stack[sp++] = make_uint2(tBase, tBits | kGroupPrims);
          stack[sp++] = make_uint2(0xFFFFFFFFu, kGroupMarker);
          inBlas = true;
          curInst = prim;
          rayInit(ray, o2, d2, true);
          gBase = (uint32_t)lp.meshes[inst.mesh].root;
          gHits = 1u << (0u ^ ray.rayOct);
          gImask = 1u;
          tBits = 0;
          continue;
        }
        QHits qh = hitQuadric(inst.kind, o2, d2, tmin, tmax);
        for (int k = 0; k < qh.n; k++) {
          const QHit& q = qh.h[k];
          if (q.t >= tmax) continue;
          bool front = dot(q.n, d2) < 0.0f;
          if ((inst.flags & kInstMasked) && !faceAccepts(lp, inst, front, q.u, q.v)) continue;
          tmax = q.t;
          found = true;
          hit.t = q.t;
          hit.inst = prim;
          hit.prim = 0;
          hit.u = q.u;
          hit.v = q.v;
          hit.nq = q.n;
          hit.front = front;
        }
        continue;
      }
      // Triangle of the current BLAS, in object space.
      const float4* tp = lp.tris + 3 * (size_t)prim;
      float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
      float t, b1, b2;
      float3 p0 = v3(a.x, a.y, a.z), p1 = v3(b.x, b.y, b.z), p2 = v3(c.x, c.y, c.z);
      if (!wtHit(ray.wt, ray.o, p0, p1, p2, tmin, tmax, t, b1, b2)) continue;
      const int tri = __float_as_int(a.w);
      const SdInstance& inst = lp.inst[curInst];
      bool front;
      if (!(inst.flags & (kInstMasked | kInstTransmissive))) {
        front = dot(cross(p1 - p0, p2 - p0), ray.d) < 0.0f;
      } else {
        ShadePt spt = triShade(lp, inst, tri, b1, b2, D);
        if ((inst.flags & kInstMasked) && !faceAccepts(lp, inst, spt.front, spt.u, spt.v)) continue;
        front = spt.front;
      }
      tmax = t;
      found = true;
      hit.t = t;
      hit.inst = curInst;
      hit.prim = tri;
      hit.u = b1;
      hit.v = b2;
      hit.front = front;
      continue;
    }
    if (gHits) {
      const int b = __ffs(gHits) - 1;
      gHits &= gHits - 1u;
      const uint32_t cs = (uint32_t)b ^ ray.rayOct;
      const int child = (int)(gBase + __popc(gImask & ((1u << cs) - 1u)));
      if (gHits && sp < kCwStack) stack[sp++] = make_uint2(gBase, gHits | (gImask << 8));
      CwHits h = cwIntersect(lp.cw, child, ray.o, ray.id, ray.rayOct, tmin, tmax);
      gBase = h.childBase;
      gHits = h.hits;
      gImask = h.imask;
      tBase = h.primBase;
      tBits = h.leafBits;
      continue;
    }
    if (sp == 0) {  // ray done
      if (!found) hit.inst = -1;
      pool.hits[slot].v = hit;
      rays++;
      slot = -1;
      continue;
    }
    const uint2 e = stack[--sp];
    if (e.y & kGroupMarker) {
      inBlas = false;
      rayInit(ray, O, D, false);
    } else if (e.y & kGroupPrims) {
      tBase = e.x;
      tBits = e.y & 0xFFFFFFu;
    } else {
      gBase = e.x;
      gHits = e.y & 0xFFu;
      gImask = (e.y >> 8) & 0xFFu;
    }
  }
  addRays<SERVE ? kWfServe : 0>(rays);
}
#else
// Sink of the trace stage's walks (binTravStep, sd_trace.cuh): closer hits go
// straight to the slot's hit record and the world ray is re-read from the
// slot when a walk leaves a BLAS, so neither stays in registers.
struct PoolSink {
  const WfPool& pool;
  int slot;
  __device__ __forceinline__ void world(float3& ro, float3& rd) const {
    ro = pool.paths[slot].v.o;
    rd = pool.paths[slot].v.d;
  }
  __device__ __forceinline__ float3 worldDir() const { return pool.paths[slot].v.d; }
  __device__ __forceinline__ void hit(float t, int inst, int prim, float u, float v, float3 nq,
                                      bool front) const {
    putHit(pool.hits[slot], t, inst, prim, u, v, nq, front);
  }
};

template <bool SERVE>
__global__ void __launch_bounds__(kRenderBlock, SDB_WF_TRACE_BLOCKS) wfTraceFetch(int in) {
  const WfPool& pool = c_pool;
  const unsigned n = pool.counts[in];
  const unsigned full = 0xFFFFFFFFu;
  const unsigned ltMask = (1u << (threadIdx.x & 31)) - 1u;
  int job = 0;  // SERVE: the lane's job slot
  unsigned long long rays = 0;
  int slot = -1;
  bool exhausted = false;  // warp-uniform
  BinTrav t;
  TravStack stack;
  float trUnused = 1.0f;
  float3 tauUnused = v3(0.0f);
  while (true) {
    const unsigned idle = __ballot_sync(full, slot < 0);
    if (!exhausted && (idle == full || __popc(idle) >= SDB_WF_FETCH_IDLE)) {
      const int leader = __ffs(idle) - 1;
      unsigned base = 0;
      if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(&pool.counts[3], (unsigned)__popc(idle));
      base = __shfl_sync(full, base, leader);
      if (base + __popc(idle) >= n) exhausted = true;
      if (slot < 0) {
        unsigned i = base + __popc(idle & ltMask);
        if (i < n) {
          slot = pool.lists[in][i];
          if (SERVE) job = pool.jobs[slot];
          const SdLaunch& jl = SERVE ? c_wjobs[job] : c_wlp;
          binTravStart(t, jl, pool.paths[slot].v.o, pool.paths[slot].v.d, 1e16f);
          pool.hits[slot].v.inst = -1;  // a miss until a hit is stored
        }
      }
    }
    if (__ballot_sync(full, slot >= 0) == 0) {
      if (exhausted) break;
      continue;
    }
    // One step for every lane with a ray; then lanes that landed on an
    // inner node keep descending (the while-while loop of Aila and Laine
    // 2009 inside the dynamic-fetch loop) while at least SDB_WF_INNER_MIN of
    // the warp's lanes do so, up to SDB_WF_INNER steps, before the warp
    // meets again at the fetch vote; lanes at a leaf wait for the next round.
    const SdLaunch& lp = SERVE ? c_wjobs[job] : c_wlp;
    PoolSink sink{pool, slot};
    int r = kTravMore;
    bool go = slot >= 0;
    for (int k = 1;; k++) {
      if (go) r = binTravStep<false, false>(t, stack, lp, sink, trUnused, tauUnused, nullptr);
      go = slot >= 0 && r == kTravMore && t.cur >= 0;
      if (k >= SDB_WF_INNER || __popc(__ballot_sync(full, go)) < SDB_WF_INNER_MIN) break;
    }
    if (slot >= 0 && r == kTravDone) {
      rays++;  // its closest hit is already in the slot
      slot = -1;
    }
  }
  addRays<SERVE ? kWfServe : 0>(rays);
}
#endif

template <int GUIDE>
__global__ void __launch_bounds__(kRenderBlock, SDB_WF_SHADE_BLOCKS) wfShadeA(int in, int out) {
  const WfPool& pool = c_pool;
  const unsigned n = pool.counts[in];
  unsigned long long rays = 0;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int slot = pool.lists[in][i];
    const SdLaunch& lp = slotLaunch<GUIDE>(slot);
    Path p = pool.paths[slot].v;
    TraceHit h = pool.hits[slot].v;
    Vertex v;
    if (shadeVertex<false>(lp, p, h.inst >= 0, h, rays, v)) {
      pool.paths[slot].v = p;
      pool.verts[slot].v = v;
      pool.pending[slot] = 1;
      if (v.nee) pool.shadowList[appendSlot(&pool.counts[2])] = slot;
    } else {
      finishPath<GUIDE>(p, slot);
      pool.pending[slot] = 0;
      refill<GUIDE>(slot, out);
    }
  }
  addRays<GUIDE>(rays);
}

// Shadow rays, one per thread to the end of its walk (grid-stride over the
// shadow list).
template <int GUIDE>
__global__ void __launch_bounds__(kRenderBlock, SDB_WF_TRACE_BLOCKS) wfShadow() {
  const WfPool& pool = c_pool;
  const unsigned n = pool.counts[2];
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int slot = pool.shadowList[i];
    const SdLaunch& lp = slotLaunch<GUIDE>(slot);
    const Vertex& v = pool.verts[slot].v;
    float3 tr = shadowTransmittance<false>(lp, v.so, v.wi, v.tmaxS, nullptr);
    pool.trs[slot] = make_float4(tr.x, tr.y, tr.z, 0.0f);
  }
}

#if !SDB_WIDE_BVH
// Sink of the shadow stage's walks: the world ray is the slot's queued
// shadow ray, re-read when a walk leaves a BLAS.
struct ShadowSink {
  const WfPool& pool;
  int slot;
  __device__ __forceinline__ void world(float3& ro, float3& rd) const {
    ro = pool.verts[slot].v.so;
    rd = pool.verts[slot].v.wi;
  }
  __device__ __forceinline__ float3 worldDir() const { return pool.verts[slot].v.wi; }
  __device__ __forceinline__ void hit(float, int, int, float, float, float3, bool) const {}
};

// Shadow rays with the trace stage's dynamic fetch (counter counts[4]) and
// node-descent runs: the walk and transmittance of shadowTransmittance, many
// rays interleaved per warp. Faster than wfShadow where walks are long and
// uneven (config 1, 1024 instances: 29.3 -> 24.5 ms per frame), slower on
// small scenes (config 0: 2,730 -> 2,672 Mrays/s; config 2: 113.7 -> 122.2
// ms), so renders choose by instance count (kShadowFetchInstances).
template <int GUIDE>
__global__ void __launch_bounds__(kRenderBlock, SDB_WF_TRACE_BLOCKS) wfShadowFetch() {
  const WfPool& pool = c_pool;
  const unsigned n = pool.counts[2];
  const unsigned full = 0xFFFFFFFFu;
  const unsigned ltMask = (1u << (threadIdx.x & 31)) - 1u;
  int slot = -1;
  bool exhausted = false;  // warp-uniform
  BinTrav t;
  TravStack stack;
  float trProd = 1.0f;
  float3 tau = v3(0.0f);
  while (true) {
    const unsigned idle = __ballot_sync(full, slot < 0);
    if (!exhausted && (idle == full || __popc(idle) >= SDB_WF_FETCH_IDLE)) {
      const int leader = __ffs(idle) - 1;
      unsigned base = 0;
      if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(&pool.counts[4], (unsigned)__popc(idle));
      base = __shfl_sync(full, base, leader);
      if (base + __popc(idle) >= n) exhausted = true;
      if (slot < 0) {
        unsigned i = base + __popc(idle & ltMask);
        if (i < n) {
          slot = pool.shadowList[i];
          const Vertex& v = pool.verts[slot].v;
          binTravStart(t, slotLaunch<GUIDE>(slot), v.so, v.wi, v.tmaxS);
          trProd = 1.0f;
          tau = v3(0.0f);
        }
      }
    }
    if (__ballot_sync(full, slot >= 0) == 0) {
      if (exhausted) break;
      continue;
    }
    const SdLaunch& lp = slotLaunch<GUIDE>(slot >= 0 ? slot : 0);
    ShadowSink sink{pool, slot};
    int r = kTravMore;
    bool go = slot >= 0;
    for (int k = 1;; k++) {
      if (go) r = binTravStep<true, false>(t, stack, lp, sink, trProd, tau, nullptr);
      go = slot >= 0 && r == kTravMore && t.cur >= 0;
      if (k >= SDB_WF_INNER || __popc(__ballot_sync(full, go)) < SDB_WF_INNER_MIN) break;
    }
    if (slot >= 0 && r != kTravMore) {
      float3 tr = v3(0.0f);
      if (r == kTravDone) {
        tau = v3(fmaxf(0.0f, tau.x), fmaxf(0.0f, tau.y), fmaxf(0.0f, tau.z));
        tr = v3(trProd);
        if (hmax(tau) > 0.0f) tr = tr * vexp(-tau);
      }
      pool.trs[slot] = make_float4(tr.x, tr.y, tr.z, 0.0f);
      slot = -1;
    }
  }
}
#else
// The 8-wide build traces shadow rays one per thread.
template <int GUIDE>
__global__ void wfShadowFetch() {}
#endif

// GUIDE & kGuideSample: the BSDF sample by MIS with the learned guide
// (sd_guide.cuh; the mixture table is in the launch block). GUIDE &
// kGuideRecord: the guided vertex joins the slot's trail.
template <int GUIDE>
__global__ void __launch_bounds__(kRenderBlock, SDB_WF_SHADEB_BLOCKS) wfShadeB(int in, int out) {
  const WfPool& pool = c_pool;
  const unsigned n = pool.counts[in];
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int slot = pool.lists[in][i];
    if (!pool.pending[slot]) continue;
    const SdLaunch& lp = slotLaunch<GUIDE>(slot);
    Path p = pool.paths[slot].v;
    const Vertex v = pool.verts[slot].v;
    float3 tr = v3(0.0f);
    if (v.nee) {
      float4 t4 = pool.trs[slot];
      tr = v3(t4.x, t4.y, t4.z);
    }
    GuideTrail* trail = (GUIDE & kGuideRecord) ? &pool.trails[slot].v : nullptr;
    if (finishVertex<GUIDE>(lp, p, v, tr, trail)) {
      pool.paths[slot].v = p;
      pool.lists[out][appendSlot(&pool.counts[out])] = slot;
    } else {
      finishPath<GUIDE>(p, slot);
      refill<GUIDE>(slot, out);
    }
  }
}

// ---- host ---------------------------------------------------------------------

template <typename K>
static int gridFor(K kernel) {
  int dev = 0, sms = 0, perSm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, kRenderBlock, 0);
  return sms * (perSm < 1 ? 1 : perSm);
}

void WfBuffers::ensure(int slots) {
  if (slots <= cap) return;
  // At most half of the device memory that is free (counting the pool about
  // to be replaced), so films, scenes and other work keep room; at least
  // 1 M slots.
  size_t freeB = 0, totB = 0;
  cudaCheck(cudaMemGetInfo(&freeB, &totB), "cudaMemGetInfo");
  const size_t budget = (freeB + (size_t)cap * wfSlotBytes()) / 2;
  const size_t fit = std::max<size_t>(budget / wfSlotBytes(), (size_t)1 << 20);
  slots = (int)std::min<size_t>((size_t)slots, fit);
  if (slots <= cap) return;
  const size_t n = (size_t)slots;
  const size_t sizes[9] = {n * sizeof(PoolSlot<Path>), n * sizeof(PoolSlot<Vertex>),
                           n * sizeof(PoolSlot<TraceHit>), n * sizeof(float4), n,
                           n * sizeof(int), n * sizeof(int), n * sizeof(int), n};
  size_t offs[9], total = 0;
  for (int k = 0; k < 9; k++) {
    offs[k] = total;
    total += (sizes[k] + 255) & ~(size_t)255;
  }
  slab.release();
  slab.alloc(total);
  void** parts[9] = {&paths, &verts, &hits, &trs, &pending, &list0, &list1, &shadow, &jobs};
  for (int k = 0; k < 9; k++) *parts[k] = (char*)slab.ptr + offs[k];
  if (!counts.ptr) counts.alloc(8 * sizeof(unsigned));
  if (!hostCount) hostCount = pinnedWords();
  cap = slots;
  gridTrace = gridFor(wfTraceFetch<false>);
  gridShadeA = gridFor(wfShadeA<0>);
  gridShadow = gridFor(wfShadow<0>);
  gridShadeB = gridFor(wfShadeB<0>);
  gridStart = gridFor(wfStart<0>);
}

void WfBuffers::ensureTrails() {
  if (trailCap >= cap) return;
  trails.alloc((size_t)cap * sizeof(PoolSlot<GuideTrail>));
  trailCap = cap;
}

WfBuffers::~WfBuffers() {
  if (hostCount) returnPinnedWords(hostCount);
  for (cudaEvent_t& e : ev)
    if (e) cudaEventDestroy(e);
}

// One idle pool per device, kept between sessions while the device-memory
// cache is on (sundog_set_device_memory_cache); otherwise a finished
// session's pool is freed with it.
static std::mutex g_poolMu;
static std::unique_ptr<WfBuffers> g_idle[64];

std::unique_ptr<WfBuffers> wfAcquire() {
  int dev = 0;
  cudaCheck(cudaGetDevice(&dev), "cudaGetDevice");
  std::lock_guard<std::mutex> lock(g_poolMu);
  if (dev >= 0 && dev < 64 && g_idle[dev]) return std::move(g_idle[dev]);
  return std::unique_ptr<WfBuffers>(new WfBuffers());
}

void wfRelease(std::unique_ptr<WfBuffers> b) {
  if (!b) return;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  if (!keepDeviceMemory()) return;  // b frees its buffers here
  std::lock_guard<std::mutex> lock(g_poolMu);
  if (!g_idle[dev] || g_idle[dev]->cap < b->cap) g_idle[dev] = std::move(b);
}

void wfReleaseIdle() {
  int cur = 0;
  if (cudaGetDevice(&cur) != cudaSuccess) return;
  std::lock_guard<std::mutex> lock(g_poolMu);
  for (int d = 0; d < 64; d++) {
    if (!g_idle[d]) continue;
    if (cudaSetDevice(d) == cudaSuccess) g_idle[d].reset();
  }
  cudaSetDevice(cur);
}

size_t wfSlotBytes() {
  return sizeof(PoolSlot<Path>) + sizeof(PoolSlot<Vertex>) + sizeof(PoolSlot<TraceHit>) +
         sizeof(float4) + 2 + 3 * sizeof(int);
}

// Renders the launch block's paths (lp.numPaths ids, counters already
// cleared) into lp.sampleL through the stages. Returns the kernels launched.
// One iteration's stage kernels for mode GUIDE (guide bits, or kWfServe).
// With `timed`, events ev[1..5] bracket the four stage launches.
template <int GUIDE>
static void wfIteration(const WfBuffers& b, cudaStream_t st, int cur, int nxt, bool timed,
                        bool shadowFetch) {
  if (timed) cudaEventRecord(b.ev[1], st);
  wfTraceFetch<(GUIDE & kWfServe) != 0><<<b.gridTrace, kRenderBlock, 0, st>>>(cur);
  if (timed) cudaEventRecord(b.ev[2], st);
  wfShadeA<GUIDE><<<b.gridShadeA, kRenderBlock, 0, st>>>(cur, nxt);
  if (timed) cudaEventRecord(b.ev[3], st);
  if (shadowFetch && !SDB_WIDE_BVH)
    wfShadowFetch<GUIDE><<<b.gridShadow, kRenderBlock, 0, st>>>();
  else
    wfShadow<GUIDE><<<b.gridShadow, kRenderBlock, 0, st>>>();
  if (timed) cudaEventRecord(b.ev[4], st);
  wfShadeB<GUIDE><<<b.gridShadeB, kRenderBlock, 0, st>>>(cur, nxt);
  if (timed) cudaEventRecord(b.ev[5], st);
}

static double evMs(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.0f;
  cudaCheck(cudaEventElapsedTime(&ms, a, b), "stage timing");
  return ms;
}

// Fills the pool with the first paths of ids [0, numPaths) and runs stage
// iterations until no path is live (the launch block or batch is already in
// constant memory). Returns the kernels launched.
static int runPool(WfBuffers& b, cudaStream_t st, unsigned long long numPaths, int mode,
                   bool shadowFetch, bool directStart, WfStageTimes* times = nullptr) {
  const bool timed = times != nullptr;
  if (timed && !b.ev[0])
    for (cudaEvent_t& e : b.ev) cudaCheck(cudaEventCreate(&e), "stage timing events");
  WfPool pool;
  pool.paths = (PoolSlot<Path>*)b.paths;
  pool.verts = (PoolSlot<Vertex>*)b.verts;
  pool.hits = (PoolSlot<TraceHit>*)b.hits;
  pool.trs = (float4*)b.trs;
  pool.pending = (unsigned char*)b.pending;
  pool.lists[0] = (int*)b.list0;
  pool.lists[1] = (int*)b.list1;
  pool.shadowList = (int*)b.shadow;
  pool.counts = (unsigned*)b.counts.ptr;
  pool.trails = (PoolSlot<GuideTrail>*)b.trails.ptr;
  pool.jobs = (unsigned char*)b.jobs;
  pool.cap = (int)std::min<unsigned long long>((unsigned long long)b.cap, numPaths);
  pool.refillOpen = (unsigned long long)pool.cap < numPaths ? 1 : 0;
  cudaCheck(cudaMemcpyToSymbolAsync(c_pool, &pool, sizeof pool, 0, cudaMemcpyHostToDevice, st),
            "wavefront pool");
  cudaCheck(cudaMemsetAsync(b.counts.ptr, 0, b.counts.bytes, st), "wavefront counts");
  int launches = 0;
  if (timed) cudaEventRecord(b.ev[0], st);
  const unsigned direct = (unsigned)pool.cap;
  if (mode & kWfServe)
    wfStart<kWfServe><<<b.gridStart, kRenderBlock, 0, st>>>();
  else if (directStart && (mode & kGuideRecord))
    wfStartDirect<kGuideRecord><<<b.gridStart, kRenderBlock, 0, st>>>(direct);
  else if (directStart)
    wfStartDirect<0><<<b.gridStart, kRenderBlock, 0, st>>>(direct);
  else if (mode & kGuideRecord)
    wfStart<kGuideRecord><<<b.gridStart, kRenderBlock, 0, st>>>();
  else
    wfStart<0><<<b.gridStart, kRenderBlock, 0, st>>>();
  cudaCheck(cudaGetLastError(), "wfStart");
  launches++;
  if (timed) {
    cudaEventRecord(b.ev[1], st);
    cudaCheck(cudaEventSynchronize(b.ev[1]), "wfStart");
    times->startMs += evMs(b.ev[0], b.ev[1]);
    times->launches++;
  }
  unsigned* counts = (unsigned*)b.counts.ptr;
  int cur = 0;
  for (int iter = 0;; iter++) {
    int nxt = 1 - cur;
    cudaCheck(cudaMemsetAsync(counts + nxt, 0, sizeof(unsigned), st), "wavefront counts");
    cudaCheck(cudaMemsetAsync(counts + 2, 0, 3 * sizeof(unsigned), st), "wavefront counts");
    switch (mode) {
      case 0: wfIteration<0>(b, st, cur, nxt, timed, shadowFetch); break;
      case kGuideSample: wfIteration<kGuideSample>(b, st, cur, nxt, timed, shadowFetch); break;
      case kGuideRecord: wfIteration<kGuideRecord>(b, st, cur, nxt, timed, shadowFetch); break;
      case kGuideSample | kGuideRecord:
        wfIteration<kGuideSample | kGuideRecord>(b, st, cur, nxt, timed, shadowFetch);
        break;
      default: wfIteration<kWfServe>(b, st, cur, nxt, timed, shadowFetch); break;
    }
    cudaCheck(cudaGetLastError(), "wavefront stage");
    launches += 4;
    cur = nxt;
    // All four counters: [cur] is now the next iteration's live list, [1 - cur]
    // the list this iteration traced, [2] its shadow rays.
    cudaCheck(cudaMemcpyAsync(b.hostCount, counts, 4 * sizeof(unsigned), cudaMemcpyDeviceToHost, st),
              "wavefront count");
    cudaCheck(cudaStreamSynchronize(st), "wavefront iteration");
    if (timed) {
      times->traceMs += evMs(b.ev[1], b.ev[2]);
      times->shadeAMs += evMs(b.ev[2], b.ev[3]);
      times->shadowMs += evMs(b.ev[3], b.ev[4]);
      times->shadeBMs += evMs(b.ev[4], b.ev[5]);
      times->iterations++;
      times->launches += 4;
      times->radianceRays += b.hostCount[1 - cur];
      times->shadowRays += b.hostCount[2];
    }
    if (b.hostCount[cur] == 0) break;
    if (iter > (1 << 24)) throw std::runtime_error("wavefront: no progress");
  }
  return launches;
}

int wfRender(const SdLaunch& lp, WfBuffers& b, cudaStream_t st, int guide, WfStageTimes* times) {
  if (guide < 0 || guide > (kGuideSample | kGuideRecord))
    throw std::runtime_error("wavefront: invalid guide mode");
  if (guide & kGuideRecord) b.ensureTrails();
  cudaCheck(cudaMemcpyToSymbolAsync(c_wlp, &lp, sizeof lp, 0, cudaMemcpyHostToDevice, st),
            "wavefront launch block");
  const bool exactTiles = lp.shardCount <= 1 && lp.npixPad == lp.width * lp.height;
  return runPool(b, st, lp.numPaths, guide, lp.numInstances >= kShadowFetchInstances, exactTiles,
                 times);
}

cudaError_t wfSetJobs(const SdLaunch* table, cudaStream_t st) {
  return cudaMemcpyToSymbolAsync(c_wjobs, table, kMaxServeJobs * sizeof(SdLaunch), 0,
                                 cudaMemcpyHostToDevice, st);
}

int wfRenderBatch(const ServeBatch& batch, WfBuffers& b, cudaStream_t st, int maxInstances) {
  cudaCheck(cudaMemcpyToSymbolAsync(c_wbatch, &batch, sizeof batch, 0, cudaMemcpyHostToDevice, st),
            "wavefront batch");
  return runPool(b, st, batch.numPaths, kWfServe, maxInstances >= kShadowFetchInstances, false);
}

}  // namespace sdb
