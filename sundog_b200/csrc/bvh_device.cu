// Two-level BVH built on the device: binned-SAH top-down construction in
// breadth-first levels, one CTA per node range.
//
// The reference builds its acceleration structures on the device through
// optixAccelBuild (src/accel.cpp:8-44, 46-121). This builder makes the binary
// two-children-per-node layout the traversal reads (BvhNode: both child boxes
// in the parent), with the same split rules as the host builder
// (bvh_build.cpp): ranges of more than 32 primitives are split by a binned
// SAH over all three axes at once (32 bins per axis over the centroid
// bounds), ranges of up to 32 by an exact SAH sweep over their sorted
// centroids, a range becomes a leaf when it holds at most maxLeaf primitives
// and intersecting them costs no more than splitting (node visit = 1.2
// primitive tests), and ranges whose centroids coincide (or below depth 40)
// are split at their middle. SAH costs use round-to-nearest FP32 intrinsics
// in the host builder's order.
//
// Each level's kernel reads that level's ranges and the current primitive
// order, and for each range either stores its primitives at their final leaf
// positions and writes the leaf link into the parent node, or allocates a
// node (its index into the parent), stores both children's boxes in it,
// partitions the range's primitives stably into the next order buffer, and
// appends the two child ranges. The host reads the next level's range count
// after each level. Nodes come out in level order (the root first).
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <stdexcept>
#include <vector>

#include "bvh_device.h"
#include "render_session.h"

namespace sdb {

namespace {

constexpr int kBuildThreads = 128;
constexpr int kBuildBins = 32;
constexpr int kBuildSmall = 32;
constexpr int kBuildDepthLimit = 40;

struct BuildRange {
  int b, e, depth;
  int parentSlot;  // int index of the parent's link word (node * 16 + 12 + side); -1: root
  float lo[3], hi[3];
};

struct BuildCtx {
  const float4* lo;    // primitive boxes (.w unused)
  const float4* hi;
  const float4* cent;  // centroids
  BvhNode* nodes;
  int* nodeCount;
  int* order;          // final leaf order
  int* maxDepth;
  int* error;          // set when a capacity bound below would be exceeded
  int maxLeaf, nodeBase, primBase;
  int nodeCap, rangeCap;
};

// Float order as signed ints, for shared-memory atomic min / max.
__device__ __forceinline__ int fkey(float f) {
  int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float fdec(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7FFFFFFF); }

struct Bx {
  float lo[3], hi[3];
};
__device__ __forceinline__ Bx bxEmpty() {
  Bx b;
  for (int a = 0; a < 3; a++) {
    b.lo[a] = FLT_MAX;
    b.hi[a] = -FLT_MAX;
  }
  return b;
}
__device__ __forceinline__ void bxGrow(Bx& b, const Bx& o) {
  for (int a = 0; a < 3; a++) {
    b.lo[a] = o.lo[a] < b.lo[a] ? o.lo[a] : b.lo[a];
    b.hi[a] = o.hi[a] > b.hi[a] ? o.hi[a] : b.hi[a];
  }
}
// Surface area as the host builder computes it: 2 (xy + yz + zx), 0 when empty.
__device__ __forceinline__ float bxArea(const Bx& b) {
  float ex = __fsub_rn(b.hi[0], b.lo[0]), ey = __fsub_rn(b.hi[1], b.lo[1]),
        ez = __fsub_rn(b.hi[2], b.lo[2]);
  if (ex < 0.0f) return 0.0f;
  return __fmul_rn(2.0f, __fadd_rn(__fadd_rn(__fmul_rn(ex, ey), __fmul_rn(ey, ez)),
                                   __fmul_rn(ez, ex)));
}
__device__ __forceinline__ Bx bxShfl(const Bx& b, int src) {
  Bx r;
  for (int a = 0; a < 3; a++) {
    r.lo[a] = __shfl_sync(0xFFFFFFFFu, b.lo[a], src);
    r.hi[a] = __shfl_sync(0xFFFFFFFFu, b.hi[a], src);
  }
  return r;
}
__device__ __forceinline__ Bx bxShflUp(const Bx& b, int d) {
  Bx r;
  for (int a = 0; a < 3; a++) {
    r.lo[a] = __shfl_up_sync(0xFFFFFFFFu, b.lo[a], d);
    r.hi[a] = __shfl_up_sync(0xFFFFFFFFu, b.hi[a], d);
  }
  return r;
}
__device__ __forceinline__ Bx bxShflDown(const Bx& b, int d) {
  Bx r;
  for (int a = 0; a < 3; a++) {
    r.lo[a] = __shfl_down_sync(0xFFFFFFFFu, b.lo[a], d);
    r.hi[a] = __shfl_down_sync(0xFFFFFFFFu, b.hi[a], d);
  }
  return r;
}
// Inclusive prefix (lanes 0..i) and suffix (lanes i..31) unions of a warp's
// boxes; unions are exact, so any order gives the host's boxes.
__device__ __forceinline__ Bx warpPrefix(Bx b) {
  const int lane = threadIdx.x & 31;
  for (int d = 1; d < 32; d <<= 1) {
    Bx o = bxShflUp(b, d);
    if (lane >= d) bxGrow(b, o);
  }
  return b;
}
__device__ __forceinline__ Bx warpSuffix(Bx b) {
  const int lane = threadIdx.x & 31;
  for (int d = 1; d < 32; d <<= 1) {
    Bx o = bxShflDown(b, d);
    if (lane + d < 32) bxGrow(b, o);
  }
  return b;
}
__device__ __forceinline__ int warpPrefixSum(int v) {
  const int lane = threadIdx.x & 31;
  for (int d = 1; d < 32; d <<= 1) {
    int o = __shfl_up_sync(0xFFFFFFFFu, v, d);
    if (lane >= d) v += o;
  }
  return v;
}
__device__ __forceinline__ int warpSuffixSum(int v) {
  const int lane = threadIdx.x & 31;
  for (int d = 1; d < 32; d <<= 1) {
    int o = __shfl_down_sync(0xFFFFFFFFu, v, d);
    if (lane + d < 32) v += o;
  }
  return v;
}

// Lowest (cost, key) over the warp; ties go to the smaller key, as the host
// keeps the first strictly smaller cost in its loop order.
__device__ __forceinline__ void warpArgmin(float& cost, int& key) {
  for (int d = 16; d > 0; d >>= 1) {
    float oc = __shfl_xor_sync(0xFFFFFFFFu, cost, d);
    int ok = __shfl_xor_sync(0xFFFFFFFFu, key, d);
    if (oc < cost || (oc == cost && ok < key)) {
      cost = oc;
      key = ok;
    }
  }
}

__device__ __forceinline__ Bx primBox(const BuildCtx& c, int id) {
  float4 l = c.lo[id], h = c.hi[id];
  Bx b;
  b.lo[0] = l.x;
  b.lo[1] = l.y;
  b.lo[2] = l.z;
  b.hi[0] = h.x;
  b.hi[1] = h.y;
  b.hi[2] = h.z;
  return b;
}
__device__ __forceinline__ float centAxis(const BuildCtx& c, int id, int ax) {
  float4 v = c.cent[id];
  return ax == 0 ? v.x : (ax == 1 ? v.y : v.z);
}

__device__ __forceinline__ void setLink(const BuildCtx& c, int parentSlot, int link) {
  if (parentSlot >= 0) reinterpret_cast<int*>(c.nodes)[parentSlot] = link;
}

__device__ __forceinline__ int leafLink(const BuildCtx& c, int b, int n) {
  return ~(((c.primBase + b) << 3) | (n - 1));
}

// Allocates the node of a range that splits into [b, m) and [m, e) and
// appends the child ranges; one thread.
__device__ void emitNode(const BuildCtx& c, const BuildRange& r, int m, const Bx& lb, const Bx& rb,
                         BuildRange* out, int* nOut) {
  const int idx = atomicAdd(c.nodeCount, 1);
  const int k = atomicAdd(nOut, 2);
  // A binary tree over n primitives has at most n - 1 inner nodes and every
  // level at most n ranges; past either bound the build is wrong: flag it.
  if (idx >= c.nodeCap || k + 2 > c.rangeCap) {
    atomicExch(c.error, 1);
    return;
  }
  BvhNode nd;
  nd.xy0 = make_float4(lb.lo[0], lb.hi[0], lb.lo[1], lb.hi[1]);
  nd.xy1 = make_float4(rb.lo[0], rb.hi[0], rb.lo[1], rb.hi[1]);
  nd.zz = make_float4(lb.lo[2], lb.hi[2], rb.lo[2], rb.hi[2]);
  nd.link = make_int4(0, 0, 0, 0);
  c.nodes[idx] = nd;
  setLink(c, r.parentSlot, c.nodeBase + idx);
  BuildRange L, R;
  L.b = r.b;
  L.e = m;
  R.b = m;
  R.e = r.e;
  L.depth = R.depth = r.depth + 1;
  L.parentSlot = idx * 16 + 12;
  R.parentSlot = idx * 16 + 13;
  for (int a = 0; a < 3; a++) {
    L.lo[a] = lb.lo[a];
    L.hi[a] = lb.hi[a];
    R.lo[a] = rb.lo[a];
    R.hi[a] = rb.hi[a];
  }
  out[k] = L;
  out[k + 1] = R;
  atomicMax(c.maxDepth, r.depth + 1);
}

__global__ void __launch_bounds__(kBuildThreads) bvhLevel(BuildCtx c, const BuildRange* in,
                                                          BuildRange* out, int* nOut,
                                                          const int* idsIn, int* idsOut) {
  __shared__ int sMin[3], sMax[3];
  __shared__ int binCnt[3][kBuildBins];
  __shared__ int binLo[3][kBuildBins][3], binHi[3][kBuildBins][3];
  __shared__ int decision[4];  // kind (0 leaf, 1 binned split, 2 middle split), axis, bin, left count
  __shared__ float splitBox[2][6];
  __shared__ int warpCnt[kBuildThreads / 32];
  const BuildRange r = in[blockIdx.x];
  const int n = r.e - r.b;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  Bx nb;
  for (int a = 0; a < 3; a++) {
    nb.lo[a] = r.lo[a];
    nb.hi[a] = r.hi[a];
  }
  const float leafCost = __fmul_rn(bxArea(nb), (float)n);

  // ---- ranges of up to 32: one warp, exact sweep over sorted centroids ----
  if (n <= kBuildSmall) {
    if (warp != 0) return;
    const bool live = lane < n;
    const int myId = live ? idsIn[r.b + lane] : -1;
    float cl[3], ch[3];
    for (int a = 0; a < 3; a++) {
      float v = live ? centAxis(c, myId, a) : 0.0f;
      float lo = live ? v : FLT_MAX, hi = live ? v : -FLT_MAX;
      for (int d = 16; d > 0; d >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, d));
        hi = fmaxf(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, d));
      }
      cl[a] = lo;
      ch[a] = hi;
    }
    float bestCost = FLT_MAX;
    int bestKey = 0x7FFFFFFF;  // axis * 64 + position
    const bool forceMiddle = r.depth >= kBuildDepthLimit;
    // Sorted order per axis: rank of this lane's primitive by (centroid, lane).
    // (Integer keys: a total order even with NaN centroids, so the ranks
    // are a permutation of 0..31 and every position is written once.)
    auto rankOn = [&](int ax) {
      int v = live ? fkey(centAxis(c, myId, ax)) : 0x7FFFFFFF;
      int rank = 0;
      for (int j = 0; j < 32; j++) {
        int o = __shfl_sync(0xFFFFFFFFu, v, j);
        rank += (o < v || (o == v && j < lane)) ? 1 : 0;
      }
      return rank;
    };
    if (n > 1 && !forceMiddle) {
      for (int ax = 0; ax < 3; ax++) {
        if (!(__fsub_rn(ch[ax], cl[ax]) > 0.0f)) continue;
        const int rank = rankOn(ax);
        // Lane p holds the box of the primitive at sorted position p.
        int src = 0;
        for (int j = 0; j < 32; j++) {
          int rj = __shfl_sync(0xFFFFFFFFu, rank, j);
          if (rj == lane) src = j;
        }
        Bx mine = live ? primBox(c, myId) : bxEmpty();
        Bx atPos = bxShfl(mine, src);
        if (lane >= n) atPos = bxEmpty();
        Bx pre = warpPrefix(atPos), suf = warpSuffix(atPos);
        Bx left = bxShflUp(pre, 1);  // union of positions < lane
        float cost = FLT_MAX;
        int key = 0x7FFFFFFF;
        if (lane >= 1 && lane < n) {
          cost = __fadd_rn(__fmul_rn(bxArea(left), (float)lane),
                           __fmul_rn(bxArea(suf), (float)(n - lane)));
          key = ax * 64 + lane;
        }
        warpArgmin(cost, key);
        if (cost < bestCost || (cost == bestCost && key < bestKey)) {
          bestCost = cost;
          bestKey = key;
        }
      }
    }
    const bool haveSplit = bestKey != 0x7FFFFFFF;
    bool leaf = n == 1;
    if (!leaf && haveSplit && n <= c.maxLeaf &&
        leafCost <= __fadd_rn(bestCost, __fmul_rn(1.2f, bxArea(nb))))
      leaf = true;
    if (!leaf && !haveSplit && n <= c.maxLeaf) leaf = true;
    if (leaf) {
      if (live) c.order[r.b + lane] = myId;
      if (lane == 0) {
        setLink(c, r.parentSlot, leafLink(c, r.b, n));
        atomicMax(c.maxDepth, r.depth);
      }
      return;
    }
    int m, ax;
    if (haveSplit) {
      ax = bestKey / 64;
      m = bestKey % 64;
    } else {  // coincident centroids or the depth limit: middle of the widest axis
      float ex = ch[0] - cl[0], ey = ch[1] - cl[1], ez = ch[2] - cl[2];
      ax = ex >= ey && ex >= ez ? 0 : (ey >= ez ? 1 : 2);
      m = n / 2;
    }
    const int rank = rankOn(ax);
    if (live) idsOut[r.b + rank] = myId;
    // Child boxes from the sorted order.
    int src = 0;
    for (int j = 0; j < 32; j++) {
      int rj = __shfl_sync(0xFFFFFFFFu, rank, j);
      if (rj == lane) src = j;
    }
    Bx mine = live ? primBox(c, myId) : bxEmpty();
    Bx atPos = bxShfl(mine, src);
    if (lane >= n) atPos = bxEmpty();
    Bx pre = warpPrefix(atPos), suf = warpSuffix(atPos);
    Bx lb = bxShfl(pre, m - 1), rb = bxShfl(suf, m);
    if (lane == 0) emitNode(c, r, r.b + m, lb, rb, out, nOut);
    return;
  }

  // ---- larger ranges: binned SAH over all three axes in one pass ----
  if (tid < 3) {
    sMin[tid] = fkey(FLT_MAX);
    sMax[tid] = fkey(-FLT_MAX);
  }
  for (int i = tid; i < 3 * kBuildBins; i += kBuildThreads) {
    (&binCnt[0][0])[i] = 0;
    for (int a = 0; a < 3; a++) {
      binLo[i / kBuildBins][i % kBuildBins][a] = fkey(FLT_MAX);
      binHi[i / kBuildBins][i % kBuildBins][a] = fkey(-FLT_MAX);
    }
  }
  __syncthreads();
  for (int i = r.b + tid; i < r.e; i += kBuildThreads) {
    float4 v = c.cent[idsIn[i]];
    atomicMin(&sMin[0], fkey(v.x));
    atomicMin(&sMin[1], fkey(v.y));
    atomicMin(&sMin[2], fkey(v.z));
    atomicMax(&sMax[0], fkey(v.x));
    atomicMax(&sMax[1], fkey(v.y));
    atomicMax(&sMax[2], fkey(v.z));
  }
  __syncthreads();
  float lo[3], sc[3];
  bool on[3];
  for (int a = 0; a < 3; a++) {
    lo[a] = fdec(sMin[a]);
    float ext = __fsub_rn(fdec(sMax[a]), lo[a]);
    on[a] = ext > 0.0f;
    sc[a] = on[a] ? __fdiv_rn((float)kBuildBins, ext) : 0.0f;
  }
  const bool forceMiddle = r.depth >= kBuildDepthLimit;
  if (!forceMiddle) {
    for (int i = r.b + tid; i < r.e; i += kBuildThreads) {
      const int id = idsIn[i];
      const float4 v = c.cent[id];
      const Bx bx = primBox(c, id);
      for (int a = 0; a < 3; a++) {
        if (!on[a]) continue;
        float cv = a == 0 ? v.x : (a == 1 ? v.y : v.z);
        int k = (int)__fmul_rn(__fsub_rn(cv, lo[a]), sc[a]);
        k = min(max(k, 0), kBuildBins - 1);
        atomicAdd(&binCnt[a][k], 1);
        for (int q = 0; q < 3; q++) {
          atomicMin(&binLo[a][k][q], fkey(bx.lo[q]));
          atomicMax(&binHi[a][k][q], fkey(bx.hi[q]));
        }
      }
    }
  }
  __syncthreads();
  if (warp == 0) {
    float bestCost = FLT_MAX;
    int bestKey = 0x7FFFFFFF;  // axis * 64 + bin
    Bx bestL = bxEmpty(), bestR = bxEmpty();
    int bestLeftN = 0;
    for (int a = 0; a < 3 && !forceMiddle; a++) {
      if (!on[a]) continue;
      Bx bb;
      for (int q = 0; q < 3; q++) {
        bb.lo[q] = fdec(binLo[a][lane][q]);
        bb.hi[q] = fdec(binHi[a][lane][q]);
      }
      const int cnt = binCnt[a][lane];
      Bx pre = warpPrefix(bb), suf = warpSuffix(bb);
      int preN = warpPrefixSum(cnt), sufN = warpSuffixSum(cnt);
      Bx right = bxShflDown(suf, 1);  // bins > lane
      int rightN = __shfl_down_sync(0xFFFFFFFFu, sufN, 1);
      float cost = FLT_MAX;
      int key = 0x7FFFFFFF;
      if (lane < kBuildBins - 1 && preN > 0 && rightN > 0) {
        cost = __fadd_rn(__fmul_rn(bxArea(pre), (float)preN), __fmul_rn(bxArea(right), (float)rightN));
        key = a * 64 + lane;
      }
      float wc = cost;
      int wk = key;
      warpArgmin(wc, wk);
      if (wc < bestCost || (wc == bestCost && wk < bestKey)) {
        bestCost = wc;
        bestKey = wk;
        const int at = wk % 64;
        bestL = bxShfl(pre, at);
        bestR = bxShfl(right, at);
        bestLeftN = __shfl_sync(0xFFFFFFFFu, preN, at);
      }
    }
    if (lane == 0) {
      const bool haveSplit = bestKey != 0x7FFFFFFF;
      int kind = haveSplit ? 1 : 2;
      if (haveSplit && n <= c.maxLeaf &&
          leafCost <= __fadd_rn(bestCost, __fmul_rn(1.2f, bxArea(nb))))
        kind = 0;
      if (!haveSplit && n <= c.maxLeaf) kind = 0;
      decision[0] = kind;
      decision[1] = haveSplit ? bestKey / 64 : 0;
      decision[2] = haveSplit ? bestKey % 64 : 0;
      decision[3] = haveSplit ? bestLeftN : n / 2;
      for (int q = 0; q < 3; q++) {
        splitBox[0][q] = bestL.lo[q];
        splitBox[0][3 + q] = bestL.hi[q];
        splitBox[1][q] = bestR.lo[q];
        splitBox[1][3 + q] = bestR.hi[q];
      }
    }
  }
  __syncthreads();
  const int kind = decision[0];
  if (kind == 0) {
    for (int i = r.b + tid; i < r.e; i += kBuildThreads) c.order[i] = idsIn[i];
    if (tid == 0) {
      setLink(c, r.parentSlot, leafLink(c, r.b, n));
      atomicMax(c.maxDepth, r.depth);
    }
    return;
  }
  const int nLeft = decision[3];
  if (kind == 1) {
    // Stable partition by bin <= split bin on the chosen axis.
    const int ax = decision[1], bin = decision[2];
    int leftBase = 0, rightBase = 0;
    for (int base = r.b; base < r.e; base += kBuildThreads) {
      const int i = base + tid;
      int id = -1;
      bool goLeft = false;
      if (i < r.e) {
        id = idsIn[i];
        int k = (int)__fmul_rn(__fsub_rn(centAxis(c, id, ax), lo[ax]), sc[ax]);
        k = min(max(k, 0), kBuildBins - 1);
        goLeft = k <= bin;
      }
      const unsigned bl = __ballot_sync(0xFFFFFFFFu, goLeft);
      const unsigned br = __ballot_sync(0xFFFFFFFFu, i < r.e && !goLeft);
      if (lane == 0) warpCnt[warp] = __popc(bl) | (__popc(br) << 16);
      __syncthreads();
      int offL = 0, offR = 0, totL = 0, totR = 0;
      for (int w = 0; w < kBuildThreads / 32; w++) {
        const int cL = warpCnt[w] & 0xFFFF, cR = warpCnt[w] >> 16;
        if (w < warp) {
          offL += cL;
          offR += cR;
        }
        totL += cL;
        totR += cR;
      }
      const unsigned lt = (1u << lane) - 1u;
      if (i < r.e) {
        // The bin counts and this test use the same arithmetic, so exactly
        // nLeft primitives go left; the bound check only guards the buffer.
        const int pos = goLeft ? r.b + leftBase + offL + __popc(bl & lt)
                               : r.b + nLeft + rightBase + offR + __popc(br & lt);
        if (pos >= r.b && pos < r.e)
          idsOut[pos] = id;
        else
          atomicExch(c.error, 1);
      }
      leftBase += totL;
      rightBase += totR;
      __syncthreads();
    }
    if (tid == 0) {
      Bx lb, rb;
      for (int q = 0; q < 3; q++) {
        lb.lo[q] = splitBox[0][q];
        lb.hi[q] = splitBox[0][3 + q];
        rb.lo[q] = splitBox[1][q];
        rb.hi[q] = splitBox[1][3 + q];
      }
      emitNode(c, r, r.b + nLeft, lb, rb, out, nOut);
    }
    return;
  }
  // kind 2: coincident centroids (or the depth limit): split at the middle in
  // the current order, boxes by reduction.
  for (int i = r.b + tid; i < r.e; i += kBuildThreads) idsOut[i] = idsIn[i];
  __syncthreads();
  if (tid < 12) {
    // reuse the bin bounds as two reduction slots
    (&binLo[0][0][0])[tid] = fkey(FLT_MAX);
    (&binHi[0][0][0])[tid] = fkey(-FLT_MAX);
  }
  __syncthreads();
  for (int i = r.b + tid; i < r.e; i += kBuildThreads) {
    const int side = i - r.b < nLeft ? 0 : 1;
    const Bx bx = primBox(c, idsIn[i]);
    for (int q = 0; q < 3; q++) {
      atomicMin(&binLo[0][side][q], fkey(bx.lo[q]));
      atomicMax(&binHi[0][side][q], fkey(bx.hi[q]));
    }
  }
  __syncthreads();
  if (tid == 0) {
    Bx lb, rb;
    for (int q = 0; q < 3; q++) {
      lb.lo[q] = fdec(binLo[0][0][q]);
      lb.hi[q] = fdec(binHi[0][0][q]);
      rb.lo[q] = fdec(binLo[0][1][q]);
      rb.hi[q] = fdec(binHi[0][1][q]);
    }
    emitNode(c, r, r.b + nLeft, lb, rb, out, nOut);
  }
}

// Root range: the union of all primitive boxes; identity order.
__global__ void __launch_bounds__(kBuildThreads) bvhRoot(const float4* lo, const float4* hi, int n,
                                                         int* ids, BuildRange* root) {
  __shared__ int s[6];
  if (threadIdx.x < 3) {
    s[threadIdx.x] = fkey(FLT_MAX);
    s[3 + threadIdx.x] = fkey(-FLT_MAX);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    ids[i] = i;
    float4 l = lo[i], h = hi[i];
    atomicMin(&s[0], fkey(l.x));
    atomicMin(&s[1], fkey(l.y));
    atomicMin(&s[2], fkey(l.z));
    atomicMax(&s[3], fkey(h.x));
    atomicMax(&s[4], fkey(h.y));
    atomicMax(&s[5], fkey(h.z));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    BuildRange r;
    r.b = 0;
    r.e = n;
    r.depth = 0;
    r.parentSlot = -1;
    for (int a = 0; a < 3; a++) {
      r.lo[a] = fdec(s[a]);
      r.hi[a] = fdec(s[3 + a]);
    }
    *root = r;
  }
}

// Triangle boxes and centroids of a mesh (object space).
__global__ void triBoxes(const float3* __restrict__ pos, const uint3* __restrict__ idx, int n,
                         float4* lo, float4* hi, float4* cent) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    uint3 i = idx[t];
    float3 a = pos[i.x], b = pos[i.y], c = pos[i.z];
    float3 l = make_float3(fminf(a.x, fminf(b.x, c.x)), fminf(a.y, fminf(b.y, c.y)),
                           fminf(a.z, fminf(b.z, c.z)));
    float3 h = make_float3(fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y)),
                           fmaxf(a.z, fmaxf(b.z, c.z)));
    lo[t] = make_float4(l.x, l.y, l.z, 0.0f);
    hi[t] = make_float4(h.x, h.y, h.z, 0.0f);
    cent[t] = make_float4(__fmul_rn(__fadd_rn(l.x, h.x), 0.5f), __fmul_rn(__fadd_rn(l.y, h.y), 0.5f),
                          __fmul_rn(__fadd_rn(l.z, h.z), 0.5f), 0.0f);
  }
}

// Triangles in leaf order: 3 float4 each, .w of the first = mesh-local index.
__global__ void gatherTris(const float3* __restrict__ pos, const uint3* __restrict__ idx,
                           const int* __restrict__ order, int n, float4* tris) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int t = order[k];
    uint3 i = idx[t];
    float3 a = pos[i.x], b = pos[i.y], c = pos[i.z];
    tris[3 * (size_t)k + 0] = make_float4(a.x, a.y, a.z, __int_as_float(t));
    tris[3 * (size_t)k + 1] = make_float4(b.x, b.y, b.z, 0.0f);
    tris[3 * (size_t)k + 2] = make_float4(c.x, c.y, c.z, 0.0f);
  }
}

// p -> xf p in the host's FP32 order ((m0 x + m1 y) + m2 z) + m3.
__device__ __forceinline__ float3 xfPointRn(const float* m, float3 p) {
  return make_float3(
      __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], p.x), __fmul_rn(m[1], p.y)), __fmul_rn(m[2], p.z)), m[3]),
      __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[4], p.x), __fmul_rn(m[5], p.y)), __fmul_rn(m[6], p.z)), m[7]),
      __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[8], p.x), __fmul_rn(m[9], p.y)), __fmul_rn(m[10], p.z)), m[11]));
}

// World box of each instance: every vertex of its mesh (or the 8 corners of
// its quadric's canonical bounds) transformed, then padded by a few ulps.
__global__ void __launch_bounds__(kBuildThreads) instanceBoxes(const DevInstanceSrc* __restrict__ src,
                                                               int n, float4* lo, float4* hi,
                                                               float4* cent) {
  __shared__ int s[6];
  const int i = blockIdx.x;
  if (i >= n) return;
  const DevInstanceSrc& in = src[i];
  if (threadIdx.x < 3) {
    s[threadIdx.x] = fkey(FLT_MAX);
    s[3 + threadIdx.x] = fkey(-FLT_MAX);
  }
  __syncthreads();
  const int count = in.pos ? in.numVerts : 8;
  for (int k = threadIdx.x; k < count; k += blockDim.x) {
    float3 p;
    if (in.pos) {
      p = in.pos[k];
    } else {
      p = make_float3(k & 1 ? in.qhi.x : in.qlo.x, k & 2 ? in.qhi.y : in.qlo.y,
                      k & 4 ? in.qhi.z : in.qlo.z);
    }
    float3 w = xfPointRn(in.xf, p);
    atomicMin(&s[0], fkey(w.x));
    atomicMin(&s[1], fkey(w.y));
    atomicMin(&s[2], fkey(w.z));
    atomicMax(&s[3], fkey(w.x));
    atomicMax(&s[4], fkey(w.y));
    atomicMax(&s[5], fkey(w.z));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float l[3], h[3], pad[3];
    for (int a = 0; a < 3; a++) {
      l[a] = fdec(s[a]);
      h[a] = fdec(s[3 + a]);
      float m = fmaxf(fmaxf(h[a], -h[a]), fmaxf(l[a], -l[a]));
      pad[a] = __fmul_rn(__fadd_rn(m, 1.0f), 1e-6f);
      l[a] = __fsub_rn(l[a], pad[a]);
      h[a] = __fadd_rn(h[a], pad[a]);
    }
    lo[i] = make_float4(l[0], l[1], l[2], 0.0f);
    hi[i] = make_float4(h[0], h[1], h[2], 0.0f);
    cent[i] = make_float4(__fmul_rn(__fadd_rn(l[0], h[0]), 0.5f), __fmul_rn(__fadd_rn(l[1], h[1]), 0.5f),
                          __fmul_rn(__fadd_rn(l[2], h[2]), 0.5f), 0.0f);
  }
}

int launchGrid(int n) { return std::max(1, std::min((n + 255) / 256, 148 * 8)); }

}  // namespace

DevBvhStats buildBvhDevice(const float4* lo, const float4* hi, const float4* cent, int n,
                           int maxLeaf, int nodeBase, int primBase, BvhNode* nodes, int nodeCap,
                           int* order, cudaStream_t st) {
  DevBvhStats stats;
  if (maxLeaf < 1 || maxLeaf > 8) throw std::runtime_error("device BVH: maxLeaf must be 1..8");
  if (n <= maxLeaf) throw std::runtime_error("device BVH: a range this small is one leaf");
  if ((long long)primBase + n >= (1ll << 28)) throw std::runtime_error("device BVH: too many primitives");
  if (nodeCap < n - 1) throw std::runtime_error("device BVH: node array too small");
  DevBuf ids0, ids1, ranges0, ranges1, counters;
  ids0.alloc((size_t)n * sizeof(int));
  ids1.alloc((size_t)n * sizeof(int));
  ranges0.alloc((size_t)n * sizeof(BuildRange));
  ranges1.alloc((size_t)n * sizeof(BuildRange));
  counters.alloc(4 * sizeof(int));
  cudaCheck(cudaMemsetAsync(counters.ptr, 0, counters.bytes, st), "device BVH counters");
  int* cnt = (int*)counters.ptr;  // [0] nodes, [1] max depth, [2] next ranges, [3] error
  bvhRoot<<<1, kBuildThreads, 0, st>>>(lo, hi, n, (int*)ids0.ptr, (BuildRange*)ranges0.ptr);
  cudaCheck(cudaGetLastError(), "device BVH root");
  BuildCtx c;
  c.lo = lo;
  c.hi = hi;
  c.cent = cent;
  c.nodes = nodes;
  c.nodeCount = cnt;
  c.order = order;
  c.maxDepth = cnt + 1;
  c.error = cnt + 3;
  c.maxLeaf = maxLeaf;
  c.nodeBase = nodeBase;
  c.primBase = primBase;
  c.nodeCap = nodeCap;
  c.rangeCap = n;
  int* pinned = reinterpret_cast<int*>(pinnedWords());
  try {
    int nIn = 1;
    void* idsIn = ids0.ptr;
    void* idsOut = ids1.ptr;
    void* rIn = ranges0.ptr;
    void* rOut = ranges1.ptr;
    for (int level = 0; nIn > 0; level++) {
      if (level > 4096) throw std::runtime_error("device BVH: no progress");
      cudaCheck(cudaMemsetAsync(cnt + 2, 0, sizeof(int), st), "device BVH counters");
      bvhLevel<<<nIn, kBuildThreads, 0, st>>>(c, (const BuildRange*)rIn, (BuildRange*)rOut,
                                              cnt + 2, (const int*)idsIn, (int*)idsOut);
      cudaCheck(cudaGetLastError(), "device BVH level");
      cudaCheck(cudaMemcpyAsync(pinned, cnt, 4 * sizeof(int), cudaMemcpyDeviceToHost, st),
                "device BVH count");
      cudaCheck(cudaStreamSynchronize(st), "device BVH level");
      if (pinned[3]) throw std::runtime_error("device BVH: capacity bound exceeded");
      nIn = pinned[2];
      std::swap(idsIn, idsOut);
      std::swap(rIn, rOut);
      stats.levels = level + 1;
    }
    stats.nodes = pinned[0];
    stats.maxDepth = pinned[1];
  } catch (...) {
    returnPinnedWords(reinterpret_cast<unsigned*>(pinned));
    throw;
  }
  returnPinnedWords(reinterpret_cast<unsigned*>(pinned));
  return stats;
}

void meshBoxesDevice(const float3* pos, const uint3* idx, int n, float4* lo, float4* hi,
                     float4* cent, cudaStream_t st) {
  triBoxes<<<launchGrid(n), 256, 0, st>>>(pos, idx, n, lo, hi, cent);
  cudaCheck(cudaGetLastError(), "triangle boxes");
}

void gatherTrisDevice(const float3* pos, const uint3* idx, const int* order, int n, float4* tris,
                      cudaStream_t st) {
  gatherTris<<<launchGrid(n), 256, 0, st>>>(pos, idx, order, n, tris);
  cudaCheck(cudaGetLastError(), "triangle gather");
}

void instanceBoxesDevice(const DevInstanceSrc* src, int n, float4* lo, float4* hi, float4* cent,
                         cudaStream_t st) {
  instanceBoxes<<<n, kBuildThreads, 0, st>>>(src, n, lo, hi, cent);
  cudaCheck(cudaGetLastError(), "instance boxes");
}

// ---- 4-wide collapse ------------------------------------------------------

namespace {

struct Collapse4Item {
  int bin;  // binary node
  int q;    // its 4-wide node
};

struct Collapse4Ctx {
  const BvhNode* bin;
  int numBin;
  Bvh4Node* out;
  int* qCount;     // 4-wide nodes allocated
  int* nextCount;  // items of the next level
  int* error;      // a link outside the binary array, or capacity exceeded
  int qCap;
};

// Child `side` of a binary node: its box and link.
__device__ __forceinline__ void binChild(const BvhNode& n, int side, float3& lo, float3& hi,
                                         int& link) {
  if (side == 0) {
    lo = make_float3(n.xy0.x, n.xy0.z, n.zz.x);
    hi = make_float3(n.xy0.y, n.xy0.w, n.zz.y);
    link = n.link.x;
  } else {
    lo = make_float3(n.xy1.x, n.xy1.z, n.zz.z);
    hi = make_float3(n.xy1.y, n.xy1.w, n.zz.w);
    link = n.link.y;
  }
}

__device__ __forceinline__ void setSlot(Bvh4Node& q, int k, float3 lo, float3 hi, int link) {
  float4& xy = k == 0 ? q.xy0 : k == 1 ? q.xy1 : k == 2 ? q.xy2 : q.xy3;
  float4& zz = k < 2 ? q.zz01 : q.zz23;
  xy = make_float4(lo.x, hi.x, lo.y, hi.y);
  if (k & 1) {
    zz.z = lo.z;
    zz.w = hi.z;
  } else {
    zz.x = lo.z;
    zz.y = hi.z;
  }
  reinterpret_cast<int*>(&q.link)[k] = link;
}

// One thread per 4-wide node of the level: the binary node's children, each
// leaf child kept as it is and each inner child replaced by its own two
// children; inner grandchildren get 4-wide nodes of their own (next level).
__global__ void collapse4Level(Collapse4Ctx c, const Collapse4Item* in, int nIn,
                               Collapse4Item* next) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nIn) return;
  const Collapse4Item it = in[i];
  const BvhNode n = c.bin[it.bin];
  Bvh4Node q;
  const float3 far = make_float3(3e30f, 3e30f, 3e30f);
  for (int k = 0; k < 4; k++) setSlot(q, k, far, far, ~0);
  q.pad = make_int4(0, 0, 0, 0);
  int k = 0;
  for (int side = 0; side < 2; side++) {
    float3 lo, hi;
    int link;
    binChild(n, side, lo, hi, link);
    if (link < 0) {
      setSlot(q, k++, lo, hi, link);
      continue;
    }
    if (link >= c.numBin) {
      atomicExch(c.error, 1);
      return;
    }
    const BvhNode m = c.bin[link];
    for (int s2 = 0; s2 < 2; s2++) {
      float3 glo, ghi;
      int g;
      binChild(m, s2, glo, ghi, g);
      if (g >= 0) {
        if (g >= c.numBin) {
          atomicExch(c.error, 1);
          return;
        }
        const int qi = atomicAdd(c.qCount, 1);
        if (qi >= c.qCap) {
          atomicExch(c.error, 1);
          return;
        }
        next[atomicAdd(c.nextCount, 1)] = Collapse4Item{g, qi};
        g = qi;
      }
      setSlot(q, k++, glo, ghi, g);
    }
  }
  c.out[it.q] = q;
}

}  // namespace

int collapseBvh4Device(const BvhNode* bin, int numBin, const int* roots, int numRoots,
                       Bvh4Node* out, int* outRoots, cudaStream_t st) {
  if (numRoots < 1 || numRoots > numBin)
    throw std::runtime_error("4-wide collapse: bad root count");
  DevBuf items0, items1, counters;
  items0.alloc((size_t)numBin * sizeof(Collapse4Item));
  items1.alloc((size_t)numBin * sizeof(Collapse4Item));
  counters.alloc(4 * sizeof(int));
  std::vector<Collapse4Item> first(numRoots);
  for (int r = 0; r < numRoots; r++) {
    if (roots[r] < 0 || roots[r] >= numBin)
      throw std::runtime_error("4-wide collapse: root outside the node array");
    first[r] = Collapse4Item{roots[r], r};
    outRoots[r] = r;
  }
  cudaCheck(cudaMemcpyAsync(items0.ptr, first.data(), first.size() * sizeof(Collapse4Item),
                            cudaMemcpyHostToDevice, st),
            "4-wide collapse roots");
  int* cnt = (int*)counters.ptr;  // [0] nodes, [1] next items, [2] error
  int init[4] = {numRoots, 0, 0, 0};
  cudaCheck(cudaMemcpyAsync(cnt, init, sizeof init, cudaMemcpyHostToDevice, st),
            "4-wide collapse counters");
  Collapse4Ctx c;
  c.bin = bin;
  c.numBin = numBin;
  c.out = out;
  c.qCount = cnt;
  c.nextCount = cnt + 1;
  c.error = cnt + 2;
  c.qCap = numBin;
  int host[4] = {0, 0, 0, 0};
  int nIn = numRoots;
  void* in = items0.ptr;
  void* nx = items1.ptr;
  for (int level = 0; nIn > 0; level++) {
    if (level > 4096) throw std::runtime_error("4-wide collapse: no progress");
    cudaCheck(cudaMemsetAsync(cnt + 1, 0, sizeof(int), st), "4-wide collapse counters");
    collapse4Level<<<(nIn + 127) / 128, 128, 0, st>>>(c, (const Collapse4Item*)in, nIn,
                                                      (Collapse4Item*)nx);
    cudaCheck(cudaGetLastError(), "4-wide collapse level");
    cudaCheck(cudaMemcpyAsync(host, cnt, sizeof host, cudaMemcpyDeviceToHost, st),
              "4-wide collapse count");
    cudaCheck(cudaStreamSynchronize(st), "4-wide collapse level");
    if (host[2]) throw std::runtime_error("4-wide collapse: malformed tree or capacity exceeded");
    nIn = host[1];
    std::swap(in, nx);
  }
  return host[0];
}

}  // namespace sdb
