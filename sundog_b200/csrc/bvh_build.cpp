// Binned SAH build (Wald, "On fast Construction of SAH-based Bounding Volume
// Hierarchies", 2007): 32 bins per axis over centroid bounds, all three axes
// binned in one pass, ranges of up to 32 primitives split exactly over their
// sorted centroids, leaf when splitting costs more than intersecting; from the
// depth limit of 40 on, median splits guarantee termination. The scene build
// checks TLAS + BLAS depth against the traversal stack (kTraversalStack).
#include "bvh_build.h"

#include <algorithm>
#include <cfloat>
#include <future>
#include <cmath>
#include <cstring>

namespace sdb {

// Plain comparisons rather than fminf / fmaxf, which the host compiler
// calls out of line (NaN rules) at this optimisation level: the builder's
// bounds are finite.
static inline float minOf(float a, float b) { return b < a ? b : a; }
static inline float maxOf(float a, float b) { return b > a ? b : a; }

Box3 boxEmpty() { return {v3(FLT_MAX), v3(-FLT_MAX)}; }
void boxGrow(Box3& b, float3 p) {
  b.lo = v3(minOf(b.lo.x, p.x), minOf(b.lo.y, p.y), minOf(b.lo.z, p.z));
  b.hi = v3(maxOf(b.hi.x, p.x), maxOf(b.hi.y, p.y), maxOf(b.hi.z, p.z));
}
void boxGrow(Box3& b, const Box3& o) {
  b.lo = v3(minOf(b.lo.x, o.lo.x), minOf(b.lo.y, o.lo.y), minOf(b.lo.z, o.lo.z));
  b.hi = v3(maxOf(b.hi.x, o.hi.x), maxOf(b.hi.y, o.hi.y), maxOf(b.hi.z, o.hi.z));
}
static float boxArea(const Box3& b) {
  float3 e = b.hi - b.lo;
  if (e.x < 0.0f) return 0.0f;
  return 2.0f * (e.x * e.y + e.y * e.z + e.z * e.x);
}

namespace {

constexpr int kBins = 32;
constexpr int kSmall = 32;  // ranges up to this size are split exactly
constexpr int kDepthLimit = 40;

// Subtrees of at least kParallelMin primitives down to depth kParallelDepth
// build their right half on another thread; the halves own disjoint ranges
// of `ids`, and the right half's nodes are appended after the left's with
// their links relocated, so the tree is the one the sequential build makes.
constexpr int kParallelMin = 1024;
constexpr int kParallelDepth = 3;

// Primitive centroids and the primitive order, shared by a build's threads.
struct BuildInput {
  std::vector<float3> cent;
  std::vector<int> ids;
  explicit BuildInput(const std::vector<Box3>& b) : cent(b.size()), ids(b.size()) {
    for (size_t i = 0; i < b.size(); i++) {
      cent[i] = (b[i].lo + b[i].hi) * 0.5f;
      ids[i] = (int)i;
    }
  }
};

struct Builder {
  const std::vector<Box3>& boxes;
  const std::vector<float3>& cent;
  std::vector<int>& ids;
  int maxLeaf, nodeBase, primBase;
  bool parallel;
  BvhBuild out;

  Builder(const std::vector<Box3>& b, BuildInput& in, int ml, int nb, int pb, bool par)
      : boxes(b), cent(in.cent), ids(in.ids), maxLeaf(ml), nodeBase(nb), primBase(pb),
        parallel(par) {}
  // A builder for a subtree of the same build, numbering its nodes from nb.
  Builder(const Builder& o, int nb)
      : boxes(o.boxes), cent(o.cent), ids(o.ids), maxLeaf(o.maxLeaf), nodeBase(nb),
        primBase(o.primBase), parallel(o.parallel) {}

  Box3 rangeBox(int b, int e) const {
    Box3 r = boxEmpty();
    for (int i = b; i < e; i++) boxGrow(r, boxes[ids[i]]);
    return r;
  }

  int leafLink(int b, int e) const {
    int code = ((primBase + b) << 3) | (e - b - 1);
    return ~code;
  }

  // Sorts ids[b, e) by centroid along ax (insertion sort: small ranges only;
  // ties keep their order, so the result is deterministic).
  void sortSmall(int b, int e, int ax) {
    for (int i = b + 1; i < e; i++) {
      int id = ids[i];
      float key = comp(cent[id], ax);
      int j = i - 1;
      while (j >= b && comp(cent[ids[j]], ax) > key) {
        ids[j + 1] = ids[j];
        j--;
      }
      ids[j + 1] = id;
    }
  }

  // Best SAH split of a small range: every position along each axis's
  // centroid order. Returns the cost; ax / pos the split (pos = primitives
  // on the left), ax = -1 if no axis has extent.
  float exactSweep(int b, int e, const float3& ext, int& bestAx, int& bestPos) {
    const int n = e - b;
    float bestCost = FLT_MAX;
    bestAx = -1;
    float rightA[kSmall];
    for (int ax = 0; ax < 3; ax++) {
      if (!(comp(ext, ax) > 0.0f)) continue;
      sortSmall(b, e, ax);
      Box3 acc = boxEmpty();
      for (int i = n - 1; i > 0; i--) {
        boxGrow(acc, boxes[ids[b + i]]);
        rightA[i] = boxArea(acc);
      }
      acc = boxEmpty();
      for (int i = 1; i < n; i++) {
        boxGrow(acc, boxes[ids[b + i - 1]]);
        float c = boxArea(acc) * i + rightA[i] * (n - i);
        if (c < bestCost) {
          bestCost = c;
          bestAx = ax;
          bestPos = i;
        }
      }
    }
    return bestCost;
  }

  // Binned SAH over all three axes in one pass over the primitives. Returns
  // the cost; ax / bin the split (bins <= bin go left), ax = -1 if none.
  float binnedSweep(int b, int e, const Box3& cb, const float3& ext, int& bestAx, int& bestBin,
                    Box3& lb, Box3& rb) {
    Box3 bb[3][kBins];
    int bc[3][kBins];
    float lo[3], sc[3];
    bool on[3];
    for (int ax = 0; ax < 3; ax++) {
      on[ax] = comp(ext, ax) > 0.0f;
      lo[ax] = comp(cb.lo, ax);
      sc[ax] = on[ax] ? kBins / comp(ext, ax) : 0.0f;
      for (int k = 0; k < kBins; k++) {
        bb[ax][k] = boxEmpty();
        bc[ax][k] = 0;
      }
    }
    for (int i = b; i < e; i++) {
      const int id = ids[i];
      const Box3& bx = boxes[id];
      const float3 c = cent[id];
      for (int ax = 0; ax < 3; ax++) {
        if (!on[ax]) continue;
        int k = (int)((comp(c, ax) - lo[ax]) * sc[ax]);
        k = std::min(std::max(k, 0), kBins - 1);
        bc[ax][k]++;
        boxGrow(bb[ax][k], bx);
      }
    }
    float bestCost = FLT_MAX;
    bestAx = -1;
    for (int ax = 0; ax < 3; ax++) {
      if (!on[ax]) continue;
      float rightA[kBins];
      int rightN[kBins];
      Box3 acc = boxEmpty();
      int cnt = 0;
      for (int k = kBins - 1; k > 0; k--) {
        boxGrow(acc, bb[ax][k]);
        cnt += bc[ax][k];
        rightA[k] = boxArea(acc);
        rightN[k] = cnt;
      }
      acc = boxEmpty();
      cnt = 0;
      for (int k = 0; k < kBins - 1; k++) {
        boxGrow(acc, bb[ax][k]);
        cnt += bc[ax][k];
        if (cnt == 0 || rightN[k + 1] == 0) continue;
        float c = boxArea(acc) * cnt + rightA[k + 1] * rightN[k + 1];
        if (c < bestCost) {
          bestCost = c;
          bestAx = ax;
          bestBin = k;
        }
      }
    }
    if (bestAx >= 0) {
      lb = boxEmpty();
      rb = boxEmpty();
      for (int k = 0; k < kBins; k++) boxGrow(k <= bestBin ? lb : rb, bb[bestAx][k]);
    }
    return bestCost;
  }

  // Returns the split position in [b+1, e-1] with the two children's bounds
  // in lb / rb, or -1 for a leaf. nb: the bounds of [b, e). Ranges of up to
  // kSmall primitives are split exactly (every centroid position), larger
  // ones by binning; the child bounds come from the sweep itself.
  int split(int b, int e, int depth, const Box3& nb, Box3& lb, Box3& rb) {
    int n = e - b;
    if (n <= 1) return -1;
    Box3 cb = boxEmpty();
    for (int i = b; i < e; i++) boxGrow(cb, cent[ids[i]]);
    float3 ext = cb.hi - cb.lo;
    bool forceMedian = depth >= kDepthLimit;
    float bestCost = FLT_MAX;
    int bestAx = -1, bestAt = -1;
    if (!forceMedian) {
      if (n <= kSmall)
        bestCost = exactSweep(b, e, ext, bestAx, bestAt);
      else
        bestCost = binnedSweep(b, e, cb, ext, bestAx, bestAt, lb, rb);
    }
    float leafCost = boxArea(nb) * n;
    const float kTraverse = 1.2f;  // node visit relative to one primitive test
    if (!forceMedian && bestAx >= 0 && n <= maxLeaf &&
        leafCost <= bestCost + kTraverse * boxArea(nb))
      return -1;
    if (bestAx < 0) {
      if (n <= maxLeaf) return -1;
      // Degenerate centroids or depth limit: median split on the widest axis.
      int ax = ext.x >= ext.y && ext.x >= ext.z ? 0 : (ext.y >= ext.z ? 1 : 2);
      int mid = b + n / 2;
      std::nth_element(ids.begin() + b, ids.begin() + mid, ids.begin() + e, [&](int x, int y) {
        return comp(cent[x], ax) < comp(cent[y], ax);
      });
      lb = rangeBox(b, mid);
      rb = rangeBox(mid, e);
      return mid;
    }
    if (n <= kSmall) {
      sortSmall(b, e, bestAx);
      int mid = b + bestAt;
      lb = rangeBox(b, mid);
      rb = rangeBox(mid, e);
      return mid;
    }
    float lo = comp(cb.lo, bestAx), sc = kBins / comp(ext, bestAx);
    int* pm = std::partition(ids.data() + b, ids.data() + e, [&](int id) {
      int k = (int)((comp(cent[id], bestAx) - lo) * sc);
      k = std::min(std::max(k, 0), kBins - 1);
      return k <= bestAt;
    });
    int mid = (int)(pm - ids.data());
    if (mid == b || mid == e) {
      mid = b + n / 2;
      lb = rangeBox(b, mid);
      rb = rangeBox(mid, e);
    }
    return mid;
  }

  // Encoded link for [b, e) with bounds nb.
  int build(int b, int e, int depth, const Box3& nb) {
    out.maxDepth = std::max(out.maxDepth, depth);
    Box3 lb, rb;
    int m = split(b, e, depth, nb, lb, rb);
    if (m < 0) return leafLink(b, e);
    int idx = (int)out.nodes.size();
    out.nodes.push_back(BvhNode{});
    int l, r;
    children(b, m, e, depth + 1, lb, rb, l, r);
    fill(out.nodes[idx], lb, rb, l, r);
    return nodeBase + idx;
  }

  // Links of the children [b, m) and [m, e) at `depth`, left subtree first.
  void children(int b, int m, int e, int depth, const Box3& lb, const Box3& rb, int& l, int& r) {
    if (!parallel || e - b < kParallelMin || depth > kParallelDepth) {
      l = build(b, m, depth, lb);
      r = build(m, e, depth, rb);
      return;
    }
    Builder sub(*this, 0);
    std::future<int> right = std::async(std::launch::async, [&sub, m, e, depth, &rb] {
      return sub.build(m, e, depth, rb);
    });
    l = build(b, m, depth, lb);
    int rs = right.get();
    const int off = nodeBase + (int)out.nodes.size();
    for (BvhNode& nd : sub.out.nodes) {
      if (nd.link.x >= 0) nd.link.x += off;
      if (nd.link.y >= 0) nd.link.y += off;
    }
    r = rs >= 0 ? rs + off : rs;
    out.nodes.insert(out.nodes.end(), sub.out.nodes.begin(), sub.out.nodes.end());
    out.maxDepth = std::max(out.maxDepth, sub.out.maxDepth);
  }

  static void fill(BvhNode& nd, const Box3& a, const Box3& c, int la, int lc) {
    nd.xy0 = make_float4(a.lo.x, a.hi.x, a.lo.y, a.hi.y);
    nd.xy1 = make_float4(c.lo.x, c.hi.x, c.lo.y, c.hi.y);
    nd.zz = make_float4(a.lo.z, a.hi.z, c.lo.z, c.hi.z);
    nd.link = make_int4(la, lc, 0, 0);
  }
};

}  // namespace

BvhBuild buildBvh(const std::vector<Box3>& boxes, int maxLeaf, int nodeBase, int primBase) {
  BuildInput in(boxes);
  Builder bd(boxes, in, std::min(std::max(maxLeaf, 1), 8), nodeBase, primBase, true);
  int n = (int)boxes.size();
  bd.out.nodes.push_back(BvhNode{});  // root slot
  if (n == 0) {
    // Empty tree: both children far away and degenerate, never entered.
    Box3 far = {v3(3e30f), v3(3e30f)};
    Builder::fill(bd.out.nodes[0], far, far, ~0, ~0);
    return bd.out;
  }
  const Box3 root = bd.rangeBox(0, n);
  Box3 lb, rb;
  int m = bd.split(0, n, 0, root, lb, rb);
  if (m < 0) {
    Box3 far = {v3(3e30f), v3(3e30f)};
    Builder::fill(bd.out.nodes[0], root, far, bd.leafLink(0, n), bd.leafLink(0, n));
  } else {
    int l, r;
    bd.children(0, m, n, 1, lb, rb, l, r);
    Builder::fill(bd.out.nodes[0], lb, rb, l, r);
  }
  bd.out.order = bd.ids;
  return bd.out;
}

}  // namespace sdb

// ---- explicit binary tree + 8-wide collapse ------------------------------------

namespace sdb {

namespace {

struct BinBuilder {
  BuildInput in;
  Builder core;
  BinTree out;
  BinBuilder(const std::vector<Box3>& b, int ml) : in(b), core(b, in, ml, 0, 0, false) {}

  int build(int b, int e, int depth, const Box3& nb) {
    out.maxDepth = std::max(out.maxDepth, depth);
    int idx = (int)out.nodes.size();
    out.nodes.push_back(BinNode{});
    out.nodes[idx].box = nb;
    Box3 lb, rb;
    int m = core.split(b, e, depth, nb, lb, rb);
    if (m < 0) {
      out.nodes[idx].start = b;
      out.nodes[idx].count = e - b;
      return idx;
    }
    int l = build(b, m, depth + 1, lb);
    int r = build(m, e, depth + 1, rb);
    out.nodes[idx].left = l;
    out.nodes[idx].right = r;
    return idx;
  }
};

inline int exponentFor(float lo, float hi) {
  double ext = (double)hi - (double)lo;
  if (!(ext > 0.0)) return -120;
  int e = (int)std::ceil(std::log2(ext / 255.0));
  if (ext / std::ldexp(1.0, e) > 255.0) e++;
  return std::min(std::max(e, -120), 120);
}

inline uint8_t byteOf(const float4& v, int k) {
  uint32_t w[4];
  std::memcpy(w, &v, 16);
  return (uint8_t)(w[k >> 2] >> (8 * (k & 3)));
}
inline void setByte(float4& v, int k, uint8_t b) {
  uint32_t w[4];
  std::memcpy(w, &v, 16);
  w[k >> 2] = (w[k >> 2] & ~(0xFFu << (8 * (k & 3)))) | ((uint32_t)b << (8 * (k & 3)));
  std::memcpy(&v, w, 16);
}
inline uint32_t wordOf(const float4& v, int k) {
  uint32_t w[4];
  std::memcpy(w, &v, 16);
  return w[k];
}
inline void setWord(float4& v, int k, uint32_t x) {
  uint32_t w[4];
  std::memcpy(w, &v, 16);
  w[k] = x;
  std::memcpy(&v, w, 16);
}

// Quantised coordinate of one bound, rounded outward and verified against
// the float decode the traversal performs (p + q * 2^e).
uint8_t quantLo(float p, int e, float v) {
  double s = std::ldexp(1.0, e);
  long q = (long)std::floor(((double)v - (double)p) / s);
  q = std::min(std::max(q, 0L), 255L);
  while (q > 0 && (float)(p + (float)((double)q * s)) > v) q--;
  return (uint8_t)q;
}
uint8_t quantHi(float p, int e, float v) {
  double s = std::ldexp(1.0, e);
  long q = (long)std::ceil(((double)v - (double)p) / s);
  q = std::min(std::max(q, 0L), 255L);
  while (q < 255 && (float)(p + (float)((double)q * s)) < v) q++;
  return (uint8_t)q;
}

}  // namespace

BinTree buildBinary(const std::vector<Box3>& boxes, int maxLeaf) {
  BinBuilder bb(boxes, maxLeaf);
  if (!boxes.empty()) bb.build(0, (int)boxes.size(), 0, bb.core.rangeBox(0, (int)boxes.size()));
  bb.out.order = bb.core.ids;
  return bb.out;
}

Box3 cwChildBox(const CwNode& n, int s) {
  float p[3] = {n.a.x, n.a.y, n.a.z};
  uint32_t ew = wordOf(n.a, 3);
  Box3 b;
  float* lo = &b.lo.x;
  float* hi = &b.hi.x;
  const float4* qlo[3] = {&n.c, &n.c, &n.d};
  const float4* qhi[3] = {&n.d, &n.e, &n.e};
  const int qloOff[3] = {0, 8, 0}, qhiOff[3] = {8, 0, 8};
  for (int a = 0; a < 3; a++) {
    int e = (int)(int8_t)(ew >> (8 * a));
    float sc = std::ldexp(1.0f, e);
    lo[a] = p[a] + (float)byteOf(*qlo[a], qloOff[a] + s) * sc;
    hi[a] = p[a] + (float)byteOf(*qhi[a], qhiOff[a] + s) * sc;
  }
  return b;
}

CwBuild buildCw(const std::vector<Box3>& boxes, int maxLeaf, int nodeBase, int primBase) {
  CwBuild out;
  int n = (int)boxes.size();
  BinTree bt = buildBinary(boxes, std::min(std::max(maxLeaf, 1), kCwLeafMax));
  if (n == 0) {
    // No primitives: one node with no valid slot.
    CwNode z;
    std::memset(&z, 0, sizeof z);
    out.nodes.push_back(z);
    return out;
  }
  struct Job {
    int bin;    // binary node collapsed into this wide node
    int slot;   // index in out.nodes
    int depth;
  };
  std::vector<Job> queue;
  out.nodes.push_back(CwNode{});
  queue.push_back({0, 0, 0});
  const float3 dirs[8] = {v3(1, 1, 1),   v3(-1, 1, 1),  v3(1, -1, 1),  v3(-1, -1, 1),
                          v3(1, 1, -1),  v3(-1, 1, -1), v3(1, -1, -1), v3(-1, -1, -1)};
  for (size_t qi = 0; qi < queue.size(); qi++) {
    Job job = queue[qi];
    out.maxDepth = std::max(out.maxDepth, job.depth);
    // Gather up to 8 children by repeatedly opening the largest internal one.
    std::vector<int> kids;
    const BinNode& root = bt.nodes[job.bin];
    if (root.left < 0) {
      kids.push_back(job.bin);  // a leaf at the top: one leaf slot
    } else {
      kids.push_back(root.left);
      kids.push_back(root.right);
      while (kids.size() < 8) {
        int best = -1;
        float bestA = -1.0f;
        for (size_t k = 0; k < kids.size(); k++) {
          const BinNode& c = bt.nodes[kids[k]];
          if (c.left < 0) continue;
          float3 e = c.box.hi - c.box.lo;
          float a = e.x * e.y + e.y * e.z + e.z * e.x;
          if (a > bestA) {
            bestA = a;
            best = (int)k;
          }
        }
        if (best < 0) break;
        int b = kids[best];
        kids.erase(kids.begin() + best);
        kids.push_back(bt.nodes[b].left);
        kids.push_back(bt.nodes[b].right);
      }
    }
    // Slot assignment: greedy auction on the alignment of each child's
    // offset from the node centre with the slot's octant diagonal.
    Box3 nb = boxEmpty();
    for (int k : kids) boxGrow(nb, bt.nodes[k].box);
    float3 ctr = (nb.lo + nb.hi) * 0.5f;
    struct Cand { float score; int kid, slot; };
    std::vector<Cand> cands;
    for (size_t k = 0; k < kids.size(); k++) {
      const BinNode& c = bt.nodes[kids[k]];
      float3 off = (c.box.lo + c.box.hi) * 0.5f - ctr;
      for (int s = 0; s < 8; s++) cands.push_back({dot(off, dirs[s]), (int)k, s});
    }
    std::sort(cands.begin(), cands.end(), [](const Cand& x, const Cand& y) {
      if (x.score != y.score) return x.score > y.score;
      if (x.kid != y.kid) return x.kid < y.kid;
      return x.slot < y.slot;
    });
    int slotKid[8];
    bool kidUsed[8] = {false, false, false, false, false, false, false, false};
    for (int s = 0; s < 8; s++) slotKid[s] = -1;
    for (const Cand& c : cands) {
      if (slotKid[c.slot] >= 0 || kidUsed[c.kid]) continue;
      slotKid[c.slot] = c.kid;
      kidUsed[c.kid] = true;
    }
    // Node header and quantisation grid.
    CwNode nd;
    std::memset(&nd, 0, sizeof nd);
    int ex = exponentFor(nb.lo.x, nb.hi.x), ey = exponentFor(nb.lo.y, nb.hi.y),
        ez = exponentFor(nb.lo.z, nb.hi.z);
    nd.a = make_float4(nb.lo.x, nb.lo.y, nb.lo.z, 0.0f);
    uint32_t imask = 0;
    int internalCount = 0;
    for (int s = 0; s < 8; s++)
      if (slotKid[s] >= 0 && bt.nodes[kids[slotKid[s]]].left >= 0) internalCount++;
    int childBase = (int)out.nodes.size();
    out.nodes.resize(out.nodes.size() + internalCount);
    int primBaseHere = (int)out.order.size();
    int internalSeen = 0, primOff = 0;
    for (int s = 0; s < 8; s++) {
      if (slotKid[s] < 0) continue;
      const BinNode& c = bt.nodes[kids[slotKid[s]]];
      setByte(nd.c, s, quantLo(nb.lo.x, ex, c.box.lo.x));
      setByte(nd.c, 8 + s, quantLo(nb.lo.y, ey, c.box.lo.y));
      setByte(nd.d, s, quantLo(nb.lo.z, ez, c.box.lo.z));
      setByte(nd.d, 8 + s, quantHi(nb.lo.x, ex, c.box.hi.x));
      setByte(nd.e, s, quantHi(nb.lo.y, ey, c.box.hi.y));
      setByte(nd.e, 8 + s, quantHi(nb.lo.z, ez, c.box.hi.z));
      uint8_t meta;
      if (c.left >= 0) {
        imask |= 1u << s;
        meta = 0xFF;
        queue.push_back({kids[slotKid[s]], childBase + internalSeen, job.depth + 1});
        internalSeen++;
      } else {
        meta = (uint8_t)((c.count << 5) | primOff);
        for (int k = 0; k < c.count; k++) out.order.push_back(bt.order[c.start + k]);
        primOff += c.count;
      }
      setByte(nd.b, 8 + s, meta);
    }
    uint32_t ew = (uint32_t)(uint8_t)(int8_t)ex | ((uint32_t)(uint8_t)(int8_t)ey << 8) |
                  ((uint32_t)(uint8_t)(int8_t)ez << 16) | (imask << 24);
    setWord(nd.a, 3, ew);
    setWord(nd.b, 0, (uint32_t)(nodeBase + childBase));
    setWord(nd.b, 1, (uint32_t)(primBase + primBaseHere));
    out.nodes[job.slot] = nd;
  }
  return out;
}

}  // namespace sdb
