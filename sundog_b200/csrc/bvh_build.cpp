// Binned SAH build (Wald, "On fast Construction of SAH-based Bounding Volume
// Hierarchies", 2007): 32 bins per axis over centroid bounds, all three axes
// evaluated, leaf when splitting costs more than intersecting; below the
// depth limit of 48 a median split guarantees termination, so a traversal
// stack of 64 entries covers TLAS + BLAS depth.
#include "bvh_build.h"

#include <algorithm>
#include <cfloat>
#include <cmath>

namespace sdb {

Box3 boxEmpty() { return {v3(FLT_MAX), v3(-FLT_MAX)}; }
void boxGrow(Box3& b, float3 p) {
  b.lo = vmin(b.lo, p);
  b.hi = vmax(b.hi, p);
}
void boxGrow(Box3& b, const Box3& o) {
  b.lo = vmin(b.lo, o.lo);
  b.hi = vmax(b.hi, o.hi);
}
static float boxArea(const Box3& b) {
  float3 e = b.hi - b.lo;
  if (e.x < 0.0f) return 0.0f;
  return 2.0f * (e.x * e.y + e.y * e.z + e.z * e.x);
}

namespace {

constexpr int kBins = 32;
constexpr int kDepthLimit = 40;

struct Builder {
  const std::vector<Box3>& boxes;
  std::vector<float3> cent;
  std::vector<int> ids;
  int maxLeaf, nodeBase, primBase;
  BvhBuild out;

  Builder(const std::vector<Box3>& b, int ml, int nb, int pb)
      : boxes(b), maxLeaf(ml), nodeBase(nb), primBase(pb) {
    cent.resize(b.size());
    ids.resize(b.size());
    for (size_t i = 0; i < b.size(); i++) {
      cent[i] = (b[i].lo + b[i].hi) * 0.5f;
      ids[i] = (int)i;
    }
  }

  Box3 rangeBox(int b, int e) const {
    Box3 r = boxEmpty();
    for (int i = b; i < e; i++) boxGrow(r, boxes[ids[i]]);
    return r;
  }

  int leafLink(int b, int e) const {
    int code = ((primBase + b) << 3) | (e - b - 1);
    return ~code;
  }

  // Returns the split position in [b+1, e-1], or -1 for a leaf.
  int split(int b, int e, int depth) {
    int n = e - b;
    if (n <= 1) return -1;
    Box3 cb = boxEmpty();
    for (int i = b; i < e; i++) boxGrow(cb, cent[ids[i]]);
    float3 ext = cb.hi - cb.lo;
    bool forceMedian = depth >= kDepthLimit;
    float bestCost = FLT_MAX;
    int bestAxis = -1, bestBin = -1;
    if (!forceMedian) {
      for (int ax = 0; ax < 3; ax++) {
        float lo = comp(cb.lo, ax), e0 = comp(ext, ax);
        if (!(e0 > 0.0f)) continue;
        Box3 bb[kBins];
        int bc[kBins];
        for (int k = 0; k < kBins; k++) {
          bb[k] = boxEmpty();
          bc[k] = 0;
        }
        float sc = kBins / e0;
        for (int i = b; i < e; i++) {
          int k = (int)((comp(cent[ids[i]], ax) - lo) * sc);
          k = std::min(std::max(k, 0), kBins - 1);
          bc[k]++;
          boxGrow(bb[k], boxes[ids[i]]);
        }
        float rightA[kBins];
        int rightN[kBins];
        Box3 acc = boxEmpty();
        int cnt = 0;
        for (int k = kBins - 1; k > 0; k--) {
          boxGrow(acc, bb[k]);
          cnt += bc[k];
          rightA[k] = boxArea(acc);
          rightN[k] = cnt;
        }
        acc = boxEmpty();
        cnt = 0;
        for (int k = 0; k < kBins - 1; k++) {
          boxGrow(acc, bb[k]);
          cnt += bc[k];
          if (cnt == 0 || rightN[k + 1] == 0) continue;
          float c = boxArea(acc) * cnt + rightA[k + 1] * rightN[k + 1];
          if (c < bestCost) {
            bestCost = c;
            bestAxis = ax;
            bestBin = k;
          }
        }
      }
    }
    Box3 nb = rangeBox(b, e);
    float leafCost = boxArea(nb) * n;
    const float kTraverse = 1.2f;  // node visit relative to one primitive test
    if (!forceMedian && bestAxis >= 0 && n <= maxLeaf &&
        leafCost <= bestCost + kTraverse * boxArea(nb))
      return -1;
    if (bestAxis < 0) {
      if (n <= maxLeaf) return -1;
      // Degenerate centroids or depth limit: median split on the widest axis.
      int ax = ext.x >= ext.y && ext.x >= ext.z ? 0 : (ext.y >= ext.z ? 1 : 2);
      int mid = b + n / 2;
      std::nth_element(ids.begin() + b, ids.begin() + mid, ids.begin() + e, [&](int x, int y) {
        return comp(cent[x], ax) < comp(cent[y], ax);
      });
      return mid;
    }
    float lo = comp(cb.lo, bestAxis), sc = kBins / comp(ext, bestAxis);
    int* pm = std::partition(ids.data() + b, ids.data() + e, [&](int id) {
      int k = (int)((comp(cent[id], bestAxis) - lo) * sc);
      k = std::min(std::max(k, 0), kBins - 1);
      return k <= bestBin;
    });
    int mid = (int)(pm - ids.data());
    if (mid == b || mid == e) mid = b + n / 2;
    return mid;
  }

  // Encoded link for [b, e).
  int build(int b, int e, int depth) {
    out.maxDepth = std::max(out.maxDepth, depth);
    int m = split(b, e, depth);
    if (m < 0) return leafLink(b, e);
    int idx = (int)out.nodes.size();
    out.nodes.push_back(BvhNode{});
    Box3 lb = rangeBox(b, m), rb = rangeBox(m, e);
    int l = build(b, m, depth + 1);
    int r = build(m, e, depth + 1);
    fill(out.nodes[idx], lb, rb, l, r);
    return nodeBase + idx;
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
  Builder bd(boxes, std::min(std::max(maxLeaf, 1), 8), nodeBase, primBase);
  int n = (int)boxes.size();
  bd.out.nodes.push_back(BvhNode{});  // root slot
  if (n == 0) {
    // Empty tree: both children far away and degenerate, never entered.
    Box3 far = {v3(3e30f), v3(3e30f)};
    Builder::fill(bd.out.nodes[0], far, far, ~0, ~0);
    return bd.out;
  }
  int m = bd.split(0, n, 0);
  if (m < 0) {
    Box3 far = {v3(3e30f), v3(3e30f)};
    Builder::fill(bd.out.nodes[0], bd.rangeBox(0, n), far, bd.leafLink(0, n), bd.leafLink(0, n));
  } else {
    Box3 lb = bd.rangeBox(0, m), rb = bd.rangeBox(m, n);
    int l = bd.build(0, m, 1);
    int r = bd.build(m, n, 1);
    Builder::fill(bd.out.nodes[0], lb, rb, l, r);
  }
  bd.out.order = bd.ids;
  return bd.out;
}

}  // namespace sdb
