// Host BVH builder: binned SAH over primitive boxes into the two-children-
// per-node layout of BvhNode (both child boxes in the parent, 64 bytes).
#pragma once

#include <vector>

#include "sd_types.h"

namespace sdb {

struct Box3 {
  float3 lo, hi;
};

Box3 boxEmpty();
void boxGrow(Box3& b, float3 p);
void boxGrow(Box3& b, const Box3& o);

struct BvhBuild {
  std::vector<BvhNode> nodes;  // node 0 is the root (always an inner node)
  std::vector<int> order;      // leaf order -> input primitive index
  int maxDepth = 0;
};

// nodeBase / primBase are added to every stored node index / leaf start so
// that several trees can live in one device array. maxLeaf <= 8.
BvhBuild buildBvh(const std::vector<Box3>& boxes, int maxLeaf, int nodeBase, int primBase);

}  // namespace sdb
