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

namespace sdb {

// Binary SAH tree kept as explicit nodes (input to the 8-wide collapse).
struct BinNode {
  Box3 box;
  int left = -1, right = -1;  // children, -1 for a leaf
  int start = 0, count = 0;   // leaf range in BinTree::order
};
struct BinTree {
  std::vector<BinNode> nodes;  // node 0 = root
  std::vector<int> order;
  int maxDepth = 0;
};
BinTree buildBinary(const std::vector<Box3>& boxes, int maxLeaf);

// Collapse to compressed 8-wide nodes. Node indices are offset by nodeBase,
// primitive indices by primBase; `order` maps leaf order -> input primitive.
struct CwBuild {
  std::vector<CwNode> nodes;
  std::vector<int> order;
  int maxDepth = 0;
};
CwBuild buildCw(const std::vector<Box3>& boxes, int maxLeaf, int nodeBase, int primBase);

// Decoded child box of slot s (what the traversal tests), for checks.
Box3 cwChildBox(const CwNode& n, int s);

}  // namespace sdb
