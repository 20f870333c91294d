// Device BVH construction (bvh_device.cu).
#pragma once

#include <cuda_runtime.h>

#include "sd_types.h"

namespace sdb {

struct DevBvhStats {
  int nodes = 0, maxDepth = 0, levels = 0;
};

// Binary BVH (BvhNode layout, root = nodes[0]) over n > maxLeaf primitive
// boxes lo / hi with centroids cent, all device arrays. Stored node links
// are offset by nodeBase and leaf starts by primBase; order (n ints, device)
// receives the leaf order (position -> input primitive). nodes must hold
// nodeCap >= n - 1 entries. Waits for the stream once per tree level.
DevBvhStats buildBvhDevice(const float4* lo, const float4* hi, const float4* cent, int n,
                           int maxLeaf, int nodeBase, int primBase, BvhNode* nodes, int nodeCap,
                           int* order, cudaStream_t st);

// 4-wide nodes from a binary node array (device, numBin nodes, links within
// it): each 4-wide node holds the grandchildren of one binary node (a leaf
// child kept as it is). roots (host, numRoots binary indices: the TLAS root,
// then each BLAS root) map to outRoots (host), roots[r] -> r. out (device)
// needs numBin entries. Returns the number of 4-wide nodes. Waits for the
// stream once per level.
int collapseBvh4Device(const BvhNode* bin, int numBin, const int* roots, int numRoots,
                       Bvh4Node* out, int* outRoots, cudaStream_t st);

// Object-space triangle boxes and centroids of a mesh.
void meshBoxesDevice(const float3* pos, const uint3* idx, int n, float4* lo, float4* hi,
                     float4* cent, cudaStream_t st);

// Triangles in leaf order: 3 float4 per triangle, .w of the first holding the
// mesh-local index.
void gatherTrisDevice(const float3* pos, const uint3* idx, const int* order, int n, float4* tris,
                      cudaStream_t st);

// One instance's geometry for its world box: a mesh's vertices (pos,
// numVerts), or when pos is null the 8 corners of the quadric bounds
// qlo / qhi; xf the object-to-world map (3x4 row-major).
struct DevInstanceSrc {
  const float3* pos;
  int numVerts;
  float xf[12];
  float3 qlo, qhi;
};
// World boxes (padded by a few ulps, as the host build does) and centroids.
void instanceBoxesDevice(const DevInstanceSrc* src, int n, float4* lo, float4* hi, float4* cent,
                         cudaStream_t st);

}  // namespace sdb
