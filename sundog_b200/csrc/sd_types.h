// Scene descriptors as the kernels see them. Filled on the host by the render
// orchestration (render.cpp), uploaded once per render, read through the
// __constant__ launch block (SdLaunch) by every kernel.
//
// Field meaning follows sundog's device/params.h (MaterialDesc 28-40,
// LightDesc 42-71, EnvDesc 84-92, FlameDesc 97-105, CameraData 107-114); the
// layouts are this library's own (pointers to device arrays, no OptiX or
// texture-object handles: image lookups use the software filter in
// sd_texture.cuh).
#pragma once

#include "sd_vec.h"

namespace sdb {

enum GeomKind : int { GK_SPHERE = 0, GK_RECT, GK_DISK, GK_CYLINDER, GK_PARABOLA, GK_MESH, GK_COUNT };
enum TexKind : int { TX_SOLID = 0, TX_IMAGE, TX_CHECKER, TX_GRID };
enum MatKind : int { MT_LAMBERT = 0, MT_METAL, MT_DIELECTRIC, MT_EMISSIVE, MT_WATER, MT_PLASTIC };
enum LightKind : int { LT_RECT = 0, LT_DISK, LT_SPHERE, LT_POINT, LT_DISTANT, LT_MESH };
enum BgKind : int { BG_SOLID = 0, BG_GRADIENT, BG_ENVMAP };

constexpr uint16_t kMatNone = 0xFFFF;  // pass-through face

struct SdTexture {
  int kind;
  float3 a, b;       // solid colour / checker + grid colours
  float2 scale;      // checker / grid tiling
  float width;       // grid line width (cell fraction)
  int imgW, imgH;    // TX_IMAGE: texel grid
  int srgb;          // TX_IMAGE: texels are sRGB-encoded
  const uchar4* img; // TX_IMAGE: row-major RGBA8, row 0 = top of the image
};

struct SdMaterial {
  int kind;
  int texId;         // -1: use color
  float3 color;
  float roughness;   // GGX alpha = roughness^2; < 1e-3 is a delta lobe
  float ior;
  float intensity;   // emissive scale
  int twoSided;      // emissive visible from both faces
  float3 absorb;     // Beer-Lambert sigma inside (glass / water)
  float waveAmp;     // water wave-normal strength
  float waveFreq;    // water wave frequency (world xz)
};

struct SdLight {
  int kind;
  float3 p;          // centre / position
  float3 u, v;       // rect / disk half-edge basis
  float3 n;          // rect / disk front normal
  float3 L;          // radiance (area, distant) or intensity (point)
  float radius;
  float area;        // rect / disk / mesh world area
  float3 dir;        // distant: direction of travel
  int twoSided;
  int texId;
  int flameId;       // owning flame (embedded lights), -1 = none
  // LT_MESH: world-space triangle soup sampled by area.
  const float3* mPos;
  const uint3* mIdx;
  const float2* mUv;
  const float* mCdf; // mNumTris + 1 entries, [0] = 0, [n] = 1
  int mNumTris;
  float mNgSign;
};

// Guide of a CDF search: kCdfGuide + 1 ints per CDF, entry k the index the
// search returns for u = k / kCdfGuide (cdf_build.cu), so a search for u
// starts from the bracket of its bucket.
constexpr int kCdfGuide = 256;

struct SdEnv {
  const float4* texels;  // width x height, row 0 = zenith
  const float* margCdf;  // height + 1
  const float* condCdf;  // height x (width + 1)
  const int* margGuide;  // kCdfGuide + 1
  const int* condGuide;  // height x (kCdfGuide + 1)
  int width, height;
  float rotate;          // radians about +Y
  float intensity;
  int importance;        // 0: uniform-sphere NEE
};

struct SdFlame {
  float3 base;
  float height, radius, intensity, sigma, noiseScale;
  unsigned seed;
  int steps;             // ray-march steps (reference: 32)
};

struct SdCamera {
  float3 origin, lowerLeft, horizontal, vertical, u, v, w;
  float lensRadius;
};

// Instance of a quadric or a mesh BLAS. w2o maps world to object space; its
// transpose maps object-space normals to world space (inverse transpose).
struct SdInstance {
  float4 w2o[3];
  int kind;          // GeomKind
  int mesh;          // GK_MESH: mesh index
  uint32_t mats;     // matFront | matBack << 16
  int lightId;       // NEE light registered for this object, -1 = none
  int cutoutTex;     // alpha-cutout texture, -1 = none
  int flags;         // kInstMasked | kInstTransmissive
  int pad0, pad1;
};
constexpr int kInstMasked = 1;        // a face is pass-through, or a cutout
constexpr int kInstTransmissive = 2;  // a face is glass or water

struct SdMesh {
  const uint3* idx;
  const float3* pos;
  const float3* nrm;   // null: geometric normal
  const float2* uv;    // null: barycentric uv
  int root;            // this mesh's BLAS root in SdLaunch::cw
  int numTris;
};

// Binary BVH node: both children's boxes in one 64-byte node so a visit is
// four 16-byte loads. child >= 0 is an inner node index; child < 0 is a leaf
// whose primitives start at ~child, count in cnt.
struct __align__(16) BvhNode {
  float4 xy0;   // c0 lo.x hi.x lo.y hi.y
  float4 xy1;   // c1 lo.x hi.x lo.y hi.y
  float4 zz;    // c0 lo.z hi.z, c1 lo.z hi.z
  int4 link;    // child0, child1, cnt0, cnt1
};

// Node layout the traversal reads: 1 (default) the 4-wide nodes below,
// collapsed from the binary build; 0 the binary nodes themselves (measured
// on the bench frames, Mrays/s, 4-wide / binary: config 1 1,652 / 1,622,
// config 0 2,772 / 2,747, config 2 2,491 / 2,424).
#ifndef SDB_BVH4
#define SDB_BVH4 1
#endif

// 4-wide node (128 bytes, seven 16-byte loads), collapsed from the binary
// tree on the device (bvh_device.cu: each node holds the grandchildren of
// one binary node, or its child where that child is a leaf): the boxes of
// children 0-1 and of children 2-3 each in BvhNode's box layout (so a pair
// is tested with the binary node's arithmetic while the other pair is not
// yet loaded), then the four links (inner node index >= 0, leaf code < 0 as
// in BvhNode). An unused slot has the far point (3e30, 3e30, 3e30) as its
// box, which no ray reaches within its tmax.
struct __align__(16) Bvh4Node {
  float4 xy0, xy1, zz01;  // children 0 and 1: lo.x hi.x lo.y hi.y / ... / lo.z hi.z lo.z hi.z
  float4 xy2, xy3, zz23;  // children 2 and 3
  int4 link;
  int4 pad;
};

// Compressed 8-wide node (80 bytes, five 16-byte loads), after Ylitie,
// Karras and Laine, "Efficient Incoherent Ray Traversal on GPUs Through
// Compressed Wide BVHs" (HPG 2017). Child boxes are stored as 8-bit offsets
// on a per-node grid: child lo = p + qlo * 2^e, hi = p + qhi * 2^e, rounded
// outward when built so no hit is lost. Internal children are stored
// contiguously from childBase; leaf primitives contiguously from primBase.
// Slots are assigned so that visiting them in increasing slot ^ (ray octant
// ^ 7) order is approximately front to back.
//   a: p.x p.y p.z | e.x e.y e.z (int8) imask (bit s: slot s is internal)
//   b: childBase | primBase | meta[0..3] | meta[4..7]
//      meta (leaf slots): count << 5 | offset from primBase; 0 = empty slot
//   c: qlo.x[8] qlo.y[8]   d: qlo.z[8] qhi.x[8]   e: qhi.y[8] qhi.z[8]
struct __align__(16) CwNode {
  float4 a, b, c, d, e;
};
constexpr int kCwLeafMax = 3;  // primitives per leaf slot

// Traversal stack entries (sd_trace.cuh, wavefront.cu). The binary walk
// pushes at most one entry per inner level plus one marker at a BLAS entry,
// so TLAS depth + BLAS depth + 2 <= kTraversalStack; the 8-wide walk pushes
// at most one group per level plus three entries at a BLAS entry, so
// TLAS depth + BLAS depth + 4 <= kCwTraversalStack. The scene build rejects
// deeper trees, so no traversal ever finds its stack full.
constexpr int kTraversalStack = 64;
// The 4-wide walk (SDB_BVH4) pushes at most three entries per 4-wide level
// (two binary levels) plus one marker at a BLAS entry.
constexpr int kTraversal4Stack = 96;
constexpr int kCwTraversalStack = 48;

// Visit counts of the traversal, gathered only by the counting variant of the
// path kernel (for the algorithmic-bytes roofline), never in timed launches.
struct TraceCount {
  unsigned long long boxTests, triTests, quadTests, blasEntries;
  // SIMT occupancy of the loops, summed by the first active lane of each
  // warp: iterations executed, and active lanes over those iterations.
  unsigned long long travIters, travLanes, loopIters, loopLanes;
  unsigned long long traces;  // traversals (rays) counted here
};

// Everything a launch needs, in constant memory.
struct SdLaunch {
  int width, height;
  int sppTotal;
  int sampleOffset;      // first sample index of this launch
  int sppThisLaunch;
  int maxDepth;
  int nStrata;
  float clampVal;
  unsigned seed;
  int transparentShadows;
  int aovOn;

  // work decomposition: path p -> (sample p / npixPad, tile-ordered pixel)
  int tilesX;
  int npixPad;
  // Tile shard (one GPU of several): shardCount > 1 renders only the 64x64
  // film tiles t (row-major over shardTilesX tiles across) with
  // t % shardCount == shardIndex; path p -> (sample p / shardPad, owned tile,
  // 8x8 block, pixel). Every pixel keeps the seeds of the whole-frame render.
  int shardCount;
  int shardIndex;
  int shardTilesX;
  int shardPad;          // owned tiles x 4096
  unsigned long long numPaths;
  unsigned long long* pathCounter;
  unsigned long long* rayCounter;

  float4* sampleL;       // [sppThisLaunch][npixPad] radiance per sample
  float4* sampleAlb;     // [sppThisLaunch][npixPad] first-hit albedo
  float4* sampleNrm;     // [sppThisLaunch][npixPad] first-hit normal (camera)
  float4* accum;         // film running means [height*width]
  float4* aovAlbedo;
  float4* aovNormal;

  SdCamera cam;
  int bgKind;
  float3 bgA, bgB;
  SdEnv env;

  const SdTexture* textures;
  const SdMaterial* materials;
  const SdLight* lights;
  int numLights;
  const SdFlame* flames;
  int numFlames;

  const BvhNode* nodes;
  const Bvh4Node* nodes4;  // 4-wide nodes (the SDB_BVH4 layout), TLAS root first
  const CwNode* cw;       // 8-wide nodes (TLAS root first, then each BLAS)
  const float4* tris;     // 3 float4 per leaf-ordered triangle; .w of the
                          // first holds the mesh-local triangle index
  const SdInstance* inst;
  const SdMesh* meshes;
  int tlasRoot;
  int numInstances;

  // learned path guiding (read only by the guided kernel variants)
  const float4* guideLobes;   // [cells][8] lobes: kappa*mu, log pdf coefficient
  const float* guideCdf;      // [cells][8] cumulative lobe weights
  float3 guideLo;             // grid origin and 1 / extent
  float3 guideInvExtent;
  float guideMix;             // probability of drawing from the guide
  float4* guideTrain;         // training records, 3 float4 each
  unsigned long long* guideTrainCount;
  unsigned long long guideTrainCap;
};

}  // namespace sdb
