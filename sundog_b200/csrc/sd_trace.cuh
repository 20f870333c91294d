// Two-level BVH traversal in software (B200 has no RT cores).
//
// One loop walks the instance BVH (TLAS) and, on reaching a mesh instance,
// the mesh's own BVH (BLAS) with the ray mapped into object space; a marker
// on the per-thread stack restores the world ray when the BLAS is done.
// Quadric instances are tested analytically at the TLAS leaf.
//
// Hit semantics reproduce what sundog obtains from OptiX
// (device/programs.cu:49-85, 112-125, 207-302; src/accel.cpp:54-58, 105-107):
//  * radiance rays: closest accepted hit in (0, tmax); a candidate whose hit
//    side has no material (MAT_NONE) or whose cutout alpha is < 0.5 is
//    ignored and traversal continues; every quadric root is a candidate;
//  * shadow rays: any accepted opaque hit in (0, tmax) occludes; a glass or
//    water crossing (transparent shadows on) multiplies the Fresnel
//    transmission 1 - F and adds the signed optical depth +-sigma t, and is
//    ignored; each crossing is visited exactly once because BVH leaves
//    partition the primitives.
// Triangles use the watertight test of Woop, Benthin and Wald (JCGT 2013).
#pragma once

#ifndef SDB_WIDE_BVH
#define SDB_WIDE_BVH 0
#endif

#include "sd_quadric.cuh"
#include "sd_texture.cuh"
#include "sd_types.h"

namespace sdb {

// The 4-wide walk pushes up to three entries per level.
constexpr int kStackSize = SDB_BVH4 ? kTraversal4Stack : kTraversalStack;
constexpr int kPop = (int)0x80000000;        // "take the next stack entry"
constexpr int kToTlas = (int)0x80000001;     // marker: leave the BLAS

struct TraceHit {
  float t;
  int inst;
  int prim;      // mesh-local triangle index (meshes)
  float u, v;    // triangle barycentrics (weights of p1, p2) or quadric uv
  float3 nq;     // quadric object-space front normal
  bool front;
};


__device__ __forceinline__ void countWarp(TraceCount* cnt, unsigned long long& iters,
                                          unsigned long long& lanes) {
  unsigned m = __activemask();
  if ((threadIdx.x & 31) == (unsigned)(__ffs(m) - 1)) {
    iters++;
    lanes += __popc(m);
  }
}

struct ShadePt {
  float3 nFront;  // world unit normal of the canonical front side
  float u, v;
  bool front;
};

__device__ __forceinline__ float3 ldg3(const float3* p) {
  const float* f = reinterpret_cast<const float*>(p);
  return v3(__ldg(f), __ldg(f + 1), __ldg(f + 2));
}

__device__ __forceinline__ float3 xfPoint(const float4* m, float3 p) {
  return v3(m[0].x * p.x + m[0].y * p.y + m[0].z * p.z + m[0].w,
            m[1].x * p.x + m[1].y * p.y + m[1].z * p.z + m[1].w,
            m[2].x * p.x + m[2].y * p.y + m[2].z * p.z + m[2].w);
}
__device__ __forceinline__ float3 xfVec(const float4* m, float3 v) {
  return v3(m[0].x * v.x + m[0].y * v.y + m[0].z * v.z,
            m[1].x * v.x + m[1].y * v.y + m[1].z * v.z,
            m[2].x * v.x + m[2].y * v.y + m[2].z * v.z);
}
// Object-space normal to world space: transpose of the world->object map.
__device__ __forceinline__ float3 xfNormal(const float4* m, float3 n) {
  return v3(m[0].x * n.x + m[1].x * n.y + m[2].x * n.z,
            m[0].y * n.x + m[1].y * n.y + m[2].y * n.z,
            m[0].z * n.x + m[1].z * n.y + m[2].z * n.z);
}

// Per-ray constants of the watertight triangle test.
struct WtRay {
  int kx, ky, kz;
  float Sx, Sy, Sz;
};
__device__ __forceinline__ WtRay wtSetup(float3 d) {
  WtRay w;
  float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  w.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  w.kx = w.kz == 2 ? 0 : w.kz + 1;
  w.ky = w.kx == 2 ? 0 : w.kx + 1;
  float dz = comp(d, w.kz);
  if (dz < 0.0f) {
    int t = w.kx;
    w.kx = w.ky;
    w.ky = t;
  }
  w.Sx = comp(d, w.kx) / dz;
  w.Sy = comp(d, w.ky) / dz;
  w.Sz = 1.0f / dz;
  return w;
}

// Watertight ray/triangle; returns t and the weights (b1, b2) of p1, p2.
__device__ __forceinline__ bool wtHit(const WtRay& w, float3 o, float3 p0, float3 p1, float3 p2,
                                      float tmin, float tmax, float& t, float& b1, float& b2) {
  float3 A = p0 - o, B = p1 - o, C = p2 - o;
  float Az = comp(A, w.kz), Bz = comp(B, w.kz), Cz = comp(C, w.kz);
  float Ax = comp(A, w.kx) - w.Sx * Az, Ay = comp(A, w.ky) - w.Sy * Az;
  float Bx = comp(B, w.kx) - w.Sx * Bz, By = comp(B, w.ky) - w.Sy * Bz;
  float Cx = comp(C, w.kx) - w.Sx * Cz, Cy = comp(C, w.ky) - w.Sy * Cz;
  float U = Cx * By - Cy * Bx;
  float V = Ax * Cy - Ay * Cx;
  float W = Bx * Ay - By * Ax;
  if (U == 0.0f || V == 0.0f || W == 0.0f) {
    // Edge case: redo the 2D edge functions in double (exact for float input).
    U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
    V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
    W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
  }
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
  float det = U + V + W;
  if (det == 0.0f) return false;
  float T = U * (w.Sz * Az) + V * (w.Sz * Bz) + W * (w.Sz * Cz);
  float inv = 1.0f / det;
  t = T * inv;
  if (!(t > tmin && t < tmax)) return false;
  b1 = V * inv;
  b2 = W * inv;
  return true;
}

// Slab test of both children of a node; robust far-plane scaling after Ize,
// "Robust BVH Ray Traversal" (JCGT 2013).
__device__ __forceinline__ void boxPair(const BvhNode& nd, float3 oi, float3 id, float tmin,
                                        float tmax, float& ta, float& tb, bool& ha, bool& hb) {
  const float kFar = 1.00000024f;
  float lx0 = nd.xy0.x * id.x - oi.x, hx0 = nd.xy0.y * id.x - oi.x;
  float ly0 = nd.xy0.z * id.y - oi.y, hy0 = nd.xy0.w * id.y - oi.y;
  float lz0 = nd.zz.x * id.z - oi.z, hz0 = nd.zz.y * id.z - oi.z;
  float lx1 = nd.xy1.x * id.x - oi.x, hx1 = nd.xy1.y * id.x - oi.x;
  float ly1 = nd.xy1.z * id.y - oi.y, hy1 = nd.xy1.w * id.y - oi.y;
  float lz1 = nd.zz.z * id.z - oi.z, hz1 = nd.zz.w * id.z - oi.z;
  float n0 = fmaxf(fmaxf(fminf(lx0, hx0), fminf(ly0, hy0)), fmaxf(fminf(lz0, hz0), tmin));
  float f0 = fminf(fminf(fmaxf(lx0, hx0), fmaxf(ly0, hy0)), fminf(fmaxf(lz0, hz0), tmax)) * kFar;
  float n1 = fmaxf(fmaxf(fminf(lx1, hx1), fminf(ly1, hy1)), fmaxf(fminf(lz1, hz1), tmin));
  float f1 = fminf(fminf(fmaxf(lx1, hx1), fmaxf(ly1, hy1)), fminf(fmaxf(lz1, hz1), tmax)) * kFar;
  ha = n0 <= f0;
  hb = n1 <= f1;
  ta = n0;
  tb = n1;
}

// Orders (d, l) pairs: the smaller distance first, ties keep their order.
__device__ __forceinline__ void cswap(float& da, int& la, float& db, int& lb) {
  if (db < da) {
    float td = da;
    da = db;
    db = td;
    int tl = la;
    la = lb;
    lb = tl;
  }
}

__device__ __forceinline__ float safeInv(float x) {
  const float e = 1e-20f;
  return 1.0f / (fabsf(x) > e ? x : copysignf(e, x));
}

__device__ __forceinline__ BvhNode loadNode(const BvhNode* nodes, int i) {
  const float4* p = reinterpret_cast<const float4*>(nodes + i);
  BvhNode n;
  n.xy0 = __ldg(p);
  n.xy1 = __ldg(p + 1);
  n.zz = __ldg(p + 2);
  float4 l = __ldg(p + 3);
  n.link = make_int4(__float_as_int(l.x), __float_as_int(l.y), __float_as_int(l.z),
                     __float_as_int(l.w));
  return n;
}

// Shade point of a triangle hit (device/programs.cu:147-190): geometric
// normal through the inverse transpose, interpolated smooth normal kept on
// the geometric side, uv from the mesh or the barycentrics, and the
// geometric normal for emissive faces of registered mesh lights.
__device__ __forceinline__ ShadePt triShade(const SdLaunch& lp, const SdInstance& in, int prim,
                                            float b1, float b2, float3 D) {
  const SdMesh& me = lp.meshes[in.mesh];
  uint3 tri = me.idx[prim];
  float3 p0 = ldg3(me.pos + tri.x), p1 = ldg3(me.pos + tri.y), p2 = ldg3(me.pos + tri.z);
  float3 ngObj = cross(p1 - p0, p2 - p0);
  float3 ng = unit(xfNormal(in.w2o, ngObj));
  float3 ns = ng;
  float w0 = 1.0f - b1 - b2;
  if (me.nrm) {
    float3 n = ldg3(me.nrm + tri.x) * w0 + ldg3(me.nrm + tri.y) * b1 + ldg3(me.nrm + tri.z) * b2;
    ns = unit(xfNormal(in.w2o, n));
    if (dot(ns, ng) < 0.0f) ns = -ns;
  }
  ShadePt sp;
  sp.nFront = ns;
  if (me.uv) {
    float2 a = me.uv[tri.x], b = me.uv[tri.y], c = me.uv[tri.z];
    sp.u = a.x * w0 + b.x * b1 + c.x * b2;
    sp.v = a.y * w0 + b.y * b1 + c.y * b2;
  } else {
    sp.u = b1;
    sp.v = b2;
  }
  sp.front = dot(ng, D) < 0.0f;
  if (in.lightId >= 0) {
    uint16_t side = sp.front ? (uint16_t)(in.mats & 0xFFFF) : (uint16_t)(in.mats >> 16);
    if (side != kMatNone && lp.materials[side].kind == MT_EMISSIVE) sp.nFront = ng;
  }
  return sp;
}

__device__ __forceinline__ ShadePt quadShade(const SdInstance& in, float3 nq, float u, float v,
                                             float3 D) {
  ShadePt sp;
  sp.nFront = unit(xfNormal(in.w2o, nq));
  sp.u = u;
  sp.v = v;
  sp.front = dot(sp.nFront, D) < 0.0f;
  return sp;
}

// Any-hit filter shared by both ray types: false = pass through.
__device__ __forceinline__ bool faceAccepts(const SdLaunch& lp, const SdInstance& in, bool front,
                                            float u, float v) {
  uint16_t m = front ? (uint16_t)(in.mats & 0xFFFF) : (uint16_t)(in.mats >> 16);
  if (m == kMatNone) return false;
  if (in.cutoutTex >= 0) {
    float4 c = texLookup(lp.textures[in.cutoutTex], u, v);
    if (c.w < 0.5f) return false;
  }
  return true;
}

// Transparent-shadow bookkeeping for one crossing; false = the crossing
// occludes (opaque material, transparent shadows off, or TIR).
// (device/programs.cu:247-292)
__device__ __forceinline__ bool shadowCross(const SdLaunch& lp, const ShadePt& sp, uint16_t mid,
                                            float t, float3 D, float& trProd, float3& tau) {
  const SdMaterial& m = lp.materials[mid];
  if (m.kind != MT_DIELECTRIC && m.kind != MT_WATER) return false;
  if (!lp.transparentShadows) return false;
  float3 n = sp.front ? sp.nFront : -sp.nFront;
  float eta = sp.front ? 1.0f / m.ior : m.ior;
  float3 refr;
  if (!snell(D, n, eta, refr)) return false;
  float f0 = (1.0f - eta) / (1.0f + eta);
  f0 = f0 * f0;
  float c = sp.front ? -dot(D, n) : -dot(refr, n);
  float F = fresnelSchlick(c, f0);
  trProd *= (1.0f - F);
  float s = sp.front ? -t : t;
  tau = v3(tau.x + m.absorb.x * s, tau.y + m.absorb.y * s, tau.z + m.absorb.z * s);
  return true;
}

// ---- 8-wide compressed traversal ----------------------------------------------

// Byte k of w as a float: assemble 2^23 + byte in one byte permute, subtract
// 2^23 (exact).
__device__ __forceinline__ float qbyte(uint32_t w, int k) {
  return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7540u | (unsigned)k)) - 8388608.0f;
}

__device__ __forceinline__ float expScale(uint32_t ew, int axis) {
  int e = (int)(signed char)((ew >> (8 * axis)) & 0xFFu);
  return __uint_as_float((uint32_t)(e + 127) << 23);
}

// Tests the 8 child boxes of node `idx` against the ray (origin o, inverse
// direction id, octant order rayOct, interval [tmin, tmax]). Returns the
// node's child/primitive bases, the internal children hit (bit i ^ rayOct
// for slot i, so the lowest set bit is the nearest-first candidate) and the
// primitives of the leaf children hit (bits relative to primBase).
struct CwHits {
  uint32_t childBase, primBase, imask, hits, leafBits, valid;
};
__device__ __forceinline__ CwHits cwIntersect(const CwNode* nodes, int idx, float3 o, float3 id,
                                              uint32_t rayOct, float tmin, float tmax) {
  const float kFar = 1.00000024f;
  const float4* p4 = reinterpret_cast<const float4*>(nodes + idx);
  float4 a = __ldg(p4), b = __ldg(p4 + 1), c = __ldg(p4 + 2), d = __ldg(p4 + 3), e = __ldg(p4 + 4);
  uint32_t ew = __float_as_uint(a.w);
  CwHits r;
  r.imask = ew >> 24;
  r.childBase = __float_as_uint(b.x);
  r.primBase = __float_as_uint(b.y);
  uint32_t meta[2] = {__float_as_uint(b.z), __float_as_uint(b.w)};
  float sx = expScale(ew, 0) * id.x, sy = expScale(ew, 1) * id.y, sz = expScale(ew, 2) * id.z;
  float ox = (a.x - o.x) * id.x, oy = (a.y - o.y) * id.y, oz = (a.z - o.z) * id.z;
  // Near / far planes per axis: lo words give the near plane unless the
  // direction is negative on that axis.
  uint32_t lx[2] = {__float_as_uint(c.x), __float_as_uint(c.y)};
  uint32_t ly[2] = {__float_as_uint(c.z), __float_as_uint(c.w)};
  uint32_t lz[2] = {__float_as_uint(d.x), __float_as_uint(d.y)};
  uint32_t hx[2] = {__float_as_uint(d.z), __float_as_uint(d.w)};
  uint32_t hy[2] = {__float_as_uint(e.x), __float_as_uint(e.y)};
  uint32_t hz[2] = {__float_as_uint(e.z), __float_as_uint(e.w)};
  uint32_t nx[2], ny[2], nz[2], fx[2], fy[2], fz[2];
#pragma unroll
  for (int w = 0; w < 2; w++) {
    bool sxn = id.x < 0.0f, syn = id.y < 0.0f, szn = id.z < 0.0f;
    nx[w] = sxn ? hx[w] : lx[w];
    fx[w] = sxn ? lx[w] : hx[w];
    ny[w] = syn ? hy[w] : ly[w];
    fy[w] = syn ? ly[w] : hy[w];
    nz[w] = szn ? hz[w] : lz[w];
    fz[w] = szn ? lz[w] : hz[w];
  }
  r.hits = 0;
  r.leafBits = 0;
  r.valid = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    int w = i >> 2, k = i & 3;
    uint32_t m = (meta[w] >> (8 * k)) & 0xFFu;
    float tn = fmaxf(fmaxf(fmaf(qbyte(nx[w], k), sx, ox), fmaf(qbyte(ny[w], k), sy, oy)),
                     fmaxf(fmaf(qbyte(nz[w], k), sz, oz), tmin));
    float tf = fminf(fminf(fmaf(qbyte(fx[w], k), sx, ox), fmaf(qbyte(fy[w], k), sy, oy)),
                     fminf(fmaf(qbyte(fz[w], k), sz, oz), tmax)) * kFar;
    bool slot = m != 0u;
    r.valid |= (slot ? 1u : 0u) << i;
    bool hit = slot && tn <= tf;
    bool inner = (r.imask >> i) & 1u;
    if (hit && inner) r.hits |= 1u << (i ^ rayOct);
    if (hit && !inner) r.leafBits |= ((1u << (m >> 5)) - 1u) << (m & 31u);
  }
  return r;
}

struct RayCtx {
  float3 o, d, id;
  uint32_t rayOct;  // slot ^ rayOct orders children near to far
  WtRay wt;
};
__device__ __forceinline__ void rayInit(RayCtx& r, float3 o, float3 d, bool tri) {
  r.o = o;
  r.d = d;
  r.id = v3(safeInv(d.x), safeInv(d.y), safeInv(d.z));
  uint32_t oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
  r.rayOct = oct ^ 7u;
  if (tri) r.wt = wtSetup(d);
}

constexpr int kCwStack = kCwTraversalStack;
constexpr uint32_t kGroupPrims = 1u << 31;   // entry holds a primitive group
constexpr uint32_t kGroupMarker = 1u << 30;  // entry returns from a BLAS

// Traversal is compiled out of line: one copy per (shadow, counting)
// variant instead of one per call site keeps the path loop's instruction
// footprint small; measured 856 vs 828 Mrays/s inlined (instancing frame,
// 16 blocks per SM).
#ifndef SDB_TRAVERSE_INLINE
#define SDB_TRAVERSE_INLINE __noinline__
#endif

// The BVH format is a build-time choice of the kernels (SDB_WIDE_BVH): the
// binary layout (BvhNode, 2 children per 64-byte node) or the compressed
// 8-wide layout (CwNode). The host builds whichever bvhWidth() reports.
#if SDB_WIDE_BVH
// SHADOW = false: closest accepted hit, returns whether one was found.
// SHADOW = true: returns false when occluded, else accumulates the
// transparent-crossing terms into trProd / tau.
template <bool SHADOW, bool COUNT = false>
__device__ SDB_TRAVERSE_INLINE bool traverse(const SdLaunch& lp, float3 O, float3 D, float tmax,
                                             TraceHit& hit, float& trProd, float3& tau,
                                             TraceCount* cnt = nullptr) {
  if (COUNT) cnt->traces++;
  if (lp.numInstances == 0) return SHADOW;
  uint2 stack[kCwStack];
  int sp = 0;
  const float tmin = 0.0f;
  const CwNode* nodes = lp.cw;
  RayCtx ray;
  rayInit(ray, O, D, false);
  bool inBlas = false;
  int curInst = -1;
  bool found = false;
  // Current node group: a virtual parent whose only child (slot 0) is the root.
  uint32_t gBase = (uint32_t)lp.tlasRoot, gHits = 1u << (0u ^ ray.rayOct), gImask = 1u;
  uint32_t tBase = 0, tBits = 0;

  while (true) {
    if (COUNT) countWarp(cnt, cnt->travIters, cnt->travLanes);
    if (gHits) {
      int b = __ffs(gHits) - 1;
      gHits &= gHits - 1u;
      uint32_t slot = (uint32_t)b ^ ray.rayOct;
      int child = (int)(gBase + __popc(gImask & ((1u << slot) - 1u)));
      if (gHits && sp < kCwStack) stack[sp++] = make_uint2(gBase, gHits | (gImask << 8));
      CwHits h = cwIntersect(nodes, child, ray.o, ray.id, ray.rayOct, tmin, tmax);
      if (COUNT) cnt->boxTests += __popc(h.valid);
      gBase = h.childBase;
      gHits = h.hits;
      gImask = h.imask;
      tBase = h.primBase;
      tBits = h.leafBits;
    }
    while (tBits) {
      int j = __ffs(tBits) - 1;
      tBits &= tBits - 1u;
      int prim = (int)tBase + j;
      if (!inBlas) {
        const SdInstance& in = lp.inst[prim];
        float3 o2 = xfPoint(in.w2o, O), d2 = xfVec(in.w2o, D);
        if (in.kind == GK_MESH) {
          if (COUNT) cnt->blasEntries++;
          // Unreachable: the scene build rejects trees whose TLAS + BLAS
          // depth could fill the stack (kCwTraversalStack).
          if (sp + 3 > kCwStack) continue;
          if (gHits) stack[sp++] = make_uint2(gBase, gHits | (gImask << 8));
          if (tBits) stack[sp++] = make_uint2(tBase, tBits | kGroupPrims);
          stack[sp++] = make_uint2(0xFFFFFFFFu, kGroupMarker);
          inBlas = true;
          curInst = prim;
          rayInit(ray, o2, d2, true);
          gBase = (uint32_t)lp.meshes[in.mesh].root;
          gHits = 1u << (0u ^ ray.rayOct);
          gImask = 1u;
          tBits = 0;
          break;
        }
        if (COUNT) cnt->quadTests++;
        QHits qh = hitQuadric(in.kind, o2, d2, tmin, tmax);
        for (int k = 0; k < qh.n; k++) {
          const QHit& q = qh.h[k];
          if (q.t >= tmax) continue;
          bool front = dot(q.n, d2) < 0.0f;
          if ((in.flags & kInstMasked) && !faceAccepts(lp, in, front, q.u, q.v)) continue;
          if (SHADOW) {
            if (!(in.flags & kInstTransmissive)) return false;
            uint16_t mid = front ? (uint16_t)(in.mats & 0xFFFF) : (uint16_t)(in.mats >> 16);
            ShadePt spt = quadShade(in, q.n, q.u, q.v, D);
            if (!shadowCross(lp, spt, mid, q.t, D, trProd, tau)) return false;
          } else {
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
        }
        continue;
      }
      // Triangle of the current BLAS, in object space.
      const float4* tp = lp.tris + 3 * (size_t)prim;
      float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
      if (COUNT) cnt->triTests++;
      float t, b1, b2;
      float3 p0 = v3(a.x, a.y, a.z), p1 = v3(b.x, b.y, b.z), p2 = v3(c.x, c.y, c.z);
      if (!wtHit(ray.wt, ray.o, p0, p1, p2, tmin, tmax, t, b1, b2)) continue;
      int tri = __float_as_int(a.w);
      const SdInstance& in = lp.inst[curInst];
      if (!(in.flags & (kInstMasked | kInstTransmissive))) {
        if (SHADOW) return false;
        tmax = t;
        found = true;
        hit.t = t;
        hit.inst = curInst;
        hit.prim = tri;
        hit.u = b1;
        hit.v = b2;
        hit.front = dot(cross(p1 - p0, p2 - p0), ray.d) < 0.0f;
        continue;
      }
      ShadePt spt = triShade(lp, in, tri, b1, b2, D);
      if ((in.flags & kInstMasked) && !faceAccepts(lp, in, spt.front, spt.u, spt.v)) continue;
      if (SHADOW) {
        if (!(in.flags & kInstTransmissive)) return false;
        uint16_t mid = spt.front ? (uint16_t)(in.mats & 0xFFFF) : (uint16_t)(in.mats >> 16);
        if (!shadowCross(lp, spt, mid, t, D, trProd, tau)) return false;
      } else {
        tmax = t;
        found = true;
        hit.t = t;
        hit.inst = curInst;
        hit.prim = tri;
        hit.u = b1;
        hit.v = b2;
        hit.front = spt.front;
      }
    }
    if (gHits || tBits) continue;
    // Both groups exhausted: take the next entry.
    bool done = true;
    while (sp > 0) {
      uint2 e = stack[--sp];
      if (e.y & kGroupMarker) {
        inBlas = false;
        rayInit(ray, O, D, false);
        continue;
      }
      if (e.y & kGroupPrims) {
        tBase = e.x;
        tBits = e.y & 0xFFFFFFu;
      } else {
        gBase = e.x;
        gHits = e.y & 0xFFu;
        gImask = (e.y >> 8) & 0xFFu;
      }
      done = false;
      break;
    }
    if (done) break;
  }
  return SHADOW ? true : found;
}

#else
// One ray's walk over the binary two-level BVH, advanced one action at a
// time by binTravStep: a node visit (both child boxes) or a leaf (a TLAS
// instance: quadric roots or entry into its BLAS; or a BLAS leaf's
// triangles), each followed by a pop when nothing is left to descend into.
// traverse() runs it to the end for one ray; the wavefront trace stage
// (wavefront.cu) interleaves many rays' walks per warp with dynamic ray
// fetch. Both visit the same nodes in the same order.
//
// The walk's scalars; its stack is a separate per-thread array (an aggregate
// holding an indexed array would be placed whole in local memory, scalars
// included).
struct BinTrav {
  float3 ro, rd, id, oi;  // the current space's ray: world in the TLAS, object in a BLAS
  WtRay wr;               // watertight-test constants of rd (inside a BLAS)
  float tmax;             // closest accepted hit so far (radiance) / the segment's end
  int cur, sp, curInst;
  bool inBlas;
};
typedef int TravStack[kStackSize];

__device__ __forceinline__ void binTravStart(BinTrav& t, const SdLaunch& lp, float3 o, float3 d,
                                             float tmax) {
  t.ro = o;
  t.rd = d;
  t.id = v3(safeInv(d.x), safeInv(d.y), safeInv(d.z));
  t.oi = o * t.id;
  t.tmax = tmax;
  t.sp = 0;
  t.inBlas = false;
  t.curInst = -1;
  t.cur = lp.numInstances > 0 ? lp.tlasRoot : kPop;
}

// Outcome of one step.
constexpr int kTravDone = 0;      // every node visited
constexpr int kTravMore = 1;      // more steps to take
constexpr int kTravOccluded = 2;  // shadow rays: an opaque crossing

// Takes the next stack entry into t.cur, the step that ends a node or a leaf
// with nothing left to descend into (done in that same step, so no loop
// iteration is spent on a pop alone). A BLAS marker restores the world ray
// and the entry below it is taken (a TLAS entry: BLASes do not nest).
// Returns kTravDone when the stack is empty.
template <class Sink>
__device__ __forceinline__ int binTravPop(BinTrav& t, TravStack& stack, Sink& sink) {
  if (t.sp == 0) return kTravDone;
  int c = stack[--t.sp];
  if (c == kToTlas) {
    t.inBlas = false;
    sink.world(t.ro, t.rd);
    t.id = v3(safeInv(t.rd.x), safeInv(t.rd.y), safeInv(t.rd.z));
    t.oi = t.ro * t.id;
    if (t.sp == 0) return kTravDone;
    c = stack[--t.sp];
  }
  t.cur = c;
  return kTravMore;
}

// One action of the walk. The sink receives what the walk finds and owns
// the world ray: sink.world(ro, rd) restores it when the walk leaves a BLAS,
// sink.worldDir() is the world direction for shading a candidate, and
// (radiance rays) sink.hit(t, inst, prim, u, v, nq, front) takes each closer
// accepted hit, t.tmax already lowered to it. Shadow rays multiply the
// transparent crossings' Fresnel transmission into trProd and add their
// signed optical depth into tau.
template <bool SHADOW, bool COUNT, class Sink>
__device__ __forceinline__ int binTravStep(BinTrav& t, TravStack& stack, const SdLaunch& lp,
                                           Sink& sink, float& trProd, float3& tau,
                                           TraceCount* cnt) {
  const float tmin = 0.0f;
  if (COUNT) countWarp(cnt, cnt->travIters, cnt->travLanes);
#if SDB_BVH4
  if (t.cur >= 0) {
    // Four child boxes; the nearest hit child next, the other hits pushed
    // (farthest first for radiance rays).
    const float4* np = reinterpret_cast<const float4*>(lp.nodes4 + t.cur);
    if (COUNT) cnt->boxTests += 4;
    const float inf = __int_as_float(0x7f800000);
    float d0, d1, d2, d3;
    {
      BvhNode pr;
      pr.xy0 = __ldg(np);
      pr.xy1 = __ldg(np + 1);
      pr.zz = __ldg(np + 2);
      bool h0, h1;
      boxPair(pr, t.oi, t.id, tmin, t.tmax, d0, d1, h0, h1);
      d0 = h0 ? d0 : inf;
      d1 = h1 ? d1 : inf;
    }
    {
      BvhNode pr;
      pr.xy0 = __ldg(np + 3);
      pr.xy1 = __ldg(np + 4);
      pr.zz = __ldg(np + 5);
      bool h2, h3;
      boxPair(pr, t.oi, t.id, tmin, t.tmax, d2, d3, h2, h3);
      d2 = h2 ? d2 : inf;
      d3 = h3 ? d3 : inf;
    }
    const int4 lk = __ldg(reinterpret_cast<const int4*>(np + 6));
    int l0 = lk.x, l1 = lk.y, l2 = lk.z, l3 = lk.w;
    // The nearest hit child first (three exchanges put the minimum in slot
    // 0); radiance rays also order the rest for front-to-back pops, shadow
    // rays, which stop at any opaque hit, take them as found (shadow stage
    // 119.0 -> 115.6 ms on config 2, 22.9 -> 22.5 ms on config 1).
    cswap(d0, l0, d1, l1);
    cswap(d2, l2, d3, l3);
    cswap(d0, l0, d2, l2);
    if (!SHADOW) {
      cswap(d1, l1, d3, l3);
      cswap(d1, l1, d2, l2);
    }
    if (!(d0 < inf)) return binTravPop(t, stack, sink);
    // Always room: the scene build bounds the tree depths by the stack.
    if (d3 < inf && t.sp < kStackSize) stack[t.sp++] = l3;
    if (d2 < inf && t.sp < kStackSize) stack[t.sp++] = l2;
    if (d1 < inf && t.sp < kStackSize) stack[t.sp++] = l1;
    t.cur = l0;
    return kTravMore;
  }
#endif
  if (t.cur >= 0) {
    BvhNode nd = loadNode(lp.nodes, t.cur);
    if (COUNT) cnt->boxTests += 2;
    float ta, tb;
    bool ha, hb;
    boxPair(nd, t.oi, t.id, tmin, t.tmax, ta, tb, ha, hb);
    if (ha && hb) {
      int first = nd.link.x, second = nd.link.y;
      if (tb < ta) {
        first = nd.link.y;
        second = nd.link.x;
      }
      if (t.sp < kStackSize) stack[t.sp++] = second;
      t.cur = first;
    } else if (ha) {
      t.cur = nd.link.x;
    } else if (hb) {
      t.cur = nd.link.y;
    } else {
      return binTravPop(t, stack, sink);
    }
    return kTravMore;
  }
  if (t.cur == kPop) return binTravPop(t, stack, sink);  // a walk with no TLAS
  // Leaf: ~cur = start << 3 | (count - 1).
  const int code = ~t.cur;
  const int start = code >> 3;
  const int count = (code & 7) + 1;
  if (!t.inBlas) {
    // TLAS leaves hold exactly one instance; ro, rd are the world ray here.
    const SdInstance& in = lp.inst[start];
    float3 o2 = xfPoint(in.w2o, t.ro), d2 = xfVec(in.w2o, t.rd);
    if (in.kind == GK_MESH) {
      if (COUNT) cnt->blasEntries++;
      // Always room: the scene build bounds TLAS + BLAS depth by the stack.
      if (t.sp < kStackSize) {
        stack[t.sp++] = kToTlas;
        t.inBlas = true;
        t.curInst = start;
        t.ro = o2;
        t.rd = d2;
        t.id = v3(safeInv(d2.x), safeInv(d2.y), safeInv(d2.z));
        t.oi = o2 * t.id;
        t.wr = wtSetup(d2);
        t.cur = lp.meshes[in.mesh].root;
        return kTravMore;
      }
      return binTravPop(t, stack, sink);
    }
    if (COUNT) cnt->quadTests++;
    QHits qh = hitQuadric(in.kind, o2, d2, tmin, t.tmax);
    for (int k = 0; k < qh.n; k++) {
      const QHit& q = qh.h[k];
      if (q.t >= t.tmax) continue;
      bool front = dot(q.n, d2) < 0.0f;
      if ((in.flags & kInstMasked) && !faceAccepts(lp, in, front, q.u, q.v)) continue;
      if (SHADOW) {
        if (!(in.flags & kInstTransmissive)) return kTravOccluded;
        uint16_t mid = front ? (uint16_t)(in.mats & 0xFFFF) : (uint16_t)(in.mats >> 16);
        ShadePt spt = quadShade(in, q.n, q.u, q.v, sink.worldDir());
        if (!shadowCross(lp, spt, mid, q.t, sink.worldDir(), trProd, tau)) return kTravOccluded;
      } else {
        t.tmax = q.t;
        sink.hit(q.t, start, 0, q.u, q.v, q.n, front);
      }
    }
    return binTravPop(t, stack, sink);
  }
  // BLAS leaf: triangles in object space of curInst.
  for (int k = 0; k < count; k++) {
    const float4* tp = lp.tris + 3 * (size_t)(start + k);
    float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
    if (COUNT) cnt->triTests++;
    float tt, b1, b2;
    float3 p0 = v3(a.x, a.y, a.z), p1 = v3(b.x, b.y, b.z), p2 = v3(c.x, c.y, c.z);
    if (!wtHit(t.wr, t.ro, p0, p1, p2, tmin, t.tmax, tt, b1, b2)) continue;
    const int prim = __float_as_int(a.w);
    const SdInstance& in = lp.inst[t.curInst];
    if (!(in.flags & (kInstMasked | kInstTransmissive))) {
      if (SHADOW) return kTravOccluded;
      t.tmax = tt;
      sink.hit(tt, t.curInst, prim, b1, b2, v3(0.0f), dot(cross(p1 - p0, p2 - p0), t.rd) < 0.0f);
      continue;
    }
    ShadePt spt = triShade(lp, in, prim, b1, b2, sink.worldDir());
    if ((in.flags & kInstMasked) && !faceAccepts(lp, in, spt.front, spt.u, spt.v)) continue;
    if (SHADOW) {
      if (!(in.flags & kInstTransmissive)) return kTravOccluded;
      uint16_t mid = spt.front ? (uint16_t)(in.mats & 0xFFFF) : (uint16_t)(in.mats >> 16);
      if (!shadowCross(lp, spt, mid, tt, sink.worldDir(), trProd, tau)) return kTravOccluded;
    } else {
      t.tmax = tt;
      sink.hit(tt, t.curInst, prim, b1, b2, v3(0.0f), spt.front);
    }
  }
  return binTravPop(t, stack, sink);
}

// Sink of a single traversal call: the world ray in registers, the closest
// hit into a TraceHit.
struct RegisterSink {
  float3 O, D;
  TraceHit* out;
  bool found;
  __device__ __forceinline__ void world(float3& ro, float3& rd) const {
    ro = O;
    rd = D;
  }
  __device__ __forceinline__ float3 worldDir() const { return D; }
  __device__ __forceinline__ void hit(float t, int inst, int prim, float u, float v, float3 nq,
                                      bool front) {
    found = true;
    out->t = t;
    out->inst = inst;
    out->prim = prim;
    out->u = u;
    out->v = v;
    out->nq = nq;
    out->front = front;
  }
};

// SHADOW = false: closest accepted hit, returns whether one was found.
// SHADOW = true: returns false when occluded, else accumulates the
// transparent-crossing terms into trProd / tau.
template <bool SHADOW, bool COUNT = false>
__device__ SDB_TRAVERSE_INLINE bool traverse(const SdLaunch& lp, float3 O, float3 D, float tmax,
                                             TraceHit& hit, float& trProd, float3& tau,
                                             TraceCount* cnt = nullptr) {
  if (COUNT) cnt->traces++;
  if (lp.numInstances == 0) return SHADOW;
  BinTrav t;
  TravStack stack;
  binTravStart(t, lp, O, D, tmax);
  RegisterSink sink{O, D, &hit, false};
  int r;
  do {
    r = binTravStep<SHADOW, COUNT>(t, stack, lp, sink, trProd, tau, cnt);
  } while (r == kTravMore);
  if (SHADOW) return r == kTravDone;
  return sink.found;
}

#endif
}  // namespace sdb
