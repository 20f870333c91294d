// Device self-tests: run one hot-path function over a batch of host-supplied
// inputs on the GPU and return the outputs, so the parity tests can compare
// the sm_100a code with the CPU oracle item by item. Item layouts are the
// packed structs below (all 4-byte fields, little endian).
#include <cstring>
#include <stdexcept>
#include <vector>

#include "../../include/sundog_api.h"
#include "cdf_build.h"
#include "abi_util.h"
#include "bvh_build.h"
#include "render_session.h"
#include "sd_bsdf.cuh"
#include "sd_lights.cuh"
#include "sd_quadric.cuh"
#include "sd_trace.cuh"
#include "sd_volume.cuh"

namespace sdb {

// 1: PCG32 stream. in {u64 seed, u64 seq}; out {u32 next[8], f32 uni[4]}
struct StPcgIn { unsigned long long seed, seq; };
struct StPcgOut { unsigned int next[8]; float uni[4]; };
// 2: BSDF value + density. in {mat, albedo, wo, wi, n, eta}; out {f, pdf}
struct StEvalIn { SdMaterial m; float3 albedo, wo, wi, n; float eta; };
struct StEvalOut { float3 f; float pdf; };
// 3: BSDF draw. in {mat, albedo, d, n, front, etaExt, rng}; out {...}
struct StDrawIn { SdMaterial m; float3 albedo, d, n; int front; float etaExt; unsigned long long state, inc; };
struct StDrawOut { float3 wi, weight; float pdf; int delta, ok; unsigned int pad; unsigned long long state; };
// 4: quadric roots. in {kind, o, d, tmin, tmax}; out {count, 2 x (t, n, u, v)}
struct StQuadIn { int kind; float3 o, d; float tmin, tmax; };
struct StQuadOut { int count; float t0; float3 n0; float u0, v0, t1; float3 n1; float u1, v1; };
// 5: watertight triangle. in {o, d, p0, p1, p2, tmin, tmax}; out {hit, t, b1, b2}
struct StTriIn { float3 o, d, p0, p1, p2; float tmin, tmax; };
struct StTriOut { int hit; float t, b1, b2; };
// 6: explicit light draw (non-mesh lights). in {light, x, rng}; out {...}
struct StLightIn { SdLight l; float3 x; unsigned long long state, inc; };
struct StLightOut { float3 wi, Li; float dist, pdf; int delta, ok; unsigned long long state; float density; float pad; };
// 7: flame march + shadow twin. in {flame, o, d, tEnd, rng, skip}; out {Lv, trans, tr, states}
struct StFlameIn { SdFlame f; float3 o, d; float tEnd; int skip; unsigned long long state, inc; };
struct StFlameOut { float3 Lv, trans; float tr; int pad; unsigned long long stateMarch, stateShadow; };
// 8: noise. in {p, seed, ns, wo, amp, freq}; out {fbm, vnoise, waveNormal}
struct StNoiseIn { float3 p; unsigned seed; float3 ns, wo; float amp, freq; };
struct StNoiseOut { float fbm, vnoise; float3 wave; };
// 9: CDF search. in {u}; shared cdf passed as a second block; out {index}
// 10: bilinear filter of a float4 grid. in {u, v}; out {rgba}
// 11: CDF search through the CDF's guide (built on the device from the
//     shared cdf, as for the environment's tables). in {u}; out {index}

__global__ void stKernel(int which, const void* in, int n, void* out, const float* aux, int auxN,
                         int auxW, int auxH, const int* guide) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  switch (which) {
    case 1: {
      const StPcgIn& a = ((const StPcgIn*)in)[i];
      StPcgOut& o = ((StPcgOut*)out)[i];
      Pcg g = Pcg::seeded(a.seed, a.seq);
      for (int k = 0; k < 8; k++) o.next[k] = g.next();
      for (int k = 0; k < 4; k++) o.uni[k] = g.uni();
      break;
    }
    case 2: {
      const StEvalIn& a = ((const StEvalIn*)in)[i];
      StEvalOut& o = ((StEvalOut*)out)[i];
      o.f = bsdfValue(a.m, a.albedo, a.wo, a.wi, a.n, a.eta);
      o.pdf = bsdfDensity(a.m, a.wo, a.wi, a.n, a.eta);
      break;
    }
    case 3: {
      const StDrawIn& a = ((const StDrawIn*)in)[i];
      StDrawOut& o = ((StDrawOut*)out)[i];
      Pcg g;
      g.state = a.state;
      g.inc = a.inc;
      BsdfDraw s = bsdfDraw(a.m, a.albedo, a.d, a.n, a.front != 0, a.etaExt, g);
      o.wi = s.wi;
      o.weight = s.weight;
      o.pdf = s.pdf;
      o.delta = s.delta;
      o.ok = s.ok;
      o.pad = 0;
      o.state = g.state;
      break;
    }
    case 4: {
      const StQuadIn& a = ((const StQuadIn*)in)[i];
      StQuadOut& o = ((StQuadOut*)out)[i];
      QHits h = hitQuadric(a.kind, a.o, a.d, a.tmin, a.tmax);
      o.count = h.n;
      o.t0 = h.n > 0 ? h.h[0].t : 0.0f;
      o.n0 = h.n > 0 ? h.h[0].n : v3(0.0f);
      o.u0 = h.n > 0 ? h.h[0].u : 0.0f;
      o.v0 = h.n > 0 ? h.h[0].v : 0.0f;
      o.t1 = h.n > 1 ? h.h[1].t : 0.0f;
      o.n1 = h.n > 1 ? h.h[1].n : v3(0.0f);
      o.u1 = h.n > 1 ? h.h[1].u : 0.0f;
      o.v1 = h.n > 1 ? h.h[1].v : 0.0f;
      break;
    }
    case 5: {
      const StTriIn& a = ((const StTriIn*)in)[i];
      StTriOut& o = ((StTriOut*)out)[i];
      WtRay w = wtSetup(a.d);
      float t = 0, b1 = 0, b2 = 0;
      o.hit = wtHit(w, a.o, a.p0, a.p1, a.p2, a.tmin, a.tmax, t, b1, b2) ? 1 : 0;
      o.t = t;
      o.b1 = b1;
      o.b2 = b2;
      break;
    }
    case 6: {
      const StLightIn& a = ((const StLightIn*)in)[i];
      StLightOut& o = ((StLightOut*)out)[i];
      Pcg g;
      g.state = a.state;
      g.inc = a.inc;
      LightDraw s = lightDraw(a.l, a.x, g, nullptr);
      o.wi = s.wi;
      o.Li = s.Li;
      o.dist = s.dist;
      o.pdf = s.pdf;
      o.delta = s.delta;
      o.ok = s.ok;
      o.state = g.state;
      o.density = s.ok ? lightDensity(a.l, a.x, a.x + s.wi * s.dist, a.l.n) : 0.0f;
      o.pad = 0.0f;
      break;
    }
    case 7: {
      const StFlameIn& a = ((const StFlameIn*)in)[i];
      StFlameOut& o = ((StFlameOut*)out)[i];
      Pcg g1, g2;
      g1.state = g2.state = a.state;
      g1.inc = g2.inc = a.inc;
      float3 trans = v3(1.0f);
      o.Lv = flameMarch(&a.f, 1, a.o, a.d, a.tEnd, g1, trans);
      o.trans = trans;
      o.tr = flameShadow(&a.f, 1, a.o, a.d, a.tEnd, g2, a.skip);
      o.pad = 0;
      o.stateMarch = g1.state;
      o.stateShadow = g2.state;
      break;
    }
    case 8: {
      const StNoiseIn& a = ((const StNoiseIn*)in)[i];
      StNoiseOut& o = ((StNoiseOut*)out)[i];
      o.fbm = fbm3(a.p, a.seed);
      o.vnoise = valueNoise(a.p, a.seed);
      o.wave = waveNormal(a.p, a.ns, a.wo, a.amp, a.freq);
      break;
    }
    case 9: {
      float u = ((const float*)in)[i];
      ((int*)out)[i] = cdfSearch(aux, auxN, u);
      break;
    }
    case 10: {
      const float2 uv = ((const float2*)in)[i];
      ((float4*)out)[i] = sampleFloat4((const float4*)aux, auxW, auxH, uv.x, uv.y);
      break;
    }
    case 11: {
      float u = ((const float*)in)[i];
      ((int*)out)[i] = cdfSearchGuided(aux, auxN, guide, u);
      break;
    }
  }
}

static size_t itemIn(int which) {
  switch (which) {
    case 1: return sizeof(StPcgIn);
    case 2: return sizeof(StEvalIn);
    case 3: return sizeof(StDrawIn);
    case 4: return sizeof(StQuadIn);
    case 5: return sizeof(StTriIn);
    case 6: return sizeof(StLightIn);
    case 7: return sizeof(StFlameIn);
    case 8: return sizeof(StNoiseIn);
    case 9: return sizeof(float);
    case 10: return sizeof(float2);
    case 11: return sizeof(float);
  }
  return 0;
}
static size_t itemOut(int which) {
  switch (which) {
    case 1: return sizeof(StPcgOut);
    case 2: return sizeof(StEvalOut);
    case 3: return sizeof(StDrawOut);
    case 4: return sizeof(StQuadOut);
    case 5: return sizeof(StTriOut);
    case 6: return sizeof(StLightOut);
    case 7: return sizeof(StFlameOut);
    case 8: return sizeof(StNoiseOut);
    case 9: return sizeof(int);
    case 10: return sizeof(float4);
    case 11: return sizeof(int);
  }
  return 0;
}

}  // namespace sdb

using namespace sdb;

// Item sizes for the Python side to check its packing against.
extern "C" __attribute__((visibility("default"))) int sundog_selftest_sizes(int which, size_t* in_bytes,
                                                                            size_t* out_bytes) {
  size_t a = itemIn(which), b = itemOut(which);
  if (!a) return SUNDOG_ERROR;
  if (in_bytes) *in_bytes = a;
  if (out_bytes) *out_bytes = b;
  return SUNDOG_OK;
}

// `in` holds n items; for which = 9 / 10 / 11 the auxiliary table (cdf
// floats, or a W x H float4 grid) follows the items: int count (9, 11) or
// int W, int H (10), then the floats.
extern "C" int sundog_selftest(int which, const void* in, int n, void* out, size_t out_bytes) {
  SDB_TRY
  size_t ib = itemIn(which), ob = itemOut(which);
  if (!ib) throw std::runtime_error("selftest: unknown function id");
  if (n <= 0 || !in || !out) throw std::runtime_error("selftest: empty batch");
  if (out_bytes < ob * (size_t)n) throw std::runtime_error("selftest: output buffer too small");
  DevBuf din, dout, daux, dguide;
  din.upload(in, ib * n);
  dout.alloc(ob * n);
  int auxN = 0, auxW = 0, auxH = 0;
  if (which == 9 || which == 10 || which == 11) {
    const char* tail = (const char*)in + ib * n;
    if (which == 9 || which == 11) {
      std::memcpy(&auxN, tail, sizeof(int));
      if (auxN < 2) throw std::runtime_error("selftest: cdf needs >= 2 entries");
      daux.upload(tail + sizeof(int), (size_t)auxN * sizeof(float));
    } else {
      std::memcpy(&auxW, tail, sizeof(int));
      std::memcpy(&auxH, tail + sizeof(int), sizeof(int));
      if (auxW < 1 || auxH < 1) throw std::runtime_error("selftest: empty grid");
      daux.upload(tail + 2 * sizeof(int), (size_t)auxW * auxH * 4 * sizeof(float));
    }
  }
  if (which == 11) {
    dguide.alloc((kCdfGuide + 1) * sizeof(int));
    buildCdfGuideDevice((const float*)daux.ptr, auxN, 0, 1, (int*)dguide.ptr, 0);
  }
  stKernel<<<(n + 127) / 128, 128>>>(which, din.ptr, n, dout.ptr, (const float*)daux.ptr, auxN, auxW,
                                     auxH, (const int*)dguide.ptr);
  cudaCheck(cudaGetLastError(), "selftest launch");
  cudaCheck(cudaDeviceSynchronize(), "selftest");
  cudaCheck(cudaMemcpy(out, dout.ptr, ob * n, cudaMemcpyDeviceToHost), "selftest download");
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

// Host-side structural check of the 8-wide BVH builder over caller boxes
// (n boxes as lo.xyz, hi.xyz floats): every primitive is referenced by
// exactly one leaf slot, every decoded (quantised) child box contains the
// exact bounds of its subtree, leaf slots hold 1..3 primitives, internal
// children are contiguous. out (6 u64): nodes, max depth, leaf slots,
// internal slots, total slots tested per full sweep, failures.
extern "C" __attribute__((visibility("default"))) int sundog_bvh_validate(const float* boxes, int n,
                                                                          int leafMax,
                                                                          unsigned long long* out) {
  SDB_TRY
  std::vector<Box3> bx((size_t)n);
  for (int i = 0; i < n; i++) {
    bx[i].lo = v3(boxes[6 * i], boxes[6 * i + 1], boxes[6 * i + 2]);
    bx[i].hi = v3(boxes[6 * i + 3], boxes[6 * i + 4], boxes[6 * i + 5]);
  }
  CwBuild b = buildCw(bx, leafMax, 0, 0);
  std::vector<int> seen((size_t)n, 0);
  unsigned long long leaves = 0, inner = 0, fails = 0;
  // subtree bounds by recursion from the root
  struct Rec {
    static Box3 walk(const CwBuild& b, const std::vector<Box3>& bx, int idx, std::vector<int>& seen,
                     unsigned long long& leaves, unsigned long long& inner, unsigned long long& fails) {
      const CwNode& nd = b.nodes[idx];
      uint32_t w[4];
      std::memcpy(w, &nd.a, 16);
      uint32_t imask = w[3] >> 24;
      uint32_t bw[4];
      std::memcpy(bw, &nd.b, 16);
      Box3 all = boxEmpty();
      int innerSeen = 0;
      for (int s = 0; s < 8; s++) {
        uint32_t m = (bw[2 + (s >> 2)] >> (8 * (s & 3))) & 0xFFu;
        if (!m) continue;
        Box3 q = cwChildBox(nd, s);
        Box3 exact = boxEmpty();
        if (imask & (1u << s)) {
          inner++;
          exact = walk(b, bx, (int)bw[0] + innerSeen, seen, leaves, inner, fails);
          innerSeen++;
        } else {
          leaves++;
          int cntp = (int)(m >> 5), off = (int)(m & 31);
          if (cntp < 1 || cntp > kCwLeafMax) fails++;
          for (int k = 0; k < cntp; k++) {
            int prim = b.order[bw[1] + off + k];
            seen[prim]++;
            boxGrow(exact, bx[prim]);
          }
        }
        if (q.lo.x > exact.lo.x || q.lo.y > exact.lo.y || q.lo.z > exact.lo.z ||
            q.hi.x < exact.hi.x || q.hi.y < exact.hi.y || q.hi.z < exact.hi.z)
          fails++;
        boxGrow(all, exact);
      }
      return all;
    }
  };
  if (n > 0) Rec::walk(b, bx, 0, seen, leaves, inner, fails);
  for (int i = 0; i < n; i++)
    if (seen[i] != 1) fails++;
  out[0] = b.nodes.size();
  out[1] = (unsigned long long)b.maxDepth;
  out[2] = leaves;
  out[3] = inner;
  out[4] = leaves + inner;
  out[5] = fails;
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}
