// Learned path guiding inside the path kernel.
//
// The guiding network (guide.cu) maps a surface point and normal to a
// mixture of 8 von Mises-Fisher lobes over incident directions. After each
// training phase it is evaluated on tensor cores for every cell of a
// 32^3 grid over the region the training samples came from, times 6 normal
// directions (+-x, +-y, +-z); a shading point reads the mixture of its voxel
// and dominant normal axis. A lobe is stored as one float4
// (kappa mu.xyz, log(w kappa / (2 pi (1 - e^-2kappa))) - kappa), so the
// mixture density is sum_k exp(dot(kappa mu_k, w) + c_k).
//
// Sampling is one-sample MIS between the guide (probability guideMix) and
// the BSDF: whichever technique drew wi, the path throughput is
// f |cos| / (a q + (1 - a) p_bsdf), so every direction the BSDF reaches keeps
// its expectation whatever the network learned. The NEE and emitter-hit
// balance weights keep using the BSDF's own density p_bsdf exactly as the
// plain kernel does: those weights then still sum to one over the two
// strategies, and every term's integrand stays the plain kernel's, so a
// guided render has the plain render's expectation also where NEE and BSDF
// sampling do not partition the light cleanly (straight-line transparent
// shadows through a refracting surface). Delta and sharp lobes use the BSDF
// alone.
//
// Training records: while recording, the first kGuidePending guided vertices
// of a path keep (x, n, wi, pdf, throughput after the vertex, radiance so
// far); when the path ends each becomes a record
// (x, n, wi, luminance(L_in) |cos(wi, n)| / pdf), with the incident radiance
// along wi L_in = (L_end - L_vertex) / throughput per channel. The target
// L_in |cos| is the integrand's shape on a diffuse surface.
#pragma once

#include "guide_net.h"
#include "sd_bsdf.cuh"
#include "sd_types.h"

namespace sdb {

constexpr int kGuidePending = 4;

struct GuideVertex {
  float3 x, n, wi, beta, L;
  float pdf;
};
struct GuideTrail {
  GuideVertex v[kGuidePending];
  int n;
};

__device__ __forceinline__ int guideNormalBin(float3 n) {
  float ax = fabsf(n.x), ay = fabsf(n.y), az = fabsf(n.z);
  if (ax >= ay && ax >= az) return n.x >= 0.0f ? 0 : 1;
  if (ay >= az) return n.y >= 0.0f ? 2 : 3;
  return n.z >= 0.0f ? 4 : 5;
}

__device__ __forceinline__ int guideCellIndex(const SdLaunch& lp, float3 x, float3 n) {
  float3 q = (x - lp.guideLo) * lp.guideInvExtent;
  int ix = min(max((int)(q.x * kGuideGrid), 0), kGuideGrid - 1);
  int iy = min(max((int)(q.y * kGuideGrid), 0), kGuideGrid - 1);
  int iz = min(max((int)(q.z * kGuideGrid), 0), kGuideGrid - 1);
  return ((ix * kGuideGrid + iy) * kGuideGrid + iz) * kGuideNormals + guideNormalBin(n);
}

__device__ __forceinline__ float mixtureDensity(const float4* lobes, float3 w) {
  float q = 0.0f;
#pragma unroll
  for (int k = 0; k < kGuideLobes; k++) {
    float4 l = __ldg(lobes + k);
    q += __expf(l.x * w.x + l.y * w.y + l.z * w.z + l.w);
  }
  return q;
}

// Lobe by cumulative weight (1 draw), then a vMF direction (2 draws) by
// inverting the cosine marginal: Jakob, "Numerically stable sampling of the
// von Mises-Fisher distribution on S^2" (2012).
__device__ __forceinline__ float3 mixtureDraw(const float4* lobes, const float* cdf, Pcg& rng) {
  float u = rng.uni();
  int k = 0;
#pragma unroll
  for (int j = 0; j < kGuideLobes - 1; j++) k += u >= __ldg(cdf + j) ? 1 : 0;
  float4 l = __ldg(lobes + k);
  float3 km = v3(l.x, l.y, l.z);
  float kappa = fmaxf(len(km), 1e-6f);
  float3 mu = km * (1.0f / kappa);
  float2 r = rng.uni2();
  float c = 1.0f + __logf(r.x + (1.0f - r.x) * __expf(-2.0f * kappa)) / kappa;
  c = clampf(c, -1.0f, 1.0f);
  float s = sqrtf(fmaxf(0.0f, 1.0f - c * c));
  float phi = 2.0f * kPi * r.y;
  float sp, cp;
  __sincosf(phi, &sp, &cp);
  Frame fr(mu);
  return unit(fr.toWorld(v3(s * cp, s * sp, c)));
}

// Guided materials: diffuse-like lobes (Lambert, plastic's diffuse base,
// metal and glass with roughness >= 0.5). Sharper lobes keep BSDF sampling
// alone: there the BSDF's own sampler is close to ideal and giving half of
// the samples to a broad guide would at most halve its efficiency.
__device__ __forceinline__ bool guideEligible(const SdMaterial& m) {
  if (m.kind == MT_LAMBERT || m.kind == MT_PLASTIC) return true;
  return (m.kind == MT_METAL || m.kind == MT_DIELECTRIC) && m.roughness >= 0.5f;
}

struct GuidedDraw {
  BsdfDraw s;
  float pdfSample;
};

// One-sample MIS draw: technique choice (1 draw), then the guide's 3 draws
// or the BSDF's own. Returns the BSDF's density at wi in .s.pdf (for the MIS
// weights) and the density wi was actually drawn with in .pdfSample. Out of
// line in device code, so its registers do not weigh on the traversal loop.
static __device__ __noinline__ GuidedDraw guidedDraw(const SdLaunch& lp, const SdMaterial& m,
                                                     float3 albedo, float3 d, float3 ns,
                                                     bool front, float etaExt, float etaRel,
                                                     float3 x, Pcg& rng) {
  GuidedDraw r;
  float& pdfSample = r.pdfSample;
  const float a = lp.guideMix;
  const int cell = guideCellIndex(lp, x, ns);
  const float4* lobes = lp.guideLobes + (size_t)cell * kGuideLobes;
  BsdfDraw s;
  float3 wi;
  if (rng.uni() < a) {
    wi = mixtureDraw(lobes, lp.guideCdf + (size_t)cell * kGuideLobes, rng);
  } else {
    s = bsdfDraw(m, albedo, d, ns, front, etaExt, rng);
    if (!s.ok || s.delta) {
      pdfSample = s.pdf;
      r.s = s;
      return r;
    }
    wi = s.wi;
  }
  // Common tail for both techniques (no divergent evaluation in the warp).
  float pb = bsdfDensity(m, -d, wi, ns, etaRel);
  float3 f = bsdfValue(m, albedo, -d, wi, ns, etaRel);
  float pmix = a * mixtureDensity(lobes, wi) + (1.0f - a) * pb;
  s.wi = wi;
  s.pdf = pb;
  s.delta = false;
  s.ok = pmix > 0.0f && hmax(f) > 0.0f;
  s.weight = s.ok ? f * (fabsf(dot(wi, ns)) / pmix) : v3(0.0f);
  pdfSample = pmix;
  r.s = s;
  return r;
}

__device__ __forceinline__ void guideRecord(GuideTrail& tr, float3 x, float3 n, float3 wi,
                                            float pdf, float3 betaAfter, float3 L) {
  if (tr.n >= kGuidePending || !(pdf > 0.0f)) return;
  GuideVertex& v = tr.v[tr.n++];
  v.x = x;
  v.n = n;
  v.wi = wi;
  v.beta = betaAfter;
  v.L = L;
  v.pdf = pdf;
}

__device__ __forceinline__ float luminance(float3 c) {
  return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z;
}

// Turns a finished path's pending vertices into training records.
__device__ __forceinline__ void guideFlush(const SdLaunch& lp, GuideTrail& tr, float3 Lend) {
  for (int i = 0; i < tr.n; i++) {
    const GuideVertex& v = tr.v[i];
    float3 dL = Lend - v.L;
    float3 Li = v3(v.beta.x > 0.0f ? dL.x / v.beta.x : 0.0f,
                   v.beta.y > 0.0f ? dL.y / v.beta.y : 0.0f,
                   v.beta.z > 0.0f ? dL.z / v.beta.z : 0.0f);
    float F = luminance(Li) * fabsf(dot(v.wi, v.n)) / v.pdf;
    if (!(F > 0.0f) || !isfinite(F)) continue;
    if (!isfinite(v.x.x + v.x.y + v.x.z + v.n.x + v.n.y + v.n.z + v.wi.x + v.wi.y + v.wi.z))
      continue;
    unsigned long long k = atomicAdd(lp.guideTrainCount, 1ull);
    if (k >= lp.guideTrainCap) continue;
    float4* r = lp.guideTrain + 3 * k;
    r[0] = make_float4(v.x.x, v.x.y, v.x.z, F);
    r[1] = make_float4(v.n.x, v.n.y, v.n.z, 0.0f);
    r[2] = make_float4(v.wi.x, v.wi.y, v.wi.z, 0.0f);
  }
  tr.n = 0;
}

}  // namespace sdb
