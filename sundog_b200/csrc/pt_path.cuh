// Per-path device code shared by the path kernels: camera sample, one path
// segment (trace, media, surface or escape, NEE, BSDF sample, roulette),
// AOV and radiance bookkeeping. Restates device/programs.cu:311-572 (cited
// inline).
#pragma once

#include "kernels.h"
#include "sd_bsdf.cuh"
#include "sd_guide.cuh"
#include "sd_lights.cuh"
#include "sd_trace.cuh"
#include "sd_volume.cuh"

namespace sdb {

__device__ __forceinline__ float3 sanitize3(float3 c) {
  if (!isfinite(c.x) || !isfinite(c.y) || !isfinite(c.z)) return v3(0.0f);
  return c;
}

__device__ __forceinline__ float3 background(const SdLaunch& lp, float3 dir) {
  if (lp.bgKind == BG_ENVMAP) return envRadiance(lp.env, dir);
  if (lp.bgKind == BG_GRADIENT) {
    float t = 0.5f * (dir.y + 1.0f);
    return lp.bgA + (lp.bgB - lp.bgA) * t;
  }
  return lp.bgA;
}

// Straight-line transmittance toward a light (device/programs.cu:70-85).
template <bool COUNT>
__device__ __forceinline__ float3 shadowTransmittance(const SdLaunch& lp, float3 o, float3 d,
                                                      float tmax, TraceCount* cnt) {
  TraceHit dummy;
  float trProd = 1.0f;
  float3 tau = v3(0.0f);
  if (!traverse<true, COUNT>(lp, o, d, tmax, dummy, trProd, tau, cnt)) return v3(0.0f);
  tau = v3(fmaxf(0.0f, tau.x), fmaxf(0.0f, tau.y), fmaxf(0.0f, tau.z));
  float3 tr = v3(trProd);
  if (hmax(tau) > 0.0f) tr = tr * vexp(-tau);
  return tr;
}

struct Path {
  float3 o, d, beta, L, prevX;
  float prevPdf;
  Pcg rng;
  unsigned long long med;  // medium stack: 4 x 16-bit material ids
  int medDepth;
  int depth;
  int pixel;
  int s;
  int slot;
  bool specular;
};

__device__ __forceinline__ uint16_t medAt(unsigned long long med, int i) {
  return (uint16_t)((med >> (16 * i)) & 0xFFFFull);
}

// Camera sample s of pixel (px, py): jittered (stratified while s < n^2)
// position, thin-lens origin, initial path state. The random stream depends
// only on (pixel, s, seed). (device/programs.cu:312-357)
__device__ __forceinline__ void startPathAt(const SdLaunch& lp, int px, int py, int s, Path& p) {
  int pixel = py * lp.width + px;
  p.pixel = pixel;
  p.s = s;
  p.rng = Pcg::seeded(((unsigned long long)pixel << 32) ^ (unsigned long long)s,
                      (unsigned long long)lp.seed);
  int ns = lp.nStrata;
  float jx, jy;
  if (s < ns * ns) {
    jx = ((s % ns) + p.rng.uni()) / ns;
    jy = ((s / ns) + p.rng.uni()) / ns;
  } else {
    jx = p.rng.uni();
    jy = p.rng.uni();
  }
  float u = (px + jx) / lp.width;
  float v = ((lp.height - 1 - py) + jy) / lp.height;
  const SdCamera& cam = lp.cam;
  float3 org = cam.origin;
  if (cam.lensRadius > 0.0f) {
    float2 rd = diskConcentric(p.rng.uni2());
    rd.x *= cam.lensRadius;
    rd.y *= cam.lensRadius;
    org = org + cam.u * rd.x + cam.v * rd.y;
  }
  p.d = unit(cam.lowerLeft + u * cam.horizontal + v * cam.vertical - org);
  p.o = org;
  p.prevX = org;
  p.L = v3(0.0f);
  p.beta = v3(1.0f);
  p.prevPdf = 0.0f;
  p.specular = true;
  p.med = 0ull;
  p.medDepth = 0;
  p.depth = 0;
}

// Camera sample for path index id; false if the index is tile padding.
__device__ __forceinline__ bool startPath(const SdLaunch& lp, unsigned long long id, Path& p) {
  int sLocal, px, py;
  if (lp.shardCount > 1) {
    sLocal = (int)(id / (unsigned long long)lp.shardPad);
    int rem = (int)(id - (unsigned long long)sLocal * lp.shardPad);
    int tile = (rem >> 12) * lp.shardCount + lp.shardIndex;
    int block = (rem >> 6) & 63, within = rem & 63;
    px = (tile % lp.shardTilesX) * 64 + (block & 7) * 8 + (within & 7);
    py = (tile / lp.shardTilesX) * 64 + (block >> 3) * 8 + (within >> 3);
  } else {
    int rem;
    if (id < (1ull << 32)) {  // a 32-bit division: the common case, far cheaper
      const unsigned id32 = (unsigned)id;
      sLocal = (int)(id32 / (unsigned)lp.npixPad);
      rem = (int)(id32 - (unsigned)sLocal * (unsigned)lp.npixPad);
    } else {
      sLocal = (int)(id / (unsigned long long)lp.npixPad);
      rem = (int)(id - (unsigned long long)sLocal * lp.npixPad);
    }
    int tile = rem >> 6, within = rem & 63;
    int tx = tile % lp.tilesX, ty = tile / lp.tilesX;
    px = tx * 8 + (within & 7);
    py = ty * 8 + (within >> 3);
  }
  if (px >= lp.width || py >= lp.height) return false;
  startPathAt(lp, px, py, lp.sampleOffset + sLocal, p);
  p.slot = sLocal * (lp.width * lp.height) + py * lp.width + px;
  return true;
}

__device__ __forceinline__ void addClamped(const SdLaunch& lp, Path& p, float3 c) {
  if (p.depth >= 1 && lp.clampVal > 0.0f) c = vmin(c, v3(lp.clampVal));
  p.L += c;
}

__device__ __forceinline__ void writeAov(const SdLaunch& lp, const Path& p, float3 alb, float3 nrm) {
  if (!lp.aovOn) return;
  lp.sampleAlb[p.slot] = make_float4(alb.x, alb.y, alb.z, 1.0f);
  lp.sampleNrm[p.slot] = make_float4(nrm.x, nrm.y, nrm.z, 1.0f);
}

// State of a surface vertex between the two halves of a path segment: the
// shading point, and the next-event estimate waiting for its shadow ray.
struct Vertex {
  float3 x, ns, albedo;
  float etaExt, etaRel;
  int matId;
  bool front;
  bool nee;            // a shadow ray toward (so, wi, tmaxS) is pending
  int lightK;          // NEE strategy (light index, or numLights for the env)
  float3 so, wi, Li;
  float tmaxS, pdf, cosS;
  bool delta;
};

// First half of a path segment, after its radiance ray was traced (hit,
// h): media, flames, escape, surface shading, emission, and the NEE light
// draw. Returns false when the path has ended; otherwise v holds the vertex
// and, if v.nee, the shadow ray to trace. (device/programs.cu:374-495)
template <bool COUNT>
__device__ __forceinline__ bool shadeVertex(const SdLaunch& lp, Path& p, bool hit,
                                            const TraceHit& h, unsigned long long& rays,
                                            Vertex& v) {
  const bool hasEnv = lp.bgKind == BG_ENVMAP;
  const int nStrat = lp.numLights + (hasEnv ? 1 : 0);

  if (p.medDepth > 0) {
    int top = min(p.medDepth, 4) - 1;
    float3 sigma = lp.materials[medAt(p.med, top)].absorb;
    if (hmax(sigma) > 0.0f) p.beta *= vexp(-sigma * (hit ? h.t : 1e4f));
  }

  if (lp.numFlames > 0) {
    float3 trans = v3(1.0f);
    float3 Lv = flameMarch(lp.flames, lp.numFlames, p.o, p.d, hit ? h.t : 1e16f, p.rng, trans);
    addClamped(lp, p, p.beta * Lv);
    p.beta *= trans;
  }

  if (!hit) {
    float3 bg = background(lp, p.d);
    float w = 1.0f;
    if (hasEnv && !p.specular) {
      float pdfE = envDensity(lp.env, p.d) / nStrat;
      w = p.prevPdf / (p.prevPdf + pdfE);
    }
    addClamped(lp, p, p.beta * bg * w);
    if (p.depth == 0) writeAov(lp, p, v3(fminf(bg.x, 1.0f), fminf(bg.y, 1.0f), fminf(bg.z, 1.0f)), v3(0.0f));
    return false;
  }

  const SdInstance& in = lp.inst[h.inst];
  ShadePt sp = in.kind == GK_MESH ? triShade(lp, in, h.prim, h.u, h.v, p.d)
                                  : quadShade(in, h.nq, h.u, h.v, p.d);
  bool front = h.front;
  int matId = front ? (int)(in.mats & 0xFFFF) : (int)(in.mats >> 16);
  float3 ns = front ? sp.nFront : -sp.nFront;
  float3 x = p.o + h.t * p.d;
  const SdMaterial mat = lp.materials[matId];
  float3 albedo = surfaceAlbedo(mat, lp.textures, sp.u, sp.v);
  if (mat.kind == MT_WATER && mat.waveAmp > 0.0f)
    ns = waveNormal(x, ns, -p.d, mat.waveAmp, mat.waveFreq);

  if (p.depth == 0) {
    const SdCamera& cam = lp.cam;
    writeAov(lp, p, albedo, v3(dot(ns, cam.u), dot(ns, cam.v), dot(ns, cam.w)));
  }

  if (mat.kind == MT_EMISSIVE) {
    if (front || mat.twoSided) {
      float3 Le = albedo * mat.intensity;
      float w = 1.0f;
      if (!p.specular && in.lightId >= 0 && lp.numLights > 0) {
        float pdfL = lightDensity(lp.lights[in.lightId], p.prevX, x, ns) / nStrat;
        w = p.prevPdf / (p.prevPdf + pdfL);
      }
      addClamped(lp, p, p.beta * Le * w);
    }
    return false;
  }

  // Relative index at this interface from the medium stack.
  float etaExt = 1.0f;
  if (mat.kind == MT_DIELECTRIC || mat.kind == MT_WATER) {
    int outer = min(front ? p.medDepth : p.medDepth - 1, 4);
    if (outer > 0) etaExt = lp.materials[medAt(p.med, outer - 1)].ior;
  }
  v.x = x;
  v.ns = ns;
  v.albedo = albedo;
  v.etaExt = etaExt;
  v.etaRel = front ? etaExt / mat.ior : mat.ior / etaExt;
  v.matId = matId;
  v.front = front;
  v.nee = false;

  // Next-event estimation with the balance heuristic: the light draw here,
  // the shadow ray and the contribution in finishVertex.
  if (nStrat > 0 && !isDeltaMaterial(mat)) {
    int k = min((int)(p.rng.uni() * nStrat), nStrat - 1);
    LightDraw ls = k < lp.numLights ? lightDraw(lp.lights[k], x, p.rng, lp.textures)
                                    : envDraw(lp.env, p.rng);
    float cosS = ls.ok ? dot(ls.wi, ns) : 0.0f;
    bool transmitNee = cosS < 0.0f && mat.kind == MT_DIELECTRIC;
    if (ls.ok && (cosS > 0.0f || transmitNee)) {
      rays++;
      v.nee = true;
      v.lightK = k;
      v.so = nudge(x, transmitNee ? -ns : ns);
      v.wi = ls.wi;
      v.Li = ls.Li;
      v.tmaxS = ls.dist * 0.999f;
      v.pdf = ls.pdf;
      v.cosS = cosS;
      v.delta = ls.delta;
    }
  }
  return true;
}

// Second half of a path segment: the NEE contribution given the shadow
// ray's transmittance tr, the BSDF sample, the medium stack and Russian
// roulette. Returns false when the path has ended. GUIDE selects the guided
// variants (kGuideSample: draw by MIS with the guide; kGuideRecord: keep
// training vertices in *trail); 0 is the reference's sampler.
// (device/programs.cu:495-558)
template <int GUIDE = 0>
__device__ __forceinline__ bool finishVertex(const SdLaunch& lp, Path& p, const Vertex& v,
                                             float3 tr, GuideTrail* trail = nullptr) {
  const bool hasEnv = lp.bgKind == BG_ENVMAP;
  const int nStrat = lp.numLights + (hasEnv ? 1 : 0);
  const SdMaterial mat = lp.materials[v.matId];
  const float3 x = v.x, ns = v.ns, albedo = v.albedo;

  if (v.nee && hmax(tr) > 0.0f) {
    if (lp.numFlames > 0 && lp.transparentShadows) {
      int skip = v.lightK < lp.numLights ? lp.lights[v.lightK].flameId : -1;
      tr = tr * flameShadow(lp.flames, lp.numFlames, v.so, v.wi, v.tmaxS, p.rng, skip);
    }
    float pdfLe = (v.delta ? 1.0f : v.pdf) / nStrat;
    float3 f = bsdfValue(mat, albedo, -p.d, v.wi, ns, v.etaRel);
    float w = 1.0f;
    if (!v.delta) {
      float pdfB = bsdfDensity(mat, -p.d, v.wi, ns, v.etaRel);
      w = pdfLe / (pdfLe + pdfB);
    }
    float3 c = p.beta * f * fabsf(v.cosS) * v.Li * w / pdfLe;
    c = c * tr;
    if (p.depth >= 1 && lp.clampVal > 0.0f) c = vmin(c, v3(lp.clampVal));
    p.L += sanitize3(c);
  }

  BsdfDraw bs;
  float pdfSample;  // density wi was drawn with (differs from bs.pdf when guided)
  if ((GUIDE & kGuideSample) && guideEligible(mat)) {
    GuidedDraw gd = guidedDraw(lp, mat, albedo, p.d, ns, v.front, v.etaExt, v.etaRel, x, p.rng);
    bs = gd.s;
    pdfSample = gd.pdfSample;
  } else {
    bs = bsdfDraw(mat, albedo, p.d, ns, v.front, v.etaExt, p.rng);
    pdfSample = bs.pdf;
  }
  if (!bs.ok) return false;
  if ((mat.kind == MT_WATER || mat.kind == MT_DIELECTRIC) && dot(bs.wi, ns) < 0.0f) {
    if (v.front) {
      if (p.medDepth < 4) {
        unsigned long long sh = 16ull * p.medDepth;
        p.med = (p.med & ~(0xFFFFull << sh)) | ((unsigned long long)v.matId << sh);
      }
      p.medDepth++;
    } else if (p.medDepth > 0) {
      p.medDepth--;
    }
  }
  if ((GUIDE & kGuideRecord) && !bs.delta && guideEligible(mat))
    guideRecord(*trail, x, ns, bs.wi, pdfSample, p.beta * bs.weight, p.L);
  p.beta *= bs.weight;
  p.specular = bs.delta;
  p.prevPdf = bs.delta ? 0.0f : bs.pdf;
  p.prevX = x;
  float3 offN = dot(bs.wi, ns) >= 0.0f ? ns : -ns;
  p.o = nudge(x, offN);
  p.d = bs.wi;

  if (p.depth >= 4) {
    float q = clampf(hmax(p.beta), 0.05f, 0.95f);
    if (p.rng.uni() >= q) return false;
    p.beta *= 1.0f / q;
  }
  if (hmax(p.beta) <= 0.0f) return false;
  p.depth++;
  return p.depth < lp.maxDepth;
}

// One segment of the path for the persistent kernels: the radiance ray,
// shadeVertex, the shadow ray and finishVertex -- the same functions the
// wavefront stages call, in the same order with the same random draws, so
// both engines trace the same samples. Returns false when the path has
// ended. GUIDE selects the guided variants (kGuideSample: draw by MIS with
// the guide; kGuideRecord: keep training vertices in *trail); 0 is the
// reference's sampler. (device/programs.cu:374-558)
template <bool COUNT, int GUIDE = 0>
__device__ __forceinline__ bool bounce(const SdLaunch& lp, Path& p, unsigned long long& rays,
                                       TraceCount* cnt, GuideTrail* trail = nullptr) {
  TraceHit h;
  float dummyTr = 1.0f;
  float3 dummyTau = v3(0.0f);
  const bool hit = traverse<false, COUNT>(lp, p.o, p.d, 1e16f, h, dummyTr, dummyTau, cnt);
  rays++;
  Vertex v;
  if (!shadeVertex<COUNT>(lp, p, hit, h, rays, v)) return false;
  float3 tr = v3(0.0f);
  // Counting build: shadow traversals go to the second counter set.
  if (v.nee) tr = shadowTransmittance<COUNT>(lp, v.so, v.wi, v.tmaxS, COUNT ? cnt + 1 : nullptr);
  return finishVertex<GUIDE>(lp, p, v, tr, trail);
}

}  // namespace sdb
