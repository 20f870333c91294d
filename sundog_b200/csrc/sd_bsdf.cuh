// Surface scattering: Lambert, GGX metal, smooth / rough dielectric (Walter et
// al. 2007 with Heitz 2018 visible-normal sampling), plastic (GGX coat over a
// Fresnel-weighted diffuse base) and water (smooth interface).
//
// Behaviour, random-draw order and the returned weight / pdf conventions are
// those of sundog's device/bsdf.cuh (cited per function) so that the same
// seed walks the same paths. Conventions: wo points away from the surface, n
// is the shading normal on wo's side, all unit length.
#pragma once

#include "sd_rng.cuh"
#include "sd_types.h"

namespace sdb {

struct BsdfDraw {
  float3 wi;
  float3 weight;  // f |cos| / pdf, or the delta weight
  float pdf;      // solid angle; 0 for delta lobes
  bool delta;
  bool ok;
};

// device/bsdf.cuh:27-33 — water is always smooth; metal and glass below the
// roughness gate are mirrors / smooth interfaces.
SDB_HD bool isDeltaMaterial(const SdMaterial& m) {
  if (m.kind == MT_WATER) return true;
  if (m.kind == MT_DIELECTRIC || m.kind == MT_METAL) return m.roughness < 1e-3f;
  return false;
}

// ---- GGX microfacet terms (local frame, n = +Z) ---------------------------

// device/bsdf.cuh:37-45: D with the alpha^2 c^2 + (1 - c^2) grouping that
// stays positive at tiny alpha.
SDB_HD float ggxD(float3 h, float a) {
  float c2 = h.z * h.z;
  float k = a * a * c2 + (1.0f - c2);
  return a * a / (kPi * k * k);
}

// device/bsdf.cuh:47-57: Smith Lambda, G1 and the height-correlated G.
SDB_HD float ggxLambda(float3 w, float a) {
  float c2 = w.z * w.z;
  if (c2 >= 1.0f) return 0.0f;
  float t2 = (1.0f - c2) / c2;
  return 0.5f * (-1.0f + sqrtf(1.0f + a * a * t2));
}
SDB_HD float ggxG1(float3 w, float a) { return 1.0f / (1.0f + ggxLambda(w, a)); }
SDB_HD float ggxG(float3 wo, float3 wi, float a) {
  return 1.0f / (1.0f + ggxLambda(wo, a) + ggxLambda(wi, a));
}

// Visible-normal sample (Heitz 2018, "Sampling the GGX Distribution of
// Visible Normals"); wo.z > 0. (device/bsdf.cuh:60-73)
SDB_HD float3 ggxSampleVisible(float3 wo, float a, float2 u) {
  float3 vh = unit(v3(a * wo.x, a * wo.y, wo.z));
  float l2 = vh.x * vh.x + vh.y * vh.y;
  float3 T1 = l2 > 0.0f ? v3(-vh.y, vh.x, 0.0f) * (1.0f / sqrtf(l2)) : v3(1.0f, 0.0f, 0.0f);
  float3 T2 = cross(vh, T1);
  float r = sqrtf(u.x);
  float phi = 2.0f * kPi * u.y;
  float t1 = r * cosf(phi);
  float t2 = r * sinf(phi);
  float s = 0.5f * (1.0f + vh.z);
  t2 = (1.0f - s) * sqrtf(fmaxf(0.0f, 1.0f - t1 * t1)) + s * t2;
  float3 nh = t1 * T1 + t2 * T2 + sqrtf(fmaxf(0.0f, 1.0f - t1 * t1 - t2 * t2)) * vh;
  return unit(v3(a * nh.x, a * nh.y, fmaxf(1e-6f, nh.z)));
}

// Reflection pdf under visible-normal sampling, G1(wo) D(h) / (4 wo.z).
// (device/bsdf.cuh:76-80)
SDB_HD float ggxPdfReflect(float3 wo, float3 wi, float a) {
  if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
  float3 h = unit(wo + wi);
  return ggxG1(wo, a) * ggxD(h, a) / (4.0f * wo.z);
}

// Schlick at the low-index side's cosine, 1 past the critical angle.
// (device/bsdf.cuh:88-92)
SDB_HD float fresnelInterface(float cosI, float eta, float f0) {
  float k = 1.0f - eta * eta * (1.0f - cosI * cosI);
  if (k <= 0.0f) return 1.0f;
  return fresnelSchlick(eta < 1.0f ? cosI : sqrtf(k), f0);
}

// Transmission pdf: visible D times the refraction Jacobian (Walter 2007
// eq. 17, relative eta). (device/bsdf.cuh:98-105)
SDB_HD float ggxPdfTransmit(float3 lo, float3 li, float3 h, float eta, float a) {
  float loh = dot(lo, h), lih = dot(li, h);
  if (lo.z <= 0.0f || li.z >= 0.0f || loh <= 0.0f || lih >= 0.0f) return 0.0f;
  float den = eta * loh + lih;
  if (fabsf(den) < 1e-6f) return 0.0f;
  return ggxG1(lo, a) * ggxD(h, a) * loh / lo.z * fabsf(lih) / (den * den);
}

// Plastic lobes: untinted GGX coat (f0 from ior, roughness floored at 1e-3)
// plus a diffuse base scaled by (1-F(cos_o))(1-F(cos_i)); sampled as an
// equal mixture. (device/bsdf.cuh:121-143)
struct PlasticLobes {
  float fSpec;
  float3 fDiff;
  float pSpec;
  float pDiff;
};
SDB_HD PlasticLobes plasticLobes(const SdMaterial& m, float3 albedo, float3 lo, float3 li) {
  PlasticLobes t;
  float r = fmaxf(m.roughness, 1e-3f);
  float a = r * r;
  float f0 = (m.ior - 1.0f) / (m.ior + 1.0f);
  f0 = f0 * f0;
  float3 h = unit(lo + li);
  float F = fresnelSchlick(dot(lo, h), f0);
  t.fSpec = F * ggxD(h, a) * ggxG(lo, li, a) / (4.0f * lo.z * li.z);
  t.fDiff = albedo * (kInvPi * (1.0f - fresnelSchlick(lo.z, f0)) *
                      (1.0f - fresnelSchlick(li.z, f0)));
  t.pSpec = ggxPdfReflect(lo, li, a);
  t.pDiff = li.z * kInvPi;
  return t;
}

// ---- evaluation (non-delta lobes) ------------------------------------------
// eta = relative index seen from wo (frontface ? etaExt/ior : ior/etaExt);
// only the rough dielectric's transmission lobe reads it.
// (device/bsdf.cuh:151-213)
SDB_HD float3 bsdfValue(const SdMaterial& m, float3 albedo, float3 wo, float3 wi,
                        float3 n, float eta) {
  float ci = dot(wi, n);
  float co = dot(wo, n);
  if (co <= 0.0f) return v3(0.0f);
  bool roughGlass = m.kind == MT_DIELECTRIC && m.roughness >= 1e-3f;
  if (ci <= 0.0f) {
    if (!roughGlass || ci == 0.0f) return v3(0.0f);
    float a = m.roughness * m.roughness;
    Frame fr(n);
    float3 lo = fr.toLocal(wo), li = fr.toLocal(wi);
    float3 h = unit(eta * lo + li);
    if (h.z < 0.0f) h = -h;
    float loh = dot(lo, h), lih = dot(li, h);
    if (loh <= 0.0f || lih >= 0.0f) return v3(0.0f);
    float den = eta * loh + lih;
    if (fabsf(den) < 1e-6f) return v3(0.0f);
    float f0 = (1.0f - eta) / (1.0f + eta);
    f0 = f0 * f0;
    float F = fresnelInterface(loh, eta, f0);
    float ft = eta * eta * (1.0f - F) * ggxD(h, a) * ggxG(lo, li, a) *
               fabsf(loh * lih) / (lo.z * fabsf(li.z) * den * den);
    return v3(ft);
  }
  if (m.kind == MT_LAMBERT) return albedo * kInvPi;
  if (m.kind == MT_PLASTIC) {
    Frame fr(n);
    PlasticLobes t = plasticLobes(m, albedo, fr.toLocal(wo), fr.toLocal(wi));
    return v3(t.fSpec) + t.fDiff;
  }
  if (m.kind == MT_METAL && m.roughness >= 1e-3f) {
    float a = m.roughness * m.roughness;
    Frame fr(n);
    float3 lo = fr.toLocal(wo), li = fr.toLocal(wi);
    float3 h = unit(lo + li);
    float3 F = fresnelSchlick3(dot(lo, h), albedo);
    return F * (ggxD(h, a) * ggxG(lo, li, a) / (4.0f * lo.z * li.z));
  }
  if (roughGlass) {
    float a = m.roughness * m.roughness;
    Frame fr(n);
    float3 lo = fr.toLocal(wo), li = fr.toLocal(wi);
    float3 h = unit(lo + li);
    float f0 = (1.0f - eta) / (1.0f + eta);
    f0 = f0 * f0;
    float F = fresnelInterface(dot(lo, h), eta, f0);
    return v3(F * ggxD(h, a) * ggxG(lo, li, a) / (4.0f * lo.z * li.z));
  }
  return v3(0.0f);
}

// Solid-angle pdf of bsdfDraw producing wi, lobe-choice probabilities
// included. (device/bsdf.cuh:215-263)
SDB_HD float bsdfDensity(const SdMaterial& m, float3 wo, float3 wi, float3 n, float eta) {
  float ci = dot(wi, n);
  float co = dot(wo, n);
  if (co <= 0.0f) return 0.0f;
  bool roughGlass = m.kind == MT_DIELECTRIC && m.roughness >= 1e-3f;
  if (ci <= 0.0f) {
    if (!roughGlass || ci == 0.0f) return 0.0f;
    float a = m.roughness * m.roughness;
    Frame fr(n);
    float3 lo = fr.toLocal(wo), li = fr.toLocal(wi);
    float3 h = unit(eta * lo + li);
    if (h.z < 0.0f) h = -h;
    float loh = dot(lo, h);
    if (loh <= 0.0f) return 0.0f;
    float f0 = (1.0f - eta) / (1.0f + eta);
    f0 = f0 * f0;
    float F = fresnelInterface(loh, eta, f0);
    return (1.0f - F) * ggxPdfTransmit(lo, li, h, eta, a);
  }
  if (m.kind == MT_LAMBERT) return ci * kInvPi;
  if (m.kind == MT_PLASTIC) {
    Frame fr(n);
    PlasticLobes t = plasticLobes(m, v3(0.0f), fr.toLocal(wo), fr.toLocal(wi));
    return 0.5f * (t.pSpec + t.pDiff);
  }
  if (m.kind == MT_METAL && m.roughness >= 1e-3f) {
    Frame fr(n);
    return ggxPdfReflect(fr.toLocal(wo), fr.toLocal(wi), m.roughness * m.roughness);
  }
  if (roughGlass) {
    float a = m.roughness * m.roughness;
    Frame fr(n);
    float3 lo = fr.toLocal(wo), li = fr.toLocal(wi);
    float3 h = unit(lo + li);
    float f0 = (1.0f - eta) / (1.0f + eta);
    f0 = f0 * f0;
    float F = fresnelInterface(dot(lo, h), eta, f0);
    return F * ggxPdfReflect(lo, li, a);
  }
  return 0.0f;
}

// ---- sampling ----------------------------------------------------------------
// d: incident direction (toward the surface); frontface: the geometric front
// side was hit; etaExt: index of the medium outside this interface.
// Draws: lambert 2; metal 0 (mirror) / 2; smooth glass & water 1 when
// refraction is possible, 0 on TIR; rough glass 2 + 1 unless the facet
// reflects totally; plastic exactly 3. (device/bsdf.cuh:271-424)
SDB_HD BsdfDraw bsdfDraw(const SdMaterial& m, float3 albedo, float3 d, float3 n,
                         bool frontface, float etaExt, Pcg& rng) {
  BsdfDraw s;
  s.ok = false;
  s.pdf = 0.0f;
  s.delta = false;
  s.weight = v3(0.0f);
  s.wi = v3(0.0f);
  float3 wo = -d;

  switch (m.kind) {
    case MT_LAMBERT: {
      Frame fr(n);
      float3 li = cosineDir(rng.uni2());
      s.wi = fr.toWorld(li);
      s.pdf = fmaxf(li.z, 1e-8f) * kInvPi;
      s.weight = albedo;
      s.ok = li.z > 0.0f;
      return s;
    }
    case MT_METAL: {
      if (m.roughness < 1e-3f) {
        s.wi = unit(mirror(d, n));
        if (dot(s.wi, n) <= 0.0f) return s;
        s.weight = fresnelSchlick3(dot(s.wi, n), albedo);
        s.delta = true;
        s.ok = true;
        return s;
      }
      float a = m.roughness * m.roughness;
      Frame fr(n);
      float3 lo = fr.toLocal(wo);
      if (lo.z <= 0.0f) return s;
      float3 h = ggxSampleVisible(lo, a, rng.uni2());
      float3 li = mirror(-lo, h);
      if (li.z <= 0.0f) return s;
      float3 F = fresnelSchlick3(dot(lo, h), albedo);
      s.wi = fr.toWorld(li);
      s.weight = F * (ggxG(lo, li, a) / ggxG1(lo, a));
      s.pdf = ggxPdfReflect(lo, li, a);
      s.ok = s.pdf > 0.0f;
      return s;
    }
    case MT_WATER:
    case MT_DIELECTRIC: {
      float3 refr;
      float eta = frontface ? etaExt / m.ior : m.ior / etaExt;
      float f0 = (1.0f - eta) / (1.0f + eta);
      f0 = f0 * f0;
      if (m.kind == MT_WATER || m.roughness < 1e-3f) {
        s.delta = true;
        if (snell(d, n, eta, refr)) {
          float c = eta < 1.0f ? -dot(d, n) : -dot(refr, n);
          float pr = fresnelSchlick(c, f0);
          if (rng.uni() < pr)
            s.wi = unit(mirror(d, n));
          else
            s.wi = unit(refr);
        } else {
          s.wi = unit(mirror(d, n));
        }
        s.weight = v3(1.0f);
        s.ok = true;
        return s;
      }
      float a = m.roughness * m.roughness;
      Frame fr(n);
      float3 lo = fr.toLocal(wo);
      if (lo.z <= 0.0f) return s;
      float3 h = ggxSampleVisible(lo, a, rng.uni2());
      float loh = dot(lo, h);
      if (loh <= 0.0f) return s;
      float3 li;
      if (!snell(-lo, h, eta, refr)) {
        li = mirror(-lo, h);
        if (li.z <= 0.0f) return s;
        s.pdf = ggxPdfReflect(lo, li, a);
      } else {
        float c = eta < 1.0f ? loh : -dot(refr, h);
        float pr = fresnelSchlick(c, f0);
        if (rng.uni() < pr) {
          li = mirror(-lo, h);
          if (li.z <= 0.0f) return s;
          s.pdf = pr * ggxPdfReflect(lo, li, a);
        } else {
          li = unit(refr);
          if (li.z >= 0.0f) return s;
          s.pdf = (1.0f - pr) * ggxPdfTransmit(lo, li, h, eta, a);
        }
      }
      s.wi = fr.toWorld(li);
      float w = ggxG(lo, li, a) / ggxG1(lo, a);
      if (li.z < 0.0f) w *= eta * eta;
      s.weight = v3(w);
      s.ok = s.pdf > 0.0f;
      return s;
    }
    case MT_PLASTIC: {
      Frame fr(n);
      float3 lo = fr.toLocal(wo);
      if (lo.z <= 0.0f) return s;
      bool coat = rng.uni() < 0.5f;
      float3 li;
      if (coat) {
        float r = fmaxf(m.roughness, 1e-3f);
        float3 h = ggxSampleVisible(lo, r * r, rng.uni2());
        li = mirror(-lo, h);
      } else {
        li = cosineDir(rng.uni2());
      }
      if (li.z <= 0.0f) return s;
      PlasticLobes t = plasticLobes(m, albedo, lo, li);
      s.pdf = 0.5f * (t.pSpec + t.pDiff);
      if (s.pdf <= 0.0f) return s;
      s.wi = fr.toWorld(li);
      s.weight = (v3(t.fSpec) + t.fDiff) * (li.z / s.pdf);
      s.ok = true;
      return s;
    }
    default:
      return s;
  }
}

}  // namespace sdb
