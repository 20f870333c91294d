// Next-event estimation: explicit light sampling and the solid-angle pdfs used
// by MIS, plus the HDR environment light (equirect lookup, 2D piecewise
// constant CDF sampling, reverse pdf).
//
// Draw order and pdf conventions follow device/light_sample.cuh:24-226 and
// device/env_light.cuh:17-116 (cited per function).
#pragma once

#include "sd_rng.cuh"
#include "sd_texture.cuh"

namespace sdb {

struct LightDraw {
  float3 wi;    // unit, shading point -> light
  float dist;   // shadow-ray length
  float3 Li;    // radiance (delta lights: already divided by their pdf)
  float pdf;    // solid angle; 1 for delta lights
  bool delta;
  bool ok;
};

// Largest i in [0, n-2] with cdf[i] <= u. (device/env_light.cuh:36-43;
// the mesh-light search in device/light_sample.cuh:99-103 is the same.)
SDB_HD int cdfSearchIn(const float* cdf, int lo, int hi, float u) {
  while (lo + 1 < hi) {
    int mid = (lo + hi) >> 1;
    if (cdf[mid] <= u)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

SDB_HD int cdfSearch(const float* cdf, int n, float u) { return cdfSearchIn(cdf, 0, n - 1, u); }

// The same index through the CDF's guide (kCdfGuide + 1 entries; null: the
// plain search). For a non-decreasing CDF the search returns the last index
// i <= n - 2 with cdf[i] <= u, a non-decreasing function of u, so for u in
// [k / K, (k + 1) / K) (exact bounds: K is a power of two) it lies between
// guide[k] and guide[k + 1], and cdf[guide[k]] <= u < cdf[guide[k + 1] + 1]
// (or guide[k + 1] = n - 2) keep the loop's invariants.
SDB_HD int cdfSearchGuided(const float* cdf, int n, const int* guide, float u) {
  if (!guide) return cdfSearch(cdf, n, u);
  const int k = min(max((int)(u * (float)kCdfGuide), 0), kCdfGuide - 1);
  return cdfSearchIn(cdf, guide[k], min(guide[k + 1] + 1, n - 1), u);
}

// ---- environment ------------------------------------------------------------

// Direction -> equirect uv with the inverse azimuth rotation; v = 0 at +Y.
// (device/env_light.cuh:17-22)
SDB_HD float2 envUv(const SdEnv& e, float3 dir) {
  float u = (atan2f(dir.z, dir.x) - e.rotate + kPi) * (0.5f * kInvPi);
  u -= floorf(u);
  float v = acosf(clampf(dir.y, -1.0f, 1.0f)) * kInvPi;
  return make_float2(u, v);
}

// (device/env_light.cuh:24-33)
SDB_HD float3 envRadiance(const SdEnv& e, float3 dir) {
  float2 uv = envUv(e, dir);
  float4 c = sampleFloat4(e.texels, e.width, e.height, uv.x, uv.y);
  return v3(c.x, c.y, c.z) * e.intensity;
}

// Marginal row then conditional column; pdf = dm dc W H / (2 pi^2 sin theta).
// Two draws in both modes. (device/env_light.cuh:54-95)
SDB_HD LightDraw envDraw(const SdEnv& e, Pcg& rng) {
  LightDraw s;
  s.ok = false;
  s.delta = false;
  s.pdf = 0.0f;
  s.dist = 1e16f;
  s.Li = v3(0.0f);
  s.wi = v3(0.0f, 1.0f, 0.0f);
  float2 rn = rng.uni2();
  if (!e.importance) {
    s.wi = sphereDir(rn);
    s.pdf = 0.25f * kInvPi;
    s.Li = envRadiance(e, s.wi);
    s.ok = true;
    return s;
  }
  int row = cdfSearchGuided(e.margCdf, e.height + 1, e.margGuide, rn.x);
  float dm = e.margCdf[row + 1] - e.margCdf[row];
  float dv = dm > 0.0f ? (rn.x - e.margCdf[row]) / dm : 0.5f;
  float v = (row + dv) / e.height;
  const float* cdf = e.condCdf + (size_t)row * (e.width + 1);
  int col = cdfSearchGuided(cdf, e.width + 1,
                            e.condGuide ? e.condGuide + (size_t)row * (kCdfGuide + 1) : nullptr,
                            rn.y);
  float dc = cdf[col + 1] - cdf[col];
  float du = dc > 0.0f ? (rn.y - cdf[col]) / dc : 0.5f;
  float u = (col + du) / e.width;
  float theta = v * kPi;
  float sinT = sinf(theta);
  if (sinT < 1e-6f || dm <= 0.0f || dc <= 0.0f) return s;
  float phi = (2.0f * kPi * u - kPi) + e.rotate;
  s.wi = v3(sinT * cosf(phi), cosf(theta), sinT * sinf(phi));
  s.pdf = dm * dc * e.width * e.height / (2.0f * kPi * kPi * sinT);
  s.Li = envRadiance(e, s.wi);
  s.ok = s.pdf > 0.0f;
  return s;
}

// Reverse query for MIS on escaped BSDF rays. (device/env_light.cuh:104-116)
SDB_HD float envDensity(const SdEnv& e, float3 dir) {
  if (!e.importance) return 0.25f * kInvPi;
  float sinT = sqrtf(fmaxf(0.0f, 1.0f - dir.y * dir.y));
  if (sinT < 1e-6f) return 0.0f;
  float2 uv = envUv(e, dir);
  int col = min((int)(uv.x * e.width), e.width - 1);
  int row = min((int)(uv.y * e.height), e.height - 1);
  float dm = e.margCdf[row + 1] - e.margCdf[row];
  const float* cdf = e.condCdf + (size_t)row * (e.width + 1);
  float dc = cdf[col + 1] - cdf[col];
  return dm * dc * e.width * e.height / (2.0f * kPi * kPi * sinT);
}

// ---- explicit lights ---------------------------------------------------------

// x: shading point. Draws: rect 2, disk 2, sphere 2, mesh 3, point 2,
// distant 0. (device/light_sample.cuh:24-188)
SDB_HD LightDraw lightDraw(const SdLight& lt, float3 x, Pcg& rng, const SdTexture* tex) {
  LightDraw s;
  s.ok = false;
  s.delta = false;
  s.pdf = 0.0f;
  s.dist = 0.0f;
  s.Li = v3(0.0f);
  s.wi = v3(0.0f, 1.0f, 0.0f);
  switch (lt.kind) {
    case LT_RECT:
    case LT_DISK: {
      float3 p;
      float tu, tv;
      if (lt.kind == LT_RECT) {
        float a = 2.0f * rng.uni() - 1.0f;
        float b = 2.0f * rng.uni() - 1.0f;
        p = lt.p + a * lt.u + b * lt.v;
        tu = (a + 1.0f) * 0.5f;
        tv = (b + 1.0f) * 0.5f;
      } else {
        float2 d = diskConcentric(rng.uni2());
        p = lt.p + d.x * lt.u + d.y * lt.v;
        tu = (atan2f(d.y, d.x) + kPi) / (2.0f * kPi);
        tv = sqrtf(d.x * d.x + d.y * d.y);
      }
      float3 to = p - x;
      float d2 = len2(to);
      if (d2 < 1e-10f) return s;
      float dist = sqrtf(d2);
      float3 wi = to / dist;
      float cosL = -dot(wi, lt.n);
      if (!lt.twoSided && cosL <= 0.0f) return s;
      cosL = fabsf(cosL);
      if (cosL < 1e-6f) return s;
      s.wi = wi;
      s.dist = dist;
      s.Li = lt.L;
      if (lt.texId >= 0 && tex) {
        float4 c = texLookup(tex[lt.texId], tu, tv);
        s.Li = lt.L * v3(c.x, c.y, c.z);
      }
      s.pdf = d2 / (cosL * lt.area);
      s.ok = true;
      return s;
    }
    case LT_SPHERE: {
      float3 to = lt.p - x;
      float d2 = len2(to);
      float r2 = lt.radius * lt.radius;
      if (d2 <= r2 * 1.0001f) return s;
      float dist = sqrtf(d2);
      float3 wc = to / dist;
      float sin2 = r2 / d2;
      float cosMax = sqrtf(fmaxf(0.0f, 1.0f - sin2));
      float2 u = rng.uni2();
      float cosT = 1.0f - u.x * (1.0f - cosMax);
      float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosT * cosT));
      float phi = 2.0f * kPi * u.y;
      Frame fr(wc);
      s.wi = fr.toWorld(v3(sinT * cosf(phi), sinT * sinf(phi), cosT));
      float b = dot(s.wi, to);
      float det = fmaxf(0.0f, b * b - d2 + r2);
      s.dist = b - sqrtf(det);
      s.Li = lt.L;
      s.pdf = 1.0f / (2.0f * kPi * (1.0f - cosMax));
      s.ok = true;
      return s;
    }
    case LT_MESH: {
      float uc = rng.uni();
      int k = cdfSearch(lt.mCdf, lt.mNumTris + 1, uc);
      uint3 tri = lt.mIdx[k];
      float3 p0 = lt.mPos[tri.x], p1 = lt.mPos[tri.y], p2 = lt.mPos[tri.z];
      float2 r = rng.uni2();
      float su = sqrtf(r.x);
      float bx = su * (1.0f - r.y);
      float by = su * r.y;
      float3 p = p0 * (1.0f - bx - by) + p1 * bx + p2 * by;
      float3 ngU = cross(p1 - p0, p2 - p0);
      float ngL2 = len2(ngU);
      if (ngL2 < 1e-20f) return s;
      float3 ng = ngU * (lt.mNgSign / sqrtf(ngL2));
      float3 to = p - x;
      float d2 = len2(to);
      if (d2 < 1e-10f) return s;
      float dist = sqrtf(d2);
      float3 wi = to / dist;
      float cosL = -dot(wi, ng);
      if (!lt.twoSided && cosL <= 0.0f) return s;
      cosL = fabsf(cosL);
      if (cosL < 1e-6f) return s;
      s.wi = wi;
      s.dist = dist;
      s.Li = lt.L;
      if (lt.texId >= 0 && tex) {
        float tu, tv;
        if (lt.mUv) {
          float2 a = lt.mUv[tri.x], b = lt.mUv[tri.y], c = lt.mUv[tri.z];
          float w0 = 1.0f - bx - by;
          tu = a.x * w0 + b.x * bx + c.x * by;
          tv = a.y * w0 + b.y * bx + c.y * by;
        } else {
          tu = bx;
          tv = by;
        }
        float4 c = texLookup(tex[lt.texId], tu, tv);
        s.Li = lt.L * v3(c.x, c.y, c.z);
      }
      s.pdf = d2 / (cosL * lt.area);
      s.ok = true;
      return s;
    }
    case LT_POINT: {
      s.delta = true;
      float3 to = lt.p - x;
      float d2c = len2(to);
      if (d2c < 1e-10f) return s;
      float3 wc = to / sqrtf(d2c);
      float2 dd = diskConcentric(rng.uni2());
      dd.x *= lt.radius;
      dd.y *= lt.radius;
      Frame fr(wc);
      float3 p = lt.p + dd.x * fr.t + dd.y * fr.b;
      float3 top = p - x;
      float d2 = len2(top);
      float dist = sqrtf(d2);
      s.wi = top / dist;
      s.dist = fmaxf(dist - 1e-4f, 1e-4f);
      s.Li = lt.L / d2;
      s.pdf = 1.0f;
      s.ok = true;
      return s;
    }
    case LT_DISTANT: {
      s.delta = true;
      s.wi = -lt.dir;
      s.dist = 1e16f;
      s.Li = lt.L;
      s.pdf = 1.0f;
      s.ok = true;
      return s;
    }
  }
  return s;
}

// Solid-angle pdf of lightDraw producing the direction from `from` to hitP on
// area light lt; nHit is the hit's packed normal (only meshes read it: the
// hit triangle's geometric normal). Delta lights: 0.
// (device/light_sample.cuh:197-226)
SDB_HD float lightDensity(const SdLight& lt, float3 from, float3 hitP, float3 nHit) {
  switch (lt.kind) {
    case LT_RECT:
    case LT_DISK:
    case LT_MESH: {
      float3 to = hitP - from;
      float d2 = len2(to);
      if (d2 < 1e-10f) return 0.0f;
      float dist = sqrtf(d2);
      float cosL = fabsf(dot(to / dist, lt.kind == LT_MESH ? nHit : lt.n));
      if (cosL < 1e-6f) return 0.0f;
      return d2 / (cosL * lt.area);
    }
    case LT_SPHERE: {
      float3 to = lt.p - from;
      float d2 = len2(to);
      float r2 = lt.radius * lt.radius;
      if (d2 <= r2 * 1.0001f) return 0.0f;
      float cosMax = sqrtf(fmaxf(0.0f, 1.0f - r2 / d2));
      return 1.0f / (2.0f * kPi * (1.0f - cosMax));
    }
    default:
      return 0.0f;
  }
}

}  // namespace sdb
