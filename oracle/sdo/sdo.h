// ORACLE — test infrastructure only. This header is the CPU checker's
// restatement of sundog's device math (device/*.cuh), scalar C++, used by
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg to judge
// the CUDA path; nothing in the product links or calls it.
//
// Types and function names follow the reference headers (namespace sd ->
// sdo) so that one harness (oracle/fnvec.cpp) compiles against either this
// restatement or the reference's own headers; that is how the golden vectors
// in tests/golden/ pin this file. Every function cites the reference
// file:line it restates. Arithmetic order is kept operation for operation:
// built with g++ -O2 -ffp-contract=off, outputs are bit-identical to the
// reference headers compiled the same way.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstddef>
#include <algorithm>

namespace sdo {

struct float2 { float x, y; };
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
struct uint3 { unsigned x, y, z; };
inline float2 make_float2(float a, float b) { return {a, b}; }
inline float3 make_float3(float a, float b, float c) { return {a, b, c}; }
inline float4 make_float4(float a, float b, float c, float d) { return {a, b, c, d}; }

// ---- device/math.cuh:17-69 ----------------------------------------------------
inline float3 f3(float v) { return {v, v, v}; }
inline float3 f3(float x, float y, float z) { return {x, y, z}; }
inline float3 operator+(float3 a, float3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline float3 operator-(float3 a, float3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline float3 operator-(float3 a) { return {-a.x, -a.y, -a.z}; }
inline float3 operator*(float3 a, float3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline float3 operator*(float3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float3 operator*(float s, float3 a) { return {a.x * s, a.y * s, a.z * s}; }
inline float3 operator/(float3 a, float s) { return a * (1.0f / s); }
inline float3& operator+=(float3& a, float3 b) { a = a + b; return a; }
inline float3& operator*=(float3& a, float3 b) { a = a * b; return a; }
inline float3& operator*=(float3& a, float s) { a = a * s; return a; }
inline float2 operator+(float2 a, float2 b) { return {a.x + b.x, a.y + b.y}; }
inline float2 operator*(float2 a, float s) { return {a.x * s, a.y * s}; }
inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float3 cross(float3 a, float3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float length2(float3 a) { return dot(a, a); }
inline float length(float3 a) { return std::sqrt(dot(a, a)); }
inline float3 normalize(float3 a) { return a * (1.0f / std::sqrt(dot(a, a))); }
inline float clampf(float x, float lo, float hi) { return std::fmin(hi, std::fmax(lo, x)); }
inline float3 min3(float3 a, float3 b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
inline float maxComp(float3 v) { return std::fmax(v.x, std::fmax(v.y, v.z)); }
inline float3 lerp3(float3 a, float3 b, float t) { return a + (b - a) * t; }
inline float3 exp3(float3 a) { return {std::exp(a.x), std::exp(a.y), std::exp(a.z)}; }
inline float3 reflect(float3 v, float3 n) { return v - 2.0f * dot(v, n) * n; }
inline bool refract(float3 v, float3 n, float eta, float3& out) {
  float ci = -dot(v, n);
  float k = 1.0f - eta * eta * (1.0f - ci * ci);
  if (k < 0.0f) return false;
  out = eta * v + (eta * ci - std::sqrt(k)) * n;
  return true;
}
inline float schlick(float c, float f0) {
  float m = clampf(1.0f - c, 0.0f, 1.0f);
  float m2 = m * m;
  return f0 + (1.0f - f0) * m2 * m2 * m;
}
inline float3 schlick3(float c, float3 f0) {
  float m = clampf(1.0f - c, 0.0f, 1.0f);
  float m2 = m * m;
  return f0 + (f3(1.0f) - f0) * (m2 * m2 * m);
}

// device/math.cuh:72-83 (Duff et al. 2017 frame)
struct Onb {
  float3 t, b, n;
  explicit Onb(float3 nn) : n(nn) {
    float s = std::copysign(1.0f, nn.z);
    float a = -1.0f / (s + nn.z);
    float c = nn.x * nn.y * a;
    t = f3(1.0f + s * nn.x * nn.x * a, s * c, -s * nn.x);
    b = f3(c, s + nn.y * nn.y * a, -nn.y);
  }
  float3 toWorld(float3 v) const { return v.x * t + v.y * b + v.z * n; }
  float3 toLocal(float3 v) const { return f3(dot(v, t), dot(v, b), dot(v, n)); }
};

constexpr float SD_PI = 3.14159265358979323846f;
constexpr float SD_INV_PI = 0.31830988618379067154f;

// device/math.cuh:151-154
inline float3 offsetRay(float3 p, float3 n) {
  float s = 1e-4f * (1.0f + std::fmax(std::fabs(p.x), std::fmax(std::fabs(p.y), std::fabs(p.z))));
  return p + n * s;
}

// ---- device/params.h:12-105 (descriptors; pointers are host arrays) -----------
enum GeomKind : int { GK_SPHERE = 0, GK_RECT, GK_DISK, GK_CYLINDER, GK_PARABOLA, GK_MESH };
enum TexKind : int { TX_SOLID = 0, TX_IMAGE, TX_CHECKER, TX_GRID };
enum MatKind : int { MT_LAMBERT = 0, MT_METAL, MT_DIELECTRIC, MT_EMISSIVE, MT_WATER, MT_PLASTIC };
enum LightKind : int { LT_RECT = 0, LT_DISK, LT_SPHERE, LT_POINT, LT_DISTANT, LT_MESH };
constexpr uint16_t MAT_NONE = 0xFFFF;

struct TextureDesc {
  int kind;
  float3 a, b;
  float2 scale;
  float width;
  const unsigned char* img;  // TX_IMAGE: RGBA8, row 0 = top
  int imgW, imgH, srgb;
};
struct MaterialDesc {
  int kind, texId;
  float3 color;
  float roughness, ior, intensity;
  int twoSided;
  float3 absorb;
  float waveAmp, waveFreq;
};
struct LightDesc {
  int kind;
  float3 p, u, v, n, L;
  float radius, area;
  float3 dir;
  int twoSided, texId, flameId;
  const float3* mPositions;
  const uint3* mIndices;
  const float2* mUvs;
  const float* mCdf;
  int mNumTris;
  float mNgSign;
};
struct EnvDesc {
  const float* texels;  // RGBA float, row 0 = zenith
  const float* margCdf;
  const float* condCdf;
  int width, height;
  float rotate, intensity;
  int importance;
};
struct FlameDesc {
  float3 base;
  float height, radius, intensity, sigma, noiseScale;
  unsigned seed;
  int steps;
};

// ---- device/rng.cuh:10-60 -------------------------------------------------------
struct Pcg32 {
  uint64_t state, inc;
  uint32_t next() {
    uint64_t old = state;
    state = old * 6364136223846793005ULL + inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
  }
  static Pcg32 init(uint64_t seed, uint64_t seq) {
    Pcg32 r;
    r.state = 0u;
    r.inc = (seq << 1u) | 1u;
    r.next();
    r.state += seed;
    r.next();
    return r;
  }
  float rnd() { return (float)(next() >> 8) * 0x1p-24f; }
  float2 rnd2() { float a = rnd(); float b = rnd(); return {a, b}; }
};
inline float3 uniformOnSphere(float2 u) {
  float z = 1.0f - 2.0f * u.x;
  float r = std::sqrt(std::fmax(0.0f, 1.0f - z * z));
  float phi = 2.0f * SD_PI * u.y;
  return f3(r * std::cos(phi), r * std::sin(phi), z);
}
inline float2 concentricDisk(float2 u) {
  float ox = 2.0f * u.x - 1.0f, oy = 2.0f * u.y - 1.0f;
  if (ox == 0.0f && oy == 0.0f) return {0.0f, 0.0f};
  float r, th;
  if (std::fabs(ox) > std::fabs(oy)) { r = ox; th = (SD_PI / 4.0f) * (oy / ox); }
  else { r = oy; th = (SD_PI / 2.0f) - (SD_PI / 4.0f) * (ox / oy); }
  return {r * std::cos(th), r * std::sin(th)};
}
inline float3 cosineHemisphere(float2 u) {
  float2 d = concentricDisk(u);
  float z = std::sqrt(std::fmax(0.0f, 1.0f - d.x * d.x - d.y * d.y));
  return f3(d.x, d.y, z);
}

// ---- device/intersect.cuh:18-162 ---------------------------------------------------
struct QuadricHit { float t; float3 n; float u, v; };
struct QuadricHits { QuadricHit hits[2]; int count; };

inline void sphereUv(float3 n, float& u, float& v) {
  u = (std::atan2(n.z, n.x) + SD_PI) / (2.0f * SD_PI);
  v = (std::asin(clampf(n.y, -1.0f, 1.0f)) + SD_PI / 2.0f) / SD_PI;
}
inline void pushRoot(QuadricHits& r, float t, float3 n, float u, float v) {
  QuadricHit& h = r.hits[r.count++];
  h.t = t; h.n = n; h.u = u; h.v = v;
}
inline QuadricHits intersectQuadric(int kind, float3 o, float3 d, float tmin, float tmax) {
  QuadricHits r; r.count = 0;
  if (kind == GK_SPHERE) {                       // intersect.cuh:37-57
    float a = dot(d, d), b = dot(o, d), c = dot(o, o) - 1.0f;
    float disc = b * b - a * c;
    if (disc <= 0.0f) return r;
    float s = std::sqrt(disc);
    float roots[2] = {(-b - s) / a, (-b + s) / a};
    for (float t : roots) {
      if (t > tmin && t < tmax) {
        float3 n = normalize(o + t * d);
        float u, v; sphereUv(n, u, v);
        pushRoot(r, t, n, u, v);
      }
    }
  } else if (kind == GK_RECT || kind == GK_DISK) {   // intersect.cuh:59-88
    if (d.y == 0.0f) return r;
    float t = -o.y / d.y;
    if (t <= tmin || t >= tmax) return r;
    float x = o.x + t * d.x, z = o.z + t * d.z;
    if (kind == GK_RECT) {
      if (std::fabs(x) > 1.0f || std::fabs(z) > 1.0f) return r;
      pushRoot(r, t, f3(0.0f, 1.0f, 0.0f), (x + 1.0f) * 0.5f, (z + 1.0f) * 0.5f);
    } else {
      float rad = std::sqrt(x * x + z * z);
      if (rad > 1.0f) return r;
      pushRoot(r, t, f3(0.0f, 1.0f, 0.0f), (std::atan2(z, x) + SD_PI) / (2.0f * SD_PI), rad);
    }
  } else if (kind == GK_CYLINDER) {              // intersect.cuh:90-114
    float a = d.x * d.x + d.z * d.z;
    if (a == 0.0f) return r;
    float b = o.x * d.x + o.z * d.z, c = o.x * o.x + o.z * o.z - 1.0f;
    float disc = b * b - a * c;
    if (disc <= 0.0f) return r;
    float s = std::sqrt(disc);
    float roots[2] = {(-b - s) / a, (-b + s) / a};
    for (float t : roots) {
      if (t > tmin && t < tmax) {
        float3 p = o + t * d;
        if (std::fabs(p.y) <= 1.0f)
          pushRoot(r, t, normalize(f3(p.x, 0.0f, p.z)),
                   (std::atan2(p.z, p.x) + SD_PI) / (2.0f * SD_PI), (p.y + 1.0f) * 0.5f);
      }
    }
  } else if (kind == GK_PARABOLA) {              // intersect.cuh:116-151
    float A = 0.5f * (d.x * d.x + d.z * d.z);
    float B = o.x * d.x + o.z * d.z - d.y;
    float C = 0.5f * (o.x * o.x + o.z * o.z) - o.y;
    float ts[2] = {0.0f, 0.0f};
    int n;
    if (std::fabs(A) < 1e-12f) {
      if (B == 0.0f) return r;
      ts[0] = -C / B; n = 1;
    } else {
      float disc = B * B - 4.0f * A * C;
      if (disc <= 0.0f) return r;
      float s = std::sqrt(disc);
      ts[0] = (-B - s) / (2.0f * A);
      ts[1] = (-B + s) / (2.0f * A);
      n = 2;
    }
    for (int i = 0; i < n; i++) {
      float t = ts[i];
      if (t > tmin && t < tmax) {
        float3 p = o + t * d;
        if (p.x * p.x + p.z * p.z <= 1.0f)
          pushRoot(r, t, normalize(f3(p.x, -1.0f, p.z)),
                   (std::atan2(p.z, p.x) + SD_PI) / (2.0f * SD_PI), std::sqrt(p.x * p.x + p.z * p.z));
      }
    }
  }
  return r;
}

// ---- textures: device/texture_eval.cuh:11-46 plus the texture unit's bilinear
// filter (1.8 fixed-point weights, taps at floor(x - 0.5)) ---------------------------
inline float texWeight(float f) { return std::rint(f * 256.0f) * (1.0f / 256.0f); }
inline void texAxis(float c, int n, bool wrap, int& i0, int& i1, float& w) {
  if (wrap) c = c - std::floor(c);
  float x = c * (float)n - 0.5f;
  float fl = std::floor(x);
  int i = (int)fl;
  w = texWeight(x - fl);
  if (wrap) {
    i0 = ((i % n) + n) % n;
    i1 = (((i + 1) % n) + n) % n;
  } else {
    i0 = std::min(std::max(i, 0), n - 1);
    i1 = std::min(std::max(i + 1, 0), n - 1);
  }
}
inline float4 lerp4(float4 a, float4 b, float w) {
  float v = 1.0f - w;
  return {v * a.x + w * b.x, v * a.y + w * b.y, v * a.z + w * b.z, v * a.w + w * b.w};
}
inline float4 texFetchF4(const float* t, int W, int H, float u, float v) {
  int x0, x1, y0, y1; float wx, wy;
  texAxis(u, W, true, x0, x1, wx);
  texAxis(v, H, false, y0, y1, wy);
  auto at = [&](int x, int y) { const float* p = t + 4 * ((size_t)y * W + x); return make_float4(p[0], p[1], p[2], p[3]); };
  return lerp4(lerp4(at(x0, y0), at(x1, y0), wx), lerp4(at(x0, y1), at(x1, y1), wx), wy);
}
inline float srgbDecode(float c) {
  return c <= 0.04045f ? c * (1.0f / 12.92f) : std::pow((c + 0.055f) * (1.0f / 1.055f), 2.4f);
}
inline float4 evalTexture(const TextureDesc& tx, float u, float v) {
  switch (tx.kind) {
    case TX_SOLID: return make_float4(tx.a.x, tx.a.y, tx.a.z, 1.0f);
    case TX_CHECKER: {
      int iu = (int)std::floor(u * tx.scale.x), iv = (int)std::floor(v * tx.scale.y);
      float3 c = (((iu + iv) & 1) == 0) ? tx.a : tx.b;
      return make_float4(c.x, c.y, c.z, 1.0f);
    }
    case TX_GRID: {
      float fu = u * tx.scale.x - std::floor(u * tx.scale.x);
      float fv = v * tx.scale.y - std::floor(v * tx.scale.y);
      float w = tx.width;
      bool line = fu < w || fv < w || fu > 1.0f - w || fv > 1.0f - w;
      float3 c = line ? tx.b : tx.a;
      return make_float4(c.x, c.y, c.z, 1.0f);
    }
    case TX_IMAGE: {
      int x0, x1, y0, y1; float wx, wy;
      texAxis(u, tx.imgW, true, x0, x1, wx);
      texAxis(1.0f - v, tx.imgH, true, y0, y1, wy);
      auto at = [&](int x, int y) {
        const unsigned char* p = tx.img + 4 * ((size_t)y * tx.imgW + x);
        float r = p[0] * (1.0f / 255.0f), g = p[1] * (1.0f / 255.0f), b = p[2] * (1.0f / 255.0f);
        if (tx.srgb) { r = srgbDecode(r); g = srgbDecode(g); b = srgbDecode(b); }
        return make_float4(r, g, b, p[3] * (1.0f / 255.0f));
      };
      return lerp4(lerp4(at(x0, y0), at(x1, y0), wx), lerp4(at(x0, y1), at(x1, y1), wx), wy);
    }
  }
  return make_float4(1.0f, 0.0f, 1.0f, 1.0f);
}
inline float3 materialAlbedo(const MaterialDesc& m, const TextureDesc* tex, float u, float v) {
  if (m.texId < 0) return m.color;
  float4 c = evalTexture(tex[m.texId], u, v);
  return f3(c.x, c.y, c.z);
}

// ---- device/bsdf.cuh ------------------------------------------------------------------
struct BsdfSample { float3 wi; float3 weight; float pdf; bool isDelta; bool valid; };

inline bool bsdfIsDelta(const MaterialDesc& m) {                   // bsdf.cuh:27-33
  if (m.kind == MT_WATER) return true;
  if (m.kind == MT_DIELECTRIC || m.kind == MT_METAL) return m.roughness < 1e-3f;
  return false;
}
inline float ggxD(float3 h, float a) {                               // bsdf.cuh:37-45
  float c2 = h.z * h.z;
  float k = a * a * c2 + (1.0f - c2);
  return a * a / (SD_PI * k * k);
}
inline float ggxLambda(float3 w, float a) {                          // bsdf.cuh:47-52
  float c2 = w.z * w.z;
  if (c2 >= 1.0f) return 0.0f;
  float t2 = (1.0f - c2) / c2;
  return 0.5f * (-1.0f + std::sqrt(1.0f + a * a * t2));
}
inline float ggxG1(float3 w, float a) { return 1.0f / (1.0f + ggxLambda(w, a)); }
inline float ggxG(float3 wo, float3 wi, float a) {
  return 1.0f / (1.0f + ggxLambda(wo, a) + ggxLambda(wi, a));
}
inline float3 ggxSampleVndf(float3 wo, float a, float2 u) {          // bsdf.cuh:60-73
  float3 vh = normalize(f3(a * wo.x, a * wo.y, wo.z));
  float l2 = vh.x * vh.x + vh.y * vh.y;
  float3 T1 = l2 > 0.0f ? f3(-vh.y, vh.x, 0.0f) * (1.0f / std::sqrt(l2)) : f3(1.0f, 0.0f, 0.0f);
  float3 T2 = cross(vh, T1);
  float r = std::sqrt(u.x), phi = 2.0f * SD_PI * u.y;
  float t1 = r * std::cos(phi), t2 = r * std::sin(phi);
  float s = 0.5f * (1.0f + vh.z);
  t2 = (1.0f - s) * std::sqrt(std::fmax(0.0f, 1.0f - t1 * t1)) + s * t2;
  float3 nh = t1 * T1 + t2 * T2 + std::sqrt(std::fmax(0.0f, 1.0f - t1 * t1 - t2 * t2)) * vh;
  return normalize(f3(a * nh.x, a * nh.y, std::fmax(1e-6f, nh.z)));
}
inline float ggxPdf(float3 wo, float3 wi, float a) {                 // bsdf.cuh:76-80
  if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
  float3 h = normalize(wo + wi);
  return ggxG1(wo, a) * ggxD(h, a) / (4.0f * wo.z);
}
inline float fresnelDielectric(float cosI, float eta, float f0) {    // bsdf.cuh:88-92
  float k = 1.0f - eta * eta * (1.0f - cosI * cosI);
  if (k <= 0.0f) return 1.0f;
  return schlick(eta < 1.0f ? cosI : std::sqrt(k), f0);
}
inline float ggxPdfTransmit(float3 lo, float3 li, float3 h, float eta, float a) {  // bsdf.cuh:98-105
  float loh = dot(lo, h), lih = dot(li, h);
  if (lo.z <= 0.0f || li.z >= 0.0f || loh <= 0.0f || lih >= 0.0f) return 0.0f;
  float den = eta * loh + lih;
  if (std::fabs(den) < 1e-6f) return 0.0f;
  return ggxG1(lo, a) * ggxD(h, a) * loh / lo.z * std::fabs(lih) / (den * den);
}
struct PlasticTerms { float fSpec; float3 fDiff; float pSpec, pDiff; };
inline PlasticTerms plasticTerms(const MaterialDesc& m, float3 albedo, float3 lo, float3 li) {  // bsdf.cuh:128-143
  PlasticTerms t;
  float rough = std::fmax(m.roughness, 1e-3f), a = rough * rough;
  float f0 = (m.ior - 1.0f) / (m.ior + 1.0f);
  f0 = f0 * f0;
  float3 h = normalize(lo + li);
  float F = schlick(dot(lo, h), f0);
  t.fSpec = F * ggxD(h, a) * ggxG(lo, li, a) / (4.0f * lo.z * li.z);
  t.fDiff = albedo * (SD_INV_PI * (1.0f - schlick(lo.z, f0)) * (1.0f - schlick(li.z, f0)));
  t.pSpec = ggxPdf(lo, li, a);
  t.pDiff = li.z * SD_INV_PI;
  return t;
}
inline float dielectricF0(float eta) {
  float f0 = (1.0f - eta) / (1.0f + eta);
  return f0 * f0;
}
inline float3 bsdfEval(const MaterialDesc& m, float3 albedo, float3 wo, float3 wi, float3 n,
                       float eta) {                                   // bsdf.cuh:151-213
  float ci = dot(wi, n), co = dot(wo, n);
  if (co <= 0.0f) return f3(0.0f);
  bool rough = m.kind == MT_DIELECTRIC && m.roughness >= 1e-3f;
  if (ci <= 0.0f) {
    if (!rough || ci == 0.0f) return f3(0.0f);
    float a = m.roughness * m.roughness;
    Onb onb(n);
    float3 lo = onb.toLocal(wo), li = onb.toLocal(wi);
    float3 h = normalize(eta * lo + li);
    if (h.z < 0.0f) h = -h;
    float loh = dot(lo, h), lih = dot(li, h);
    if (loh <= 0.0f || lih >= 0.0f) return f3(0.0f);
    float den = eta * loh + lih;
    if (std::fabs(den) < 1e-6f) return f3(0.0f);
    float F = fresnelDielectric(loh, eta, dielectricF0(eta));
    float ft = eta * eta * (1.0f - F) * ggxD(h, a) * ggxG(lo, li, a) * std::fabs(loh * lih) /
               (lo.z * std::fabs(li.z) * den * den);
    return f3(ft);
  }
  if (m.kind == MT_LAMBERT) return albedo * SD_INV_PI;
  if (m.kind == MT_PLASTIC) {
    Onb onb(n);
    PlasticTerms t = plasticTerms(m, albedo, onb.toLocal(wo), onb.toLocal(wi));
    return f3(t.fSpec) + t.fDiff;
  }
  if (m.kind == MT_METAL && m.roughness >= 1e-3f) {
    float a = m.roughness * m.roughness;
    Onb onb(n);
    float3 lo = onb.toLocal(wo), li = onb.toLocal(wi);
    float3 h = normalize(lo + li);
    return schlick3(dot(lo, h), albedo) * (ggxD(h, a) * ggxG(lo, li, a) / (4.0f * lo.z * li.z));
  }
  if (rough) {
    float a = m.roughness * m.roughness;
    Onb onb(n);
    float3 lo = onb.toLocal(wo), li = onb.toLocal(wi);
    float3 h = normalize(lo + li);
    float F = fresnelDielectric(dot(lo, h), eta, dielectricF0(eta));
    return f3(F * ggxD(h, a) * ggxG(lo, li, a) / (4.0f * lo.z * li.z));
  }
  return f3(0.0f);
}
inline float bsdfPdf(const MaterialDesc& m, float3 wo, float3 wi, float3 n, float eta) {  // bsdf.cuh:215-263
  float ci = dot(wi, n), co = dot(wo, n);
  if (co <= 0.0f) return 0.0f;
  bool rough = m.kind == MT_DIELECTRIC && m.roughness >= 1e-3f;
  if (ci <= 0.0f) {
    if (!rough || ci == 0.0f) return 0.0f;
    float a = m.roughness * m.roughness;
    Onb onb(n);
    float3 lo = onb.toLocal(wo), li = onb.toLocal(wi);
    float3 h = normalize(eta * lo + li);
    if (h.z < 0.0f) h = -h;
    float loh = dot(lo, h);
    if (loh <= 0.0f) return 0.0f;
    float F = fresnelDielectric(loh, eta, dielectricF0(eta));
    return (1.0f - F) * ggxPdfTransmit(lo, li, h, eta, a);
  }
  if (m.kind == MT_LAMBERT) return ci * SD_INV_PI;
  if (m.kind == MT_PLASTIC) {
    Onb onb(n);
    PlasticTerms t = plasticTerms(m, f3(0.0f), onb.toLocal(wo), onb.toLocal(wi));
    return 0.5f * (t.pSpec + t.pDiff);
  }
  if (m.kind == MT_METAL && m.roughness >= 1e-3f) {
    Onb onb(n);
    return ggxPdf(onb.toLocal(wo), onb.toLocal(wi), m.roughness * m.roughness);
  }
  if (rough) {
    float a = m.roughness * m.roughness;
    Onb onb(n);
    float3 lo = onb.toLocal(wo), li = onb.toLocal(wi);
    float3 h = normalize(lo + li);
    float F = fresnelDielectric(dot(lo, h), eta, dielectricF0(eta));
    return F * ggxPdf(lo, li, a);
  }
  return 0.0f;
}
inline BsdfSample bsdfSample(const MaterialDesc& m, float3 albedo, float3 rayDir, float3 n,
                             bool frontface, float etaExt, Pcg32& rng) {  // bsdf.cuh:271-424
  BsdfSample s;
  s.valid = false; s.pdf = 0.0f; s.isDelta = false;
  s.wi = f3(0.0f); s.weight = f3(0.0f);
  float3 wo = -rayDir;
  if (m.kind == MT_LAMBERT) {
    Onb onb(n);
    float3 li = cosineHemisphere(rng.rnd2());
    s.wi = onb.toWorld(li);
    s.pdf = std::fmax(li.z, 1e-8f) * SD_INV_PI;
    s.weight = albedo;
    s.valid = li.z > 0.0f;
    return s;
  }
  if (m.kind == MT_METAL) {
    if (m.roughness < 1e-3f) {
      s.wi = normalize(reflect(rayDir, n));
      if (dot(s.wi, n) <= 0.0f) return s;
      s.weight = schlick3(dot(s.wi, n), albedo);
      s.isDelta = true; s.valid = true;
      return s;
    }
    float a = m.roughness * m.roughness;
    Onb onb(n);
    float3 lo = onb.toLocal(wo);
    if (lo.z <= 0.0f) return s;
    float3 h = ggxSampleVndf(lo, a, rng.rnd2());
    float3 li = reflect(-lo, h);
    if (li.z <= 0.0f) return s;
    float3 F = schlick3(dot(lo, h), albedo);
    s.wi = onb.toWorld(li);
    s.weight = F * (ggxG(lo, li, a) / ggxG1(lo, a));
    s.pdf = ggxPdf(lo, li, a);
    s.valid = s.pdf > 0.0f;
    return s;
  }
  if (m.kind == MT_WATER || m.kind == MT_DIELECTRIC) {
    float3 refr;
    float eta = frontface ? etaExt / m.ior : m.ior / etaExt;
    float f0 = dielectricF0(eta);
    if (m.kind == MT_WATER || m.roughness < 1e-3f) {
      s.isDelta = true;
      if (refract(rayDir, n, eta, refr)) {
        float c = eta < 1.0f ? -dot(rayDir, n) : -dot(refr, n);
        if (rng.rnd() < schlick(c, f0)) s.wi = normalize(reflect(rayDir, n));
        else s.wi = normalize(refr);
      } else {
        s.wi = normalize(reflect(rayDir, n));
      }
      s.weight = f3(1.0f);
      s.valid = true;
      return s;
    }
    float a = m.roughness * m.roughness;
    Onb onb(n);
    float3 lo = onb.toLocal(wo);
    if (lo.z <= 0.0f) return s;
    float3 h = ggxSampleVndf(lo, a, rng.rnd2());
    float loh = dot(lo, h);
    if (loh <= 0.0f) return s;
    float3 li;
    if (!refract(-lo, h, eta, refr)) {
      li = reflect(-lo, h);
      if (li.z <= 0.0f) return s;
      s.pdf = ggxPdf(lo, li, a);
    } else {
      float c = eta < 1.0f ? loh : -dot(refr, h);
      float pr = schlick(c, f0);
      if (rng.rnd() < pr) {
        li = reflect(-lo, h);
        if (li.z <= 0.0f) return s;
        s.pdf = pr * ggxPdf(lo, li, a);
      } else {
        li = normalize(refr);
        if (li.z >= 0.0f) return s;
        s.pdf = (1.0f - pr) * ggxPdfTransmit(lo, li, h, eta, a);
      }
    }
    s.wi = onb.toWorld(li);
    float w = ggxG(lo, li, a) / ggxG1(lo, a);
    if (li.z < 0.0f) w *= eta * eta;
    s.weight = f3(w);
    s.valid = s.pdf > 0.0f;
    return s;
  }
  if (m.kind == MT_PLASTIC) {
    Onb onb(n);
    float3 lo = onb.toLocal(wo);
    if (lo.z <= 0.0f) return s;
    bool coat = rng.rnd() < 0.5f;
    float3 li;
    if (coat) {
      float rough = std::fmax(m.roughness, 1e-3f);
      li = reflect(-lo, ggxSampleVndf(lo, rough * rough, rng.rnd2()));
    } else {
      li = cosineHemisphere(rng.rnd2());
    }
    if (li.z <= 0.0f) return s;
    PlasticTerms t = plasticTerms(m, albedo, lo, li);
    s.pdf = 0.5f * (t.pSpec + t.pDiff);
    if (s.pdf <= 0.0f) return s;
    s.wi = onb.toWorld(li);
    s.weight = (f3(t.fSpec) + t.fDiff) * (li.z / s.pdf);
    s.valid = true;
    return s;
  }
  return s;
}

// ---- device/light_sample.cuh + device/env_light.cuh --------------------------------------
struct LightSample { float3 wi; float dist; float3 Li; float pdf; bool isDelta; bool valid; };

inline int findInterval(const float* cdf, int n, float u) {          // env_light.cuh:36-43
  int lo = 0, hi = n - 1;
  while (lo + 1 < hi) {
    int mid = (lo + hi) >> 1;
    if (cdf[mid] <= u) lo = mid; else hi = mid;
  }
  return lo;
}
inline float2 envDirToUv(const EnvDesc& env, float3 dir) {           // env_light.cuh:17-22
  float u = (std::atan2(dir.z, dir.x) - env.rotate + SD_PI) * (0.5f * SD_INV_PI);
  u -= std::floor(u);
  float v = std::acos(clampf(dir.y, -1.0f, 1.0f)) * SD_INV_PI;
  return {u, v};
}
inline float3 envEval(const EnvDesc& env, float3 dir) {              // env_light.cuh:24-33
  float2 uv = envDirToUv(env, dir);
  float4 c = texFetchF4(env.texels, env.width, env.height, uv.x, uv.y);
  return f3(c.x, c.y, c.z) * env.intensity;
}
inline LightSample sampleEnv(const EnvDesc& env, Pcg32& rng) {       // env_light.cuh:54-95
  LightSample s;
  s.valid = false; s.isDelta = false; s.pdf = 0.0f; s.dist = 1e16f;
  s.wi = f3(0.0f, 1.0f, 0.0f); s.Li = f3(0.0f);
  float2 rn = rng.rnd2();
  if (!env.importance) {
    s.wi = uniformOnSphere(rn);
    s.pdf = 0.25f * SD_INV_PI;
    s.Li = envEval(env, s.wi);
    s.valid = true;
    return s;
  }
  int row = findInterval(env.margCdf, env.height + 1, rn.x);
  float dm = env.margCdf[row + 1] - env.margCdf[row];
  float dv = dm > 0.0f ? (rn.x - env.margCdf[row]) / dm : 0.5f;
  float v = (row + dv) / env.height;
  const float* cdf = env.condCdf + (size_t)row * (env.width + 1);
  int col = findInterval(cdf, env.width + 1, rn.y);
  float dc = cdf[col + 1] - cdf[col];
  float du = dc > 0.0f ? (rn.y - cdf[col]) / dc : 0.5f;
  float u = (col + du) / env.width;
  float theta = v * SD_PI;
  float sinT = std::sin(theta);
  if (sinT < 1e-6f || dm <= 0.0f || dc <= 0.0f) return s;
  float phi = (2.0f * SD_PI * u - SD_PI) + env.rotate;
  s.wi = f3(sinT * std::cos(phi), std::cos(theta), sinT * std::sin(phi));
  s.pdf = dm * dc * env.width * env.height / (2.0f * SD_PI * SD_PI * sinT);
  s.Li = envEval(env, s.wi);
  s.valid = s.pdf > 0.0f;
  return s;
}
inline float envPdfSolidAngle(const EnvDesc& env, float3 dir) {      // env_light.cuh:104-116
  if (!env.importance) return 0.25f * SD_INV_PI;
  float sinT = std::sqrt(std::fmax(0.0f, 1.0f - dir.y * dir.y));
  if (sinT < 1e-6f) return 0.0f;
  float2 uv = envDirToUv(env, dir);
  int col = std::min((int)(uv.x * env.width), env.width - 1);
  int row = std::min((int)(uv.y * env.height), env.height - 1);
  float dm = env.margCdf[row + 1] - env.margCdf[row];
  const float* cdf = env.condCdf + (size_t)row * (env.width + 1);
  float dc = cdf[col + 1] - cdf[col];
  return dm * dc * env.width * env.height / (2.0f * SD_PI * SD_PI * sinT);
}

inline LightSample sampleLight(const LightDesc& lt, float3 x, Pcg32& rng,
                               const TextureDesc* textures) {        // light_sample.cuh:24-188
  LightSample s;
  s.valid = false; s.isDelta = false; s.pdf = 0.0f; s.dist = 0.0f;
  s.wi = f3(0.0f, 1.0f, 0.0f); s.Li = f3(0.0f);
  if (lt.kind == LT_RECT || lt.kind == LT_DISK) {
    float3 p;
    float tu, tv;
    if (lt.kind == LT_RECT) {
      float a = 2.0f * rng.rnd() - 1.0f;
      float b = 2.0f * rng.rnd() - 1.0f;
      p = lt.p + a * lt.u + b * lt.v;
      tu = (a + 1.0f) * 0.5f; tv = (b + 1.0f) * 0.5f;
    } else {
      float2 d = concentricDisk(rng.rnd2());
      p = lt.p + d.x * lt.u + d.y * lt.v;
      tu = (std::atan2(d.y, d.x) + SD_PI) / (2.0f * SD_PI);
      tv = std::sqrt(d.x * d.x + d.y * d.y);
    }
    float3 to = p - x;
    float d2 = length2(to);
    if (d2 < 1e-10f) return s;
    float dist = std::sqrt(d2);
    float3 wi = to / dist;
    float cosL = -dot(wi, lt.n);
    if (!lt.twoSided && cosL <= 0.0f) return s;
    cosL = std::fabs(cosL);
    if (cosL < 1e-6f) return s;
    s.wi = wi; s.dist = dist; s.Li = lt.L;
    if (lt.texId >= 0 && textures) {
      float4 c = evalTexture(textures[lt.texId], tu, tv);
      s.Li = lt.L * f3(c.x, c.y, c.z);
    }
    s.pdf = d2 / (cosL * lt.area);
    s.valid = true;
    return s;
  }
  if (lt.kind == LT_SPHERE) {
    float3 to = lt.p - x;
    float d2 = length2(to), r2 = lt.radius * lt.radius;
    if (d2 <= r2 * 1.0001f) return s;
    float dist = std::sqrt(d2);
    float3 wc = to / dist;
    float cosMax = std::sqrt(std::fmax(0.0f, 1.0f - r2 / d2));
    float2 u = rng.rnd2();
    float cosT = 1.0f - u.x * (1.0f - cosMax);
    float sinT = std::sqrt(std::fmax(0.0f, 1.0f - cosT * cosT));
    float phi = 2.0f * SD_PI * u.y;
    Onb onb(wc);
    s.wi = onb.toWorld(f3(sinT * std::cos(phi), sinT * std::sin(phi), cosT));
    float b = dot(s.wi, to);
    float det = std::fmax(0.0f, b * b - d2 + r2);
    s.dist = b - std::sqrt(det);
    s.Li = lt.L;
    s.pdf = 1.0f / (2.0f * SD_PI * (1.0f - cosMax));
    s.valid = true;
    return s;
  }
  if (lt.kind == LT_MESH) {
    float uc = rng.rnd();
    int k = findInterval(lt.mCdf, lt.mNumTris + 1, uc);
    uint3 tri = lt.mIndices[k];
    float3 p0 = lt.mPositions[tri.x], p1 = lt.mPositions[tri.y], p2 = lt.mPositions[tri.z];
    float2 r = rng.rnd2();
    float su = std::sqrt(r.x);
    float bx = su * (1.0f - r.y), by = su * r.y;
    float3 p = p0 * (1.0f - bx - by) + p1 * bx + p2 * by;
    float3 ngU = cross(p1 - p0, p2 - p0);
    float ngL2 = length2(ngU);
    if (ngL2 < 1e-20f) return s;
    float3 ng = ngU * (lt.mNgSign / std::sqrt(ngL2));
    float3 to = p - x;
    float d2 = length2(to);
    if (d2 < 1e-10f) return s;
    float dist = std::sqrt(d2);
    float3 wi = to / dist;
    float cosL = -dot(wi, ng);
    if (!lt.twoSided && cosL <= 0.0f) return s;
    cosL = std::fabs(cosL);
    if (cosL < 1e-6f) return s;
    s.wi = wi; s.dist = dist; s.Li = lt.L;
    if (lt.texId >= 0 && textures) {
      float tu, tv;
      if (lt.mUvs) {
        float2 t = lt.mUvs[tri.x] * (1.0f - bx - by) + lt.mUvs[tri.y] * bx + lt.mUvs[tri.z] * by;
        tu = t.x; tv = t.y;
      } else {
        tu = bx; tv = by;
      }
      float4 c = evalTexture(textures[lt.texId], tu, tv);
      s.Li = lt.L * f3(c.x, c.y, c.z);
    }
    s.pdf = d2 / (cosL * lt.area);
    s.valid = true;
    return s;
  }
  if (lt.kind == LT_POINT) {
    s.isDelta = true;
    float3 to = lt.p - x;
    float d2c = length2(to);
    if (d2c < 1e-10f) return s;
    float3 wc = to / std::sqrt(d2c);
    float2 d = concentricDisk(rng.rnd2()) * lt.radius;
    Onb onb(wc);
    float3 p = lt.p + d.x * onb.t + d.y * onb.b;
    float3 top = p - x;
    float d2 = length2(top);
    float dist = std::sqrt(d2);
    s.wi = top / dist;
    s.dist = std::fmax(dist - 1e-4f, 1e-4f);
    s.Li = lt.L / d2;
    s.pdf = 1.0f;
    s.valid = true;
    return s;
  }
  if (lt.kind == LT_DISTANT) {
    s.isDelta = true;
    s.wi = -lt.dir; s.dist = 1e16f; s.Li = lt.L; s.pdf = 1.0f; s.valid = true;
    return s;
  }
  return s;
}
inline float lightPdfSolidAngle(const LightDesc& lt, float3 from, float3 hitP, float3 nHit) {  // light_sample.cuh:197-226
  if (lt.kind == LT_RECT || lt.kind == LT_DISK || lt.kind == LT_MESH) {
    float3 to = hitP - from;
    float d2 = length2(to);
    if (d2 < 1e-10f) return 0.0f;
    float dist = std::sqrt(d2);
    float cosL = std::fabs(dot(to / dist, lt.kind == LT_MESH ? nHit : lt.n));
    if (cosL < 1e-6f) return 0.0f;
    return d2 / (cosL * lt.area);
  }
  if (lt.kind == LT_SPHERE) {
    float3 to = lt.p - from;
    float d2 = length2(to), r2 = lt.radius * lt.radius;
    if (d2 <= r2 * 1.0001f) return 0.0f;
    float cosMax = std::sqrt(std::fmax(0.0f, 1.0f - r2 / d2));
    return 1.0f / (2.0f * SD_PI * (1.0f - cosMax));
  }
  return 0.0f;
}

// ---- device/noise.cuh:12-79 -------------------------------------------------------------
inline float smoothstepf(float e0, float e1, float x) {
  float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
inline unsigned hashU(unsigned x) {
  x = x * 747796405u + 2891336453u;
  x = ((x >> ((x >> 28u) + 4u)) ^ x) * 277803737u;
  return (x >> 22u) ^ x;
}
inline float hashLattice(int x, int y, int z, unsigned seed) {
  unsigned h = hashU((unsigned)x * 73856093u ^ (unsigned)y * 19349663u ^ (unsigned)z * 83492791u ^ seed);
  return (float)h * (1.0f / 4294967296.0f);
}
inline float vnoise(float3 p, unsigned seed) {
  float fx = std::floor(p.x), fy = std::floor(p.y), fz = std::floor(p.z);
  int ix = (int)fx, iy = (int)fy, iz = (int)fz;
  float tx = p.x - fx, ty = p.y - fy, tz = p.z - fz;
  tx = tx * tx * (3.0f - 2.0f * tx);
  ty = ty * ty * (3.0f - 2.0f * ty);
  tz = tz * tz * (3.0f - 2.0f * tz);
  float c[2][2][2];
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++)
      for (int e = 0; e < 2; e++) c[a][b][e] = hashLattice(ix + a, iy + b, iz + e, seed);
  float x00 = c[0][0][0] + (c[1][0][0] - c[0][0][0]) * tx;
  float x10 = c[0][1][0] + (c[1][1][0] - c[0][1][0]) * tx;
  float x01 = c[0][0][1] + (c[1][0][1] - c[0][0][1]) * tx;
  float x11 = c[0][1][1] + (c[1][1][1] - c[0][1][1]) * tx;
  float y0 = x00 + (x10 - x00) * ty;
  float y1 = x01 + (x11 - x01) * ty;
  return y0 + (y1 - y0) * tz;
}
inline float fbm3(float3 p, unsigned seed) {
  float amp = 0.5f, sum = 0.0f;
  for (int i = 0; i < 3; i++) {
    sum += amp * vnoise(p, seed + (unsigned)i * 101u);
    p = 2.03f * p + f3(11.7f, 5.3f, 7.9f);
    amp *= 0.5f;
  }
  return sum;
}
inline float3 waterNormal(float3 x, float3 ns, float3 wo, float amp, float freq) {
  const unsigned SEED = 1337u;
  const float e = 0.05f;
  float3 p = f3(x.x * freq, 0.0f, x.z * freq);
  float hx1 = fbm3(p + f3(e, 0.0f, 0.0f), SEED), hx0 = fbm3(p - f3(e, 0.0f, 0.0f), SEED);
  float hz1 = fbm3(p + f3(0.0f, 0.0f, e), SEED), hz0 = fbm3(p - f3(0.0f, 0.0f, e), SEED);
  float dhdx = (hx1 - hx0) / (2.0f * e), dhdz = (hz1 - hz0) / (2.0f * e);
  float side = ns.y >= 0.0f ? 1.0f : -1.0f;
  float3 n = normalize(f3(-amp * dhdx, 1.0f, -amp * dhdz)) * side;
  if (dot(n, wo) <= 1e-4f) return ns;
  return n;
}

// ---- device/volume.cuh:27-153 (step count from the descriptor) ---------------------------
inline void flameField(const FlameDesc& fl, float3 p, float& sigma, float3& emission) {
  sigma = 0.0f;
  emission = f3(0.0f);
  float h = (p.y - fl.base.y) / fl.height;
  if (h <= 0.0f || h >= 1.0f) return;
  float rx = p.x - fl.base.x, rz = p.z - fl.base.z;
  float d = std::sqrt(rx * rx + rz * rz) / fl.radius;
  float prof = 3.2f * std::sqrt(h) * std::pow(1.0f - h, 1.55f);
  float3 q = f3(rx / fl.radius, (p.y - fl.base.y) / fl.radius * 0.32f, rz / fl.radius);
  float n = fbm3(q * fl.noiseScale, fl.seed);
  float dd = d / std::fmax(prof, 1e-3f) + (n - 0.45f) * 1.0f;
  float mask = smoothstepf(1.0f, 0.62f, dd) * smoothstepf(0.0f, 0.12f, h);
  if (mask <= 0.0f) return;
  sigma = fl.sigma * mask;
  float heat = clampf((0.88f - dd) * (1.25f - h), 0.0f, 1.0f);
  float3 col = f3(std::fmin(heat * 2.6f, 1.0f), std::fmin(heat * heat * 2.1f, 1.0f),
                  std::fmin(heat * heat * heat * 1.7f, 1.0f));
  emission = col * (fl.intensity * mask);
}
inline bool clipFlameBounds(const FlameDesc& fl, float3 o, float3 d, float& t0, float& t1) {
  if (std::fabs(d.y) < 1e-8f) {
    if (o.y < fl.base.y || o.y > fl.base.y + fl.height) return false;
  } else {
    float ta = (fl.base.y - o.y) / d.y;
    float tb = (fl.base.y + fl.height - o.y) / d.y;
    if (ta > tb) std::swap(ta, tb);
    t0 = std::fmax(t0, ta);
    t1 = std::fmin(t1, tb);
  }
  float ox = o.x - fl.base.x, oz = o.z - fl.base.z;
  float a = d.x * d.x + d.z * d.z;
  if (a < 1e-12f) {
    if (ox * ox + oz * oz > fl.radius * fl.radius) return false;
  } else {
    float b = ox * d.x + oz * d.z;
    float c = ox * ox + oz * oz - fl.radius * fl.radius;
    float disc = b * b - a * c;
    if (disc <= 0.0f) return false;
    float s = std::sqrt(disc);
    t0 = std::fmax(t0, (-b - s) / a);
    t1 = std::fmin(t1, (-b + s) / a);
  }
  return t0 < t1;
}
inline float3 marchFlames(const FlameDesc* flames, int nf, float3 o, float3 d, float tEnd, Pcg32& rng,
                          float3& trans) {
  float3 Lv = f3(0.0f);
  for (int i = 0; i < nf; i++) {
    const FlameDesc& fl = flames[i];
    const int STEPS = fl.steps;
    float t0 = 1e-4f, t1 = tEnd;
    if (!clipFlameBounds(fl, o, d, t0, t1)) continue;
    float dt = (t1 - t0) / STEPS;
    float jitter = rng.rnd();
    float tl = 1.0f;
    float3 acc = f3(0.0f);
    for (int k = 0; k < STEPS; k++) {
      float3 p = o + (t0 + (k + jitter) * dt) * d;
      float sg; float3 e;
      flameField(fl, p, sg, e);
      acc += (tl * dt) * e;
      tl *= std::exp(-sg * dt);
      if (tl < 1e-4f) break;
    }
    Lv += trans * acc;
    trans *= tl;
  }
  return Lv;
}
inline float flameTransmittance(const FlameDesc* flames, int nf, float3 o, float3 d, float tEnd,
                                Pcg32& rng, int skip) {
  float tr = 1.0f;
  for (int i = 0; i < nf; i++) {
    if (i == skip) continue;
    const FlameDesc& fl = flames[i];
    const int STEPS = fl.steps;
    float t0 = 1e-4f, t1 = tEnd;
    if (!clipFlameBounds(fl, o, d, t0, t1)) continue;
    float dt = (t1 - t0) / STEPS;
    float jitter = rng.rnd();
    float tl = 1.0f;
    for (int k = 0; k < STEPS; k++) {
      float3 p = o + (t0 + (k + jitter) * dt) * d;
      float sg; float3 e;
      flameField(fl, p, sg, e);
      tl *= std::exp(-sg * dt);
      if (tl < 1e-4f) break;
    }
    tr *= tl;
  }
  return tr;
}

}  // namespace sdo
