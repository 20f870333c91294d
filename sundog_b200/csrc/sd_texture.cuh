// Texture lookups. Procedural kinds follow device/texture_eval.cuh:11-46.
// Image and environment lookups restate the CUDA texture unit's bilinear
// filter in software (CUDA C Programming Guide, "Texture Fetching": taps at
// floor(x - 0.5), weights quantised to 1.8 fixed point), which is what the
// reference gets from tex2D (device/texture_eval.cuh:31,
// device/env_light.cuh:27): wrap on u, wrap (images) or clamp (environment)
// on v, sRGB decode per texel before filtering for sRGB images.
#pragma once

#include "sd_types.h"

namespace sdb {

// Bilinear weight as the texture unit stores it: 8 fractional bits.
SDB_HD float texWeight(float f) { return rintf(f * 256.0f) * (1.0f / 256.0f); }

SDB_HD float srgbToLinear(float c) {
  return c <= 0.04045f ? c * (1.0f / 12.92f) : powf((c + 0.055f) * (1.0f / 1.055f), 2.4f);
}

SDB_HD int wrapIndex(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}
SDB_HD int clampIndex(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

// Tap coordinates and weights for a normalised coordinate on an axis of n
// texels. wrap: coordinate folded into [0,1) first, taps modulo n.
struct TexAxis {
  int i0, i1;
  float w;  // weight of i1
};
SDB_HD TexAxis texAxis(float c, int n, bool wrap) {
  if (wrap) c = c - floorf(c);
  float x = c * (float)n - 0.5f;
  float fl = floorf(x);
  TexAxis a;
  int i = (int)fl;
  a.w = texWeight(x - fl);
  if (wrap) {
    a.i0 = wrapIndex(i, n);
    a.i1 = wrapIndex(i + 1, n);
  } else {
    a.i0 = clampIndex(i, n);
    a.i1 = clampIndex(i + 1, n);
  }
  return a;
}

SDB_HD float4 lerp4(float4 a, float4 b, float w) {
  float v = 1.0f - w;
  return make_float4(v * a.x + w * b.x, v * a.y + w * b.y, v * a.z + w * b.z,
                     v * a.w + w * b.w);
}

// Float RGBA texel grid, bilinear, wrap u / clamp v (environment maps).
SDB_HD float4 sampleFloat4(const float4* tex, int W, int H, float u, float v) {
  TexAxis ax = texAxis(u, W, true);
  TexAxis ay = texAxis(v, H, false);
  float4 t00 = tex[(size_t)ay.i0 * W + ax.i0], t10 = tex[(size_t)ay.i0 * W + ax.i1];
  float4 t01 = tex[(size_t)ay.i1 * W + ax.i0], t11 = tex[(size_t)ay.i1 * W + ax.i1];
  return lerp4(lerp4(t00, t10, ax.w), lerp4(t01, t11, ax.w), ay.w);
}

SDB_HD float4 texelRgba8(uchar4 c, bool srgb) {
  float r = c.x * (1.0f / 255.0f), g = c.y * (1.0f / 255.0f), b = c.z * (1.0f / 255.0f);
  if (srgb) {
    r = srgbToLinear(r);
    g = srgbToLinear(g);
    b = srgbToLinear(b);
  }
  return make_float4(r, g, b, c.w * (1.0f / 255.0f));
}

// RGBA8 image, bilinear, wrap both axes; v = 0 is the bottom of the image
// (the reference samples tex2D(u, 1 - v) on a top-row-first array).
SDB_HD float4 sampleImage(const SdTexture& t, float u, float v) {
  TexAxis ax = texAxis(u, t.imgW, true);
  TexAxis ay = texAxis(1.0f - v, t.imgH, true);
  bool s = t.srgb != 0;
  const uchar4* im = t.img;
  float4 t00 = texelRgba8(im[(size_t)ay.i0 * t.imgW + ax.i0], s);
  float4 t10 = texelRgba8(im[(size_t)ay.i0 * t.imgW + ax.i1], s);
  float4 t01 = texelRgba8(im[(size_t)ay.i1 * t.imgW + ax.i0], s);
  float4 t11 = texelRgba8(im[(size_t)ay.i1 * t.imgW + ax.i1], s);
  return lerp4(lerp4(t00, t10, ax.w), lerp4(t01, t11, ax.w), ay.w);
}

// rgb + alpha (alpha is only meaningful for image cutouts).
// (device/texture_eval.cuh:11-38)
SDB_HD float4 texLookup(const SdTexture& t, float u, float v) {
  switch (t.kind) {
    case TX_SOLID:
      return make_float4(t.a.x, t.a.y, t.a.z, 1.0f);
    case TX_CHECKER: {
      int iu = (int)floorf(u * t.scale.x);
      int iv = (int)floorf(v * t.scale.y);
      float3 c = (((iu + iv) & 1) == 0) ? t.a : t.b;
      return make_float4(c.x, c.y, c.z, 1.0f);
    }
    case TX_GRID: {
      float fu = u * t.scale.x - floorf(u * t.scale.x);
      float fv = v * t.scale.y - floorf(v * t.scale.y);
      float w = t.width;
      bool line = fu < w || fv < w || fu > 1.0f - w || fv > 1.0f - w;
      float3 c = line ? t.b : t.a;
      return make_float4(c.x, c.y, c.z, 1.0f);
    }
    case TX_IMAGE:
      return sampleImage(t, u, v);
    default:
      return make_float4(1.0f, 0.0f, 1.0f, 1.0f);
  }
}

// device/texture_eval.cuh:41-46
SDB_HD float3 surfaceAlbedo(const SdMaterial& m, const SdTexture* tex, float u, float v) {
  if (m.texId < 0) return m.color;
  float4 c = texLookup(tex[m.texId], u, v);
  return v3(c.x, c.y, c.z);
}

}  // namespace sdb
