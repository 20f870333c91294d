// Procedural noise (integer hash -> trilinear value noise -> 3-octave fBm),
// water wave normals, and the emissive flame volumes (emission + absorption,
// no scattering) ray-marched along radiance and shadow segments.
//
// Field definitions, step placement, the per-flame jitter draw and the early
// exit follow device/noise.cuh:18-79 and device/volume.cuh:27-153. The step
// count is a per-flame field (the reference fixes it at 32).
#pragma once

#include "sd_rng.cuh"
#include "sd_types.h"

// Paths most pixels never take (water normals, flame marches, quadric
// roots) are compiled out of line in device code, keeping the hot loop's
// instruction footprint small; host code inlines them as usual.
#ifndef SDB_COLD
#if defined(__CUDA_ARCH__)
#define SDB_COLD static __host__ __device__ __noinline__
#else
#define SDB_COLD static inline
#endif
#endif

namespace sdb {

// Smoothstep that also accepts inverted edges. (device/noise.cuh:12-15)
SDB_HD float smoothRamp(float e0, float e1, float x) {
  float t = clamp01((x - e0) / (e1 - e0));
  return t * t * (3.0f - 2.0f * t);
}

// PCG-style output permutation of a Weyl-stepped word. (device/noise.cuh:18-23)
SDB_HD unsigned mixHash(unsigned x) {
  x = x * 747796405u + 2891336453u;
  x = ((x >> ((x >> 28u) + 4u)) ^ x) * 277803737u;
  return (x >> 22u) ^ x;
}

// Lattice value in [0,1). (device/noise.cuh:25-29)
SDB_HD float latticeValue(int x, int y, int z, unsigned seed) {
  unsigned h = mixHash((unsigned)x * 73856093u ^ (unsigned)y * 19349663u ^
                       (unsigned)z * 83492791u ^ seed);
  return (float)h * (1.0f / 4294967296.0f);
}

// Trilinear value noise with smoothstep fade. (device/noise.cuh:32-50)
SDB_HD float valueNoise(float3 p, unsigned seed) {
  float fx = floorf(p.x), fy = floorf(p.y), fz = floorf(p.z);
  int ix = (int)fx, iy = (int)fy, iz = (int)fz;
  float tx = p.x - fx, ty = p.y - fy, tz = p.z - fz;
  tx = tx * tx * (3.0f - 2.0f * tx);
  ty = ty * ty * (3.0f - 2.0f * ty);
  tz = tz * tz * (3.0f - 2.0f * tz);
  float c000 = latticeValue(ix, iy, iz, seed), c100 = latticeValue(ix + 1, iy, iz, seed);
  float c010 = latticeValue(ix, iy + 1, iz, seed), c110 = latticeValue(ix + 1, iy + 1, iz, seed);
  float c001 = latticeValue(ix, iy, iz + 1, seed), c101 = latticeValue(ix + 1, iy, iz + 1, seed);
  float c011 = latticeValue(ix, iy + 1, iz + 1, seed), c111 = latticeValue(ix + 1, iy + 1, iz + 1, seed);
  float x00 = c000 + (c100 - c000) * tx;
  float x10 = c010 + (c110 - c010) * tx;
  float x01 = c001 + (c101 - c001) * tx;
  float x11 = c011 + (c111 - c011) * tx;
  float y0 = x00 + (x10 - x00) * ty;
  float y1 = x01 + (x11 - x01) * ty;
  return y0 + (y1 - y0) * tz;
}

// Three octaves, lacunarity 2.03, gain 0.5. (device/noise.cuh:53-61)
SDB_HD float fbm3(float3 p, unsigned seed) {
  float amp = 0.5f, sum = 0.0f;
  for (int i = 0; i < 3; i++) {
    sum += amp * valueNoise(p, seed + (unsigned)i * 101u);
    p = 2.03f * p + v3(11.7f, 5.3f, 7.9f);
    amp *= 0.5f;
  }
  return sum;
}

// valueNoise at a point with p.y == 0: the y fade weight is exactly 0, so
// each y lerp returns its lower end unchanged (a + (b - a) * 0 == a for the
// finite lattice values) and the four lattice values at iy + 1 never count.
// The same value from half the hashes.
SDB_HD float valueNoiseY0(float3 p, unsigned seed) {
  float fx = floorf(p.x), fz = floorf(p.z);
  int ix = (int)fx, iz = (int)fz;
  float tx = p.x - fx, tz = p.z - fz;
  tx = tx * tx * (3.0f - 2.0f * tx);
  tz = tz * tz * (3.0f - 2.0f * tz);
  float c000 = latticeValue(ix, 0, iz, seed), c100 = latticeValue(ix + 1, 0, iz, seed);
  float c001 = latticeValue(ix, 0, iz + 1, seed), c101 = latticeValue(ix + 1, 0, iz + 1, seed);
  float x00 = c000 + (c100 - c000) * tx;
  float x01 = c001 + (c101 - c001) * tx;
  return x00 + (x01 - x00) * tz;
}

// fbm3 of a point on the plane y == 0 (the wave height field): the first
// octave through valueNoiseY0, the others as in fbm3.
SDB_HD float fbm3Y0(float3 p, unsigned seed) {
  float sum = 0.5f * valueNoiseY0(p, seed);
  p = 2.03f * p + v3(11.7f, 5.3f, 7.9f);
  sum += 0.25f * valueNoise(p, seed + 101u);
  p = 2.03f * p + v3(11.7f, 5.3f, 7.9f);
  sum += 0.125f * valueNoise(p, seed + 202u);
  return sum;
}

// Wave normal from an fBm height field over world xz by central differences;
// falls back to ns when the perturbed normal would face away from wo.
// (device/noise.cuh:67-79)
SDB_COLD float3 waveNormal(float3 x, float3 ns, float3 wo, float amp, float freq) {
  const unsigned seed = 1337u;
  const float e = 0.05f;
  float3 p = v3(x.x * freq, 0.0f, x.z * freq);
  float hx1 = fbm3Y0(p + v3(e, 0.0f, 0.0f), seed), hx0 = fbm3Y0(p - v3(e, 0.0f, 0.0f), seed);
  float hz1 = fbm3Y0(p + v3(0.0f, 0.0f, e), seed), hz0 = fbm3Y0(p - v3(0.0f, 0.0f, e), seed);
  float dhdx = (hx1 - hx0) / (2.0f * e);
  float dhdz = (hz1 - hz0) / (2.0f * e);
  float side = ns.y >= 0.0f ? 1.0f : -1.0f;
  float3 n = unit(v3(-amp * dhdx, 1.0f, -amp * dhdz)) * side;
  if (dot(n, wo) <= 1e-4f) return ns;
  return n;
}

// Absorption density and emitted radiance per unit length of a flame at p.
// (device/volume.cuh:27-56)
SDB_HD void flameAt(const SdFlame& fl, float3 p, float& sigma, float3& eps) {
  sigma = 0.0f;
  eps = v3(0.0f);
  float h = (p.y - fl.base.y) / fl.height;
  if (h <= 0.0f || h >= 1.0f) return;
  float rx = p.x - fl.base.x, rz = p.z - fl.base.z;
  float d = sqrtf(rx * rx + rz * rz) / fl.radius;
  const float sh = sqrtf(h);
  // (1 - h)^1.55 <= 1 - h on [0, 1], so 3.2001 sqrt(h) (1 - h) bounds the
  // profile from above (the margin covers powf's error and the roundings);
  // where even that bound puts the step outside the mask for every noise
  // value (the test below with 1.4502 for 1.45), the exact test would too:
  // the empty medium, without powf.
  if (d >= 1.4502f * fmaxf(3.2001f * sh * (1.0f - h), 1e-3f)) return;
  float prof = 3.2f * sh * powf(1.0f - h, 1.55f);
  const float dp = d / fmaxf(prof, 1e-3f);
  // The noise term n - 0.45 is at least -0.45 (fBm is non-negative), so where
  // dp - 0.45 already reaches the mask's outer edge (1) the mask is 0 for
  // every noise value: return the empty medium without evaluating the noise
  // (the same result: rounding is monotonic).
  if (dp - 0.45f >= 1.0f) return;
  float3 q = v3(rx / fl.radius, (p.y - fl.base.y) / fl.radius * 0.32f, rz / fl.radius);
  float n = fbm3(q * fl.noiseScale, fl.seed);
  float dd = dp + (n - 0.45f) * 1.0f;
  float mask = smoothRamp(1.0f, 0.62f, dd) * smoothRamp(0.0f, 0.12f, h);
  if (mask <= 0.0f) return;
  sigma = fl.sigma * mask;
  float heat = clamp01((0.88f - dd) * (1.25f - h));
  float3 col = v3(fminf(heat * 2.6f, 1.0f), fminf(heat * heat * 2.1f, 1.0f),
                  fminf(heat * heat * heat * 1.7f, 1.0f));
  eps = col * (fl.intensity * mask);
}

// Clip [t0,t1] to the flame's upright bounding cylinder. (device/volume.cuh:59-85)
SDB_HD bool flameClip(const SdFlame& fl, float3 o, float3 d, float& t0, float& t1) {
  if (fabsf(d.y) < 1e-8f) {
    if (o.y < fl.base.y || o.y > fl.base.y + fl.height) return false;
  } else {
    float ta = (fl.base.y - o.y) / d.y;
    float tb = (fl.base.y + fl.height - o.y) / d.y;
    if (ta > tb) {
      float tmp = ta;
      ta = tb;
      tb = tmp;
    }
    t0 = fmaxf(t0, ta);
    t1 = fminf(t1, tb);
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
    float s = sqrtf(disc);
    t0 = fmaxf(t0, (-b - s) / a);
    t1 = fminf(t1, (-b + s) / a);
  }
  return t0 < t1;
}

// Emission along [1e-4, tEnd] of o + t d through every flame, weighted by the
// running transmittance; the segment's transmittance is folded into trans.
// One draw per entered flame. (device/volume.cuh:90-115)
SDB_COLD float3 flameMarch(const SdFlame* fls, int nfl, float3 o, float3 d, float tEnd,
                         Pcg& rng, float3& trans) {
  float3 Lv = v3(0.0f);
  for (int i = 0; i < nfl; i++) {
    const SdFlame& fl = fls[i];
    float t0 = 1e-4f, t1 = tEnd;
    if (!flameClip(fl, o, d, t0, t1)) continue;
    int steps = fl.steps;
    float dt = (t1 - t0) / steps;
    float jit = rng.uni();
    float tl = 1.0f;
    float3 acc = v3(0.0f);
    for (int k = 0; k < steps; k++) {
      float3 p = o + (t0 + (k + jit) * dt) * d;
      float sg;
      float3 e;
      flameAt(fl, p, sg, e);
      acc += (tl * dt) * e;
      tl *= expf(-sg * dt);
      if (tl < 1e-4f) break;
    }
    Lv += trans * acc;
    trans *= tl;
  }
  return Lv;
}

// Transmittance-only twin of flameMarch for shadow segments: same steps, same
// jitter draw, same exponentials; skip exempts a light's owning flame.
// (device/volume.cuh:129-153)
SDB_COLD float flameShadow(const SdFlame* fls, int nfl, float3 o, float3 d, float tEnd,
                         Pcg& rng, int skip) {
  float tr = 1.0f;
  for (int i = 0; i < nfl; i++) {
    if (i == skip) continue;
    const SdFlame& fl = fls[i];
    float t0 = 1e-4f, t1 = tEnd;
    if (!flameClip(fl, o, d, t0, t1)) continue;
    int steps = fl.steps;
    float dt = (t1 - t0) / steps;
    float jit = rng.uni();
    float tl = 1.0f;
    for (int k = 0; k < steps; k++) {
      float3 p = o + (t0 + (k + jit) * dt) * d;
      float sg;
      float3 e;
      flameAt(fl, p, sg, e);
      tl *= expf(-sg * dt);
      if (tl < 1e-4f) break;
    }
    tr *= tl;
  }
  return tr;
}

}  // namespace sdb
