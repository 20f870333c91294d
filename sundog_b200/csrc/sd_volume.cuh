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

// Smoothstep fade of the fractional part; f receives the cell's floor.
SDB_HD float fadeFrac(float x, int& f) {
  float fx = floorf(x);
  f = (int)fx;
  float t = x - fx;
  return t * t * (3.0f - 2.0f * t);
}

// Trilinear blend of a cell's eight lattice values (cYZX naming: c100 is
// x + 1), x first, then y, then z.
SDB_HD float trilerp(float c000, float c100, float c010, float c110, float c001, float c101,
                     float c011, float c111, float tx, float ty, float tz) {
  float x00 = c000 + (c100 - c000) * tx;
  float x10 = c010 + (c110 - c010) * tx;
  float x01 = c001 + (c101 - c001) * tx;
  float x11 = c011 + (c111 - c011) * tx;
  float y0 = x00 + (x10 - x00) * ty;
  float y1 = x01 + (x11 - x01) * ty;
  return y0 + (y1 - y0) * tz;
}

// The same blend on the plane y == 0 (y fade 0: each y lerp returns its
// lower end, a + (b - a) * 0 == a for the finite lattice values).
SDB_HD float bilerpXZ(float c000, float c100, float c001, float c101, float tx, float tz) {
  float x00 = c000 + (c100 - c000) * tx;
  float x01 = c001 + (c101 - c001) * tx;
  return x00 + (x01 - x00) * tz;
}

// Trilinear value noise with smoothstep fade. (device/noise.cuh:32-50)
SDB_HD float valueNoise(float3 p, unsigned seed) {
  int ix, iy, iz;
  float tx = fadeFrac(p.x, ix), ty = fadeFrac(p.y, iy), tz = fadeFrac(p.z, iz);
  return trilerp(latticeValue(ix, iy, iz, seed), latticeValue(ix + 1, iy, iz, seed),
                 latticeValue(ix, iy + 1, iz, seed), latticeValue(ix + 1, iy + 1, iz, seed),
                 latticeValue(ix, iy, iz + 1, seed), latticeValue(ix + 1, iy, iz + 1, seed),
                 latticeValue(ix, iy + 1, iz + 1, seed), latticeValue(ix + 1, iy + 1, iz + 1, seed),
                 tx, ty, tz);
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
  int ix, iz;
  float tx = fadeFrac(p.x, ix), tz = fadeFrac(p.z, iz);
  return bilerpXZ(latticeValue(ix, 0, iz, seed), latticeValue(ix + 1, 0, iz, seed),
                  latticeValue(ix, 0, iz + 1, seed), latticeValue(ix + 1, 0, iz + 1, seed), tx, tz);
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

// The four heights of waveNormal's central differences, fbm3Y0 at
// (x +- e, 0, z) and (x, 0, z +- e), with the lattice values they share read
// once. Per octave the four points' coordinates come from the same
// arithmetic as fbm3Y0's, so the x samples share z and the z samples share
// x, and all share y; e is under half a lattice cell at every octave (0.05,
// 0.10, 0.21), so the x pair spans the cells ixm and ixm + 1 along x and the
// z pair izm and izm + 1 along z (the centre's cells lie between). Block A
// holds x = ixm .. ixm + 2 at the x samples' z cells (izc, izc + 1); the z
// samples' x cells (ixc = ixm or ixm + 1) are inside it, and of their z
// values izm .. izm + 2 block A has the two at izc, izc + 1, so one more
// z row (E) completes them: 16 lattice values instead of 32 per octave (8
// instead of 16 on the plane y == 0). Each sample then blends its own
// cell's eight values with its own fade weights, exactly as valueNoise.
SDB_HD void waveHeights(float3 p, float e, unsigned seed, float& hx1, float& hx0, float& hz1,
                        float& hz0) {
  float3 qxp = p + v3(e, 0.0f, 0.0f), qxm = p - v3(e, 0.0f, 0.0f);
  float3 qzp = p + v3(0.0f, 0.0f, e), qzm = p - v3(0.0f, 0.0f, e);
  float sxp = 0.0f, sxm = 0.0f, szp = 0.0f, szm = 0.0f;
  for (int oct = 0; oct < 3; oct++) {
    const unsigned sd = seed + (unsigned)oct * 101u;
    int ixp, ixm, ixc, izc, izp, izm, iy = 0;
    const float txp = fadeFrac(qxp.x, ixp), txm = fadeFrac(qxm.x, ixm), txc = fadeFrac(qzp.x, ixc);
    const float tzc = fadeFrac(qxp.z, izc), tzp = fadeFrac(qzp.z, izp), tzm = fadeFrac(qzm.z, izm);
    const float ty = oct == 0 ? 0.0f : fadeFrac(qxp.y, iy);
    const int ny = oct == 0 ? 1 : 2;  // y rows that count (one on y == 0)
    // A[dx][dy][dz]: x = ixm + dx, y = iy + dy, z = izc + dz.
    float A[3][2][2];
#pragma unroll
    for (int dx = 0; dx < 3; dx++)
#pragma unroll
      for (int dy = 0; dy < 2; dy++)
#pragma unroll
        for (int dz = 0; dz < 2; dz++)
          A[dx][dy][dz] = dy < ny ? latticeValue(ixm + dx, iy + dy, izc + dz, sd) : 0.0f;
    // E[dx][dy]: the z samples' remaining z row, x = ixc + dx.
    const int zE = izc == izm ? izm + 2 : izm;
    float E[2][2];
#pragma unroll
    for (int dx = 0; dx < 2; dx++)
#pragma unroll
      for (int dy = 0; dy < 2; dy++)
        E[dx][dy] = dy < ny ? latticeValue(ixc + dx, iy + dy, zE, sd) : 0.0f;
    // The z samples' column at x = ixc + dx: z = izc, izc + 1 from A, zE from E.
    const bool oc = ixc != ixm;
    auto col = [&](int dx, int dy, int z) -> float {
      const float a0 = oc ? A[dx + 1][dy][0] : A[dx][dy][0];
      const float a1 = oc ? A[dx + 1][dy][1] : A[dx][dy][1];
      return z == izc ? a0 : (z == izc + 1 ? a1 : E[dx][dy]);
    };
    const bool ob = ixp != ixm;
    float v[4];
    if (oct == 0) {
      v[0] = bilerpXZ(ob ? A[1][0][0] : A[0][0][0], ob ? A[2][0][0] : A[1][0][0],
                      ob ? A[1][0][1] : A[0][0][1], ob ? A[2][0][1] : A[1][0][1], txp, tzc);
      v[1] = bilerpXZ(A[0][0][0], A[1][0][0], A[0][0][1], A[1][0][1], txm, tzc);
      v[2] = bilerpXZ(col(0, 0, izp), col(1, 0, izp), col(0, 0, izp + 1), col(1, 0, izp + 1), txc,
                      tzp);
      v[3] = bilerpXZ(col(0, 0, izm), col(1, 0, izm), col(0, 0, izm + 1), col(1, 0, izm + 1), txc,
                      tzm);
    } else {
      v[0] = trilerp(ob ? A[1][0][0] : A[0][0][0], ob ? A[2][0][0] : A[1][0][0],
                     ob ? A[1][1][0] : A[0][1][0], ob ? A[2][1][0] : A[1][1][0],
                     ob ? A[1][0][1] : A[0][0][1], ob ? A[2][0][1] : A[1][0][1],
                     ob ? A[1][1][1] : A[0][1][1], ob ? A[2][1][1] : A[1][1][1], txp, ty, tzc);
      v[1] = trilerp(A[0][0][0], A[1][0][0], A[0][1][0], A[1][1][0], A[0][0][1], A[1][0][1],
                     A[0][1][1], A[1][1][1], txm, ty, tzc);
      v[2] = trilerp(col(0, 0, izp), col(1, 0, izp), col(0, 1, izp), col(1, 1, izp),
                     col(0, 0, izp + 1), col(1, 0, izp + 1), col(0, 1, izp + 1),
                     col(1, 1, izp + 1), txc, ty, tzp);
      v[3] = trilerp(col(0, 0, izm), col(1, 0, izm), col(0, 1, izm), col(1, 1, izm),
                     col(0, 0, izm + 1), col(1, 0, izm + 1), col(0, 1, izm + 1),
                     col(1, 1, izm + 1), txc, ty, tzm);
    }
    const float amp = oct == 0 ? 0.5f : (oct == 1 ? 0.25f : 0.125f);
    if (oct == 0) {
      sxp = amp * v[0];
      sxm = amp * v[1];
      szp = amp * v[2];
      szm = amp * v[3];
    } else {
      sxp += amp * v[0];
      sxm += amp * v[1];
      szp += amp * v[2];
      szm += amp * v[3];
    }
    qxp = 2.03f * qxp + v3(11.7f, 5.3f, 7.9f);
    qxm = 2.03f * qxm + v3(11.7f, 5.3f, 7.9f);
    qzp = 2.03f * qzp + v3(11.7f, 5.3f, 7.9f);
    qzm = 2.03f * qzm + v3(11.7f, 5.3f, 7.9f);
  }
  hx1 = sxp;
  hx0 = sxm;
  hz1 = szp;
  hz0 = szm;
}

// Wave normal from an fBm height field over world xz by central differences;
// falls back to ns when the perturbed normal would face away from wo.
// (device/noise.cuh:67-79)
SDB_COLD float3 waveNormal(float3 x, float3 ns, float3 wo, float amp, float freq) {
  const unsigned seed = 1337u;
  const float e = 0.05f;
  float3 p = v3(x.x * freq, 0.0f, x.z * freq);
  float hx1, hx0, hz1, hz0;
  // Below 2^20 every octave's coordinates keep a float spacing of at most
  // 0.5, so each pair of samples spans at most two cells, as waveHeights
  // needs; farther out the four fBm sums are taken one by one.
  if (fabsf(p.x) < 1048576.0f && fabsf(p.z) < 1048576.0f) {
    waveHeights(p, e, seed, hx1, hx0, hz1, hz0);
  } else {
    hx1 = fbm3Y0(p + v3(e, 0.0f, 0.0f), seed);
    hx0 = fbm3Y0(p - v3(e, 0.0f, 0.0f), seed);
    hz1 = fbm3Y0(p + v3(0.0f, 0.0f, e), seed);
    hz0 = fbm3Y0(p - v3(0.0f, 0.0f, e), seed);
  }
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
