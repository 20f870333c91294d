// PCG32 (O'Neill 2014, pcg-random.org: 64-bit LCG state, XSH-RR output) and
// the sample warps built on it. Integer stream is bit-identical to
// device/rng.cuh:10-35; seeding is init((pixel << 32) ^ sample, seed)
// (device/programs.cu:329-330).
#pragma once

#include "sd_vec.h"

namespace sdb {

constexpr uint64_t kPcgMul = 6364136223846793005ULL;

struct Pcg {
  uint64_t state;
  uint64_t inc;

  SDB_HD uint32_t next() {
    uint64_t s = state;
    state = s * kPcgMul + inc;
    uint32_t x = (uint32_t)(((s >> 18u) ^ s) >> 27u);
    uint32_t r = (uint32_t)(s >> 59u);
    return (x >> r) | (x << ((32u - r) & 31u));
  }
  // Stream selection and seeding as in the PCG reference implementation's
  // pcg32_srandom_r: inc = 2*seq + 1, step, add the seed, step.
  SDB_HD static Pcg seeded(uint64_t seed, uint64_t seq) {
    Pcg g;
    g.state = 0u;
    g.inc = (seq << 1u) | 1u;
    g.next();
    g.state += seed;
    g.next();
    return g;
  }
  // 24 high bits -> float in [0, 1).
  SDB_HD float uni() { return (float)(next() >> 8) * 0x1p-24f; }
  SDB_HD float2 uni2() {
    float a = uni();
    float b = uni();
    return make_float2(a, b);
  }
};

// Uniform direction on the unit sphere. (device/rng.cuh:38-43)
SDB_HD float3 sphereDir(float2 u) {
  float z = 1.0f - 2.0f * u.x;
  float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
  float phi = 2.0f * kPi * u.y;
  return v3(r * cosf(phi), r * sinf(phi), z);
}

// Shirley-Chiu concentric square -> disk map. (device/rng.cuh:46-53)
SDB_HD float2 diskConcentric(float2 u) {
  float ox = 2.0f * u.x - 1.0f, oy = 2.0f * u.y - 1.0f;
  if (ox == 0.0f && oy == 0.0f) return make_float2(0.0f, 0.0f);
  float r, th;
  if (fabsf(ox) > fabsf(oy)) {
    r = ox;
    th = (kPi / 4.0f) * (oy / ox);
  } else {
    r = oy;
    th = (kPi / 2.0f) - (kPi / 4.0f) * (ox / oy);
  }
  return make_float2(r * cosf(th), r * sinf(th));
}

// Cosine-weighted direction about +Z via Malley's method. (device/rng.cuh:56-60)
SDB_HD float3 cosineDir(float2 u) {
  float2 d = diskConcentric(u);
  float z = sqrtf(fmaxf(0.0f, 1.0f - d.x * d.x - d.y * d.y));
  return v3(d.x, d.y, z);
}

}  // namespace sdb
