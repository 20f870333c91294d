// The five analytic primitives in canonical object space (ray direction not
// normalised; t is shared with world space). Each returns up to two roots in
// (tmin, tmax) with the object-space front normal and uv.
//   sphere    r = 1 at the origin
//   rect      [-1,1]^2 in the XZ plane, front +Y
//   disk      r <= 1 in the XZ plane, front +Y
//   cylinder  x^2 + z^2 = 1, |y| <= 1, open, front outward
//   parabola  y = (x^2 + z^2) / 2, x^2 + z^2 <= 1, front on the convex side
// Root formulas and uv maps follow device/intersect.cuh:32-182.
#pragma once

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

struct QHit {
  float t;
  float3 n;
  float u, v;
};
struct QHits {
  QHit h[2];
  int n;
};

SDB_HD void sphereUv(float3 n, float& u, float& v) {
  u = (atan2f(n.z, n.x) + kPi) / (2.0f * kPi);
  v = (asinf(clampf(n.y, -1.0f, 1.0f)) + kPi / 2.0f) / kPi;
}

SDB_HD QHits hitSphere(float3 o, float3 d, float tmin, float tmax) {
  QHits r;
  r.n = 0;
  float a = dot(d, d);
  float b = dot(o, d);
  float c = dot(o, o) - 1.0f;
  float disc = b * b - a * c;
  if (disc <= 0.0f) return r;
  float s = sqrtf(disc);
  float roots[2] = {(-b - s) / a, (-b + s) / a};
  for (int i = 0; i < 2; i++) {
    float t = roots[i];
    if (t > tmin && t < tmax) {
      QHit& h = r.h[r.n++];
      float3 p = o + t * d;
      h.t = t;
      h.n = unit(p);
      sphereUv(h.n, h.u, h.v);
    }
  }
  return r;
}

SDB_HD QHits hitRect(float3 o, float3 d, float tmin, float tmax) {
  QHits r;
  r.n = 0;
  if (d.y == 0.0f) return r;
  float t = -o.y / d.y;
  if (t <= tmin || t >= tmax) return r;
  float x = o.x + t * d.x, z = o.z + t * d.z;
  if (fabsf(x) > 1.0f || fabsf(z) > 1.0f) return r;
  QHit& h = r.h[r.n++];
  h.t = t;
  h.n = v3(0.0f, 1.0f, 0.0f);
  h.u = (x + 1.0f) * 0.5f;
  h.v = (z + 1.0f) * 0.5f;
  return r;
}

SDB_HD QHits hitDisk(float3 o, float3 d, float tmin, float tmax) {
  QHits r;
  r.n = 0;
  if (d.y == 0.0f) return r;
  float t = -o.y / d.y;
  if (t <= tmin || t >= tmax) return r;
  float x = o.x + t * d.x, z = o.z + t * d.z;
  float rad = sqrtf(x * x + z * z);
  if (rad > 1.0f) return r;
  QHit& h = r.h[r.n++];
  h.t = t;
  h.n = v3(0.0f, 1.0f, 0.0f);
  h.u = (atan2f(z, x) + kPi) / (2.0f * kPi);
  h.v = rad;
  return r;
}

SDB_HD QHits hitCylinder(float3 o, float3 d, float tmin, float tmax) {
  QHits r;
  r.n = 0;
  float a = d.x * d.x + d.z * d.z;
  if (a == 0.0f) return r;
  float b = o.x * d.x + o.z * d.z;
  float c = o.x * o.x + o.z * o.z - 1.0f;
  float disc = b * b - a * c;
  if (disc <= 0.0f) return r;
  float s = sqrtf(disc);
  float roots[2] = {(-b - s) / a, (-b + s) / a};
  for (int i = 0; i < 2; i++) {
    float t = roots[i];
    if (t > tmin && t < tmax) {
      float3 p = o + t * d;
      if (fabsf(p.y) <= 1.0f) {
        QHit& h = r.h[r.n++];
        h.t = t;
        h.n = unit(v3(p.x, 0.0f, p.z));
        h.u = (atan2f(p.z, p.x) + kPi) / (2.0f * kPi);
        h.v = (p.y + 1.0f) * 0.5f;
      }
    }
  }
  return r;
}

SDB_HD QHits hitParabola(float3 o, float3 d, float tmin, float tmax) {
  QHits r;
  r.n = 0;
  float A = 0.5f * (d.x * d.x + d.z * d.z);
  float B = o.x * d.x + o.z * d.z - d.y;
  float C = 0.5f * (o.x * o.x + o.z * o.z) - o.y;
  float t0 = 0.0f, t1 = 0.0f;
  int n;
  if (fabsf(A) < 1e-12f) {
    if (B == 0.0f) return r;
    t0 = -C / B;
    n = 1;
  } else {
    float disc = B * B - 4.0f * A * C;
    if (disc <= 0.0f) return r;
    float s = sqrtf(disc);
    t0 = (-B - s) / (2.0f * A);
    t1 = (-B + s) / (2.0f * A);
    n = 2;
  }
  for (int i = 0; i < n; i++) {
    float t = i == 0 ? t0 : t1;
    if (t > tmin && t < tmax) {
      float3 p = o + t * d;
      if (p.x * p.x + p.z * p.z <= 1.0f) {
        QHit& h = r.h[r.n++];
        h.t = t;
        h.n = unit(v3(p.x, -1.0f, p.z));
        h.u = (atan2f(p.z, p.x) + kPi) / (2.0f * kPi);
        h.v = sqrtf(p.x * p.x + p.z * p.z);
      }
    }
  }
  return r;
}

SDB_COLD QHits hitQuadric(int kind, float3 o, float3 d, float tmin, float tmax) {
  switch (kind) {
    case GK_SPHERE: return hitSphere(o, d, tmin, tmax);
    case GK_RECT: return hitRect(o, d, tmin, tmax);
    case GK_DISK: return hitDisk(o, d, tmin, tmax);
    case GK_CYLINDER: return hitCylinder(o, d, tmin, tmax);
    case GK_PARABOLA: return hitParabola(o, d, tmin, tmax);
    default: {
      QHits r;
      r.n = 0;
      return r;
    }
  }
}

// Object-space bounds (rect/disk/parabola padded by 1e-4 in y).
// (device/intersect.cuh:165-182)
SDB_HD void quadricBounds(int kind, float3& lo, float3& hi) {
  const float e = 1e-4f;
  switch (kind) {
    case GK_RECT:
    case GK_DISK:
      lo = v3(-1.0f, -e, -1.0f);
      hi = v3(1.0f, e, 1.0f);
      break;
    case GK_PARABOLA:
      lo = v3(-1.0f, -e, -1.0f);
      hi = v3(1.0f, 0.5f + e, 1.0f);
      break;
    default:
      lo = v3(-1.0f);
      hi = v3(1.0f);
      break;
  }
}

}  // namespace sdb
