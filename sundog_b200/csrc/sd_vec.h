// Vector / affine math shared by host scene assembly and the sm_100a kernels.
//
// float3 operations are spelled out component-wise so that host (g++) and
// device (nvcc) evaluate the same IEEE operations; the device build keeps
// FMA contraction on, so device results may differ from host ones by a few
// ulp where a multiply feeds an add.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define SDB_HD __host__ __device__ __forceinline__
#else
#define SDB_HD inline
#endif

namespace sdb {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618379067154f;

SDB_HD float3 v3(float s) { return make_float3(s, s, s); }
SDB_HD float3 v3(float x, float y, float z) { return make_float3(x, y, z); }

SDB_HD float3 operator+(float3 a, float3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
SDB_HD float3 operator-(float3 a, float3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
SDB_HD float3 operator-(float3 a) { return v3(-a.x, -a.y, -a.z); }
SDB_HD float3 operator*(float3 a, float3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
SDB_HD float3 operator*(float3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
SDB_HD float3 operator*(float s, float3 a) { return v3(a.x * s, a.y * s, a.z * s); }
SDB_HD float3 operator/(float3 a, float s) {
  float r = 1.0f / s;  // one reciprocal, three multiplies
  return v3(a.x * r, a.y * r, a.z * r);
}
SDB_HD float3& operator+=(float3& a, float3 b) { a = a + b; return a; }
SDB_HD float3& operator*=(float3& a, float3 b) { a = a * b; return a; }
SDB_HD float3& operator*=(float3& a, float s) { a = a * s; return a; }

SDB_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
SDB_HD float3 cross(float3 a, float3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
SDB_HD float len2(float3 a) { return dot(a, a); }
SDB_HD float len(float3 a) { return sqrtf(dot(a, a)); }
SDB_HD float3 unit(float3 a) { return a * (1.0f / sqrtf(dot(a, a))); }
SDB_HD float clamp01(float x) { return fminf(1.0f, fmaxf(0.0f, x)); }
SDB_HD float clampf(float x, float lo, float hi) { return fminf(hi, fmaxf(lo, x)); }
SDB_HD float3 vmin(float3 a, float3 b) { return v3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
SDB_HD float3 vmax(float3 a, float3 b) { return v3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
SDB_HD float hmax(float3 v) { return fmaxf(v.x, fmaxf(v.y, v.z)); }
SDB_HD float3 vexp(float3 a) { return v3(expf(a.x), expf(a.y), expf(a.z)); }
SDB_HD float3 mirror(float3 v, float3 n) { return v - 2.0f * dot(v, n) * n; }
SDB_HD float comp(float3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

// Snell: v unit incident (toward the surface), n unit normal facing v's
// origin side, eta = n_incident / n_transmitted. False on total internal
// reflection. (device/math.cuh:52-58)
SDB_HD bool snell(float3 v, float3 n, float eta, float3& t) {
  float ci = -dot(v, n);
  float k = 1.0f - eta * eta * (1.0f - ci * ci);
  if (k < 0.0f) return false;
  t = eta * v + (eta * ci - sqrtf(k)) * n;
  return true;
}

// Schlick Fresnel, scalar and per-channel F0. (device/math.cuh:60-69)
SDB_HD float fresnelSchlick(float c, float f0) {
  float m = clamp01(1.0f - c);
  float m2 = m * m;
  return f0 + (1.0f - f0) * m2 * m2 * m;
}
SDB_HD float3 fresnelSchlick3(float c, float3 f0) {
  float m = clamp01(1.0f - c);
  float m2 = m * m;
  float w = m2 * m2 * m;
  return f0 + (v3(1.0f) - f0) * w;
}

// Orthonormal frame around a unit normal, branch-free (Duff et al. 2017,
// "Building an Orthonormal Basis, Revisited"). (device/math.cuh:72-83)
struct Frame {
  float3 t, b, n;
  SDB_HD explicit Frame(float3 nn) : n(nn) {
    float sg = copysignf(1.0f, nn.z);
    float a = -1.0f / (sg + nn.z);
    float c = nn.x * nn.y * a;
    t = v3(1.0f + sg * nn.x * nn.x * a, sg * c, -sg * nn.x);
    b = v3(c, sg + nn.y * nn.y * a, -nn.y);
  }
  SDB_HD float3 toWorld(float3 v) const { return v.x * t + v.y * b + v.z * n; }
  SDB_HD float3 toLocal(float3 v) const { return v3(dot(v, t), dot(v, b), dot(v, n)); }
};

// Row-major 3x4 affine map (object -> world).
struct Xform {
  float m[12];
  SDB_HD static Xform ident() {
    Xform x = {{1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0}};
    return x;
  }
  SDB_HD float3 point(float3 p) const {
    return v3(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3],
              m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
              m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]);
  }
  SDB_HD float3 vec(float3 v) const {
    return v3(m[0] * v.x + m[1] * v.y + m[2] * v.z,
              m[4] * v.x + m[5] * v.y + m[6] * v.z,
              m[8] * v.x + m[9] * v.y + m[10] * v.z);
  }
};

// a after b. Same accumulation order as device/math.cuh:103-117 so that
// composed object transforms are bit-identical to the reference's.
SDB_HD Xform compose(const Xform& a, const Xform& b) {
  Xform r;
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++)
      r.m[i * 4 + j] = a.m[i * 4 + 0] * b.m[j] + a.m[i * 4 + 1] * b.m[4 + j] +
                       a.m[i * 4 + 2] * b.m[8 + j];
    r.m[i * 4 + 3] = a.m[i * 4 + 0] * b.m[3] + a.m[i * 4 + 1] * b.m[7] +
                     a.m[i * 4 + 2] * b.m[11] + a.m[i * 4 + 3];
  }
  return r;
}

// Orientation sign of the mapped unit axes; cross products of world vectors
// carry it, inverse-transpose normals do not. (device/math.cuh:123-125)
SDB_HD float orientSign(float3 ux, float3 uy, float3 uz) {
  return dot(uy, cross(uz, ux)) < 0.0f ? -1.0f : 1.0f;
}

// Ray origin pushed off a surface along n (which faces the outgoing side),
// scaled with the point's magnitude. (device/math.cuh:151-154)
SDB_HD float3 nudge(float3 p, float3 n) {
  float s = 1e-4f * (1.0f + fmaxf(fabsf(p.x), fmaxf(fabsf(p.y), fabsf(p.z))));
  return p + n * s;
}

}  // namespace sdb
