// Sampling tables built on the device: the environment map's 2D CDF and the
// area CDF of each emissive mesh instance, with FP64 prefix sums.
//
// Environment (src/env_light.cpp:27-56): per row, the values
// max(lum, 0) * sin(theta_row) (lum the Rec. 709 luminance of the texel, in
// FP32; the product with sin theta exact in FP64) are prefix-summed in FP64,
// each prefix is stored as a float, then divided in FP64 by the row total and
// stored as a float again; the last entry is pinned to 1 and an all-black row
// gets the uniform ramp c / W. The marginal CDF does the same over the row
// totals. Mesh light (src/capi_render.cpp:126-155): world-space vertices
// (the instance transform in FP32), triangle areas 0.5 |e1 x e2| in FP32
// widened to FP64, FP64 prefix, entries normalised the same way.
//
// The reference sums sequentially; here one CTA scans a row (or the whole
// mesh / the marginal) with per-thread sequential segments and a warp-shuffle
// scan of the segment totals, so a double prefix can differ from the
// sequential one in its last bits, which reaches the stored float only when
// the prefix sits next to a float rounding boundary. Every FP32 operation of
// the reference's formula is written with round-to-nearest intrinsics (no
// contraction into FMAs), so the inputs of the sums are the reference's bit
// for bit. sin(theta) comes from the host (sinf, as in the reference) per row.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>

#include "cdf_build.h"
#include "render_session.h"
#include "sd_lights.cuh"

namespace sdb {

constexpr int kScanThreads = 256;

// Exclusive prefix of `v` over the CTA (kScanThreads threads) in FP64, in a
// fixed order: an inclusive shuffle scan within each warp, then a scan of the
// warps' totals. *total (shared) receives the CTA's sum.
__device__ __forceinline__ double blockExclusiveScan(double v, double* total) {
  constexpr int kWarps = kScanThreads / 32;
  __shared__ double warpBase[kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double incl = v;
  for (int off = 1; off < 32; off <<= 1) {
    double y = __shfl_up_sync(0xFFFFFFFFu, incl, off);
    if (lane >= off) incl = __dadd_rn(incl, y);
  }
  double excl = __shfl_up_sync(0xFFFFFFFFu, incl, 1);
  if (lane == 0) excl = 0.0;
  if (lane == 31) warpBase[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    double w = lane < kWarps ? warpBase[lane] : 0.0;
    double wi = w;
    for (int off = 1; off < 32; off <<= 1) {
      double y = __shfl_up_sync(0xFFFFFFFFu, wi, off);
      if (lane >= off) wi = __dadd_rn(wi, y);
    }
    double we = __shfl_up_sync(0xFFFFFFFFu, wi, 1);
    if (lane == 0) we = 0.0;
    if (lane < kWarps) warpBase[lane] = we;
    if (lane == kWarps - 1) *total = wi;
  }
  __syncthreads();
  double r = warp == 0 ? excl : __dadd_rn(warpBase[warp], excl);
  __syncthreads();
  return r;
}

// Luminance of a texel as the reference computes it in FP32, NaN -> 0 and
// negatives -> 0 (fmaxf(lum, 0)).
__device__ __forceinline__ float texelLum(float4 p) {
  float lum = __fadd_rn(__fadd_rn(__fmul_rn(0.2126f, p.x), __fmul_rn(0.7152f, p.y)),
                        __fmul_rn(0.0722f, p.z));
  return lum > 0.0f ? lum : 0.0f;
}

// Stores the running FP64 prefix of values f(i), i in [0, n), as floats at
// out[i + 1] (out[0] = 0), one CTA; returns the total (all threads).
template <typename F>
__device__ double scanSegmented(int n, F f, float* out) {
  __shared__ double total;
  const int per = (n + kScanThreads - 1) / kScanThreads;
  const int b = threadIdx.x * per, e = min(n, b + per);
  double seg = 0.0;
  for (int i = b; i < e; i++) seg = __dadd_rn(seg, f(i));
  double run = blockExclusiveScan(seg, &total);
  for (int i = b; i < e; i++) {
    run = __dadd_rn(run, f(i));
    out[i + 1] = __double2float_rn(run);
  }
  if (threadIdx.x == 0) out[0] = 0.0f;
  __syncthreads();
  return total;
}

// Normalises out[1..n-1] by the total (float prefix / total, FP64), pins
// out[n] = 1; a zero total gives the uniform ramp c / n.
__device__ void normalise(int n, double total, float* out) {
  if (total > 0.0) {
    for (int c = 1 + threadIdx.x; c < n; c += blockDim.x)
      out[c] = __double2float_rn(__ddiv_rn((double)out[c], total));
  } else {
    for (int c = threadIdx.x; c <= n; c += blockDim.x) out[c] = __fdiv_rn((float)c, (float)n);
  }
  __syncthreads();
  if (threadIdx.x == 0) out[n] = 1.0f;
}

__global__ void __launch_bounds__(kScanThreads) envRowCdf(const float4* __restrict__ tex, int W,
                                                          const float* __restrict__ sinT,
                                                          float* cond, double* rowSum) {
  const int row = blockIdx.x;
  const float4* px = tex + (size_t)row * W;
  const double s = (double)sinT[row];
  float* cdf = cond + (size_t)row * (W + 1);
  double total = scanSegmented(W, [&](int i) { return (double)texelLum(px[i]) * s; }, cdf);
  normalise(W, total, cdf);
  if (threadIdx.x == 0) rowSum[row] = total;
}

__global__ void __launch_bounds__(kScanThreads) envMarginalCdf(const double* __restrict__ rowSum,
                                                               int H, float* marg, int* degenerate) {
  double total = scanSegmented(H, [&](int i) { return rowSum[i]; }, marg);
  normalise(H, total, marg);
  if (threadIdx.x == 0) *degenerate = total > 0.0 ? 0 : 1;
}

// World-space vertices of a mesh light: the instance transform applied in
// the reference's FP32 order, m0 x + m1 y + m2 z + m3 per row.
__global__ void meshLightWorld(const float3* __restrict__ pos, int n, Xform xf, float3* wp) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float3 p = pos[i];
    const float* m = xf.m;
    float3 r;
    r.x = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], p.x), __fmul_rn(m[1], p.y)),
                              __fmul_rn(m[2], p.z)), m[3]);
    r.y = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[4], p.x), __fmul_rn(m[5], p.y)),
                              __fmul_rn(m[6], p.z)), m[7]);
    r.z = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[8], p.x), __fmul_rn(m[9], p.y)),
                              __fmul_rn(m[10], p.z)), m[11]);
    wp[i] = r;
  }
}

// 0.5 |(b - a) x (c - a)| in FP32, widened to FP64 (the reference's
// 0.5 * (double)length(cross(...))).
__device__ __forceinline__ double triArea(const float3* wp, uint3 t) {
  float3 a = wp[t.x], b = wp[t.y], c = wp[t.z];
  float ux = __fsub_rn(b.x, a.x), uy = __fsub_rn(b.y, a.y), uz = __fsub_rn(b.z, a.z);
  float vx = __fsub_rn(c.x, a.x), vy = __fsub_rn(c.y, a.y), vz = __fsub_rn(c.z, a.z);
  float cx = __fsub_rn(__fmul_rn(uy, vz), __fmul_rn(uz, vy));
  float cy = __fsub_rn(__fmul_rn(uz, vx), __fmul_rn(ux, vz));
  float cz = __fsub_rn(__fmul_rn(ux, vy), __fmul_rn(uy, vx));
  float len = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(cx, cx), __fmul_rn(cy, cy)),
                                   __fmul_rn(cz, cz)));
  return 0.5 * (double)len;
}

__global__ void __launch_bounds__(kScanThreads) meshLightCdf(const float3* __restrict__ wp,
                                                             const uint3* __restrict__ idx, int n,
                                                             float* cdf, double* total) {
  double t = scanSegmented(n, [&](int i) { return triArea(wp, idx[i]); }, cdf);
  if (t > 0.0) {
    for (int c = 1 + threadIdx.x; c < n; c += blockDim.x)
      cdf[c] = __double2float_rn(__ddiv_rn((double)cdf[c], t));
    __syncthreads();
    if (threadIdx.x == 0) cdf[n] = 1.0f;
  }
  if (threadIdx.x == 0) *total = t;
}

// Guide entries of `rows` CDFs of n entries (row r at cdf + r * stride):
// entry k of a row is the index the plain search (sd_lights.cuh cdfSearch)
// returns for u = k / kCdfGuide, exact in FP32.
__global__ void cdfGuide(const float* cdf, int n, size_t stride, int rows, int* guide) {
  const int total = rows * (kCdfGuide + 1);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int r = i / (kCdfGuide + 1), k = i - r * (kCdfGuide + 1);
    guide[i] = cdfSearch(cdf + (size_t)r * stride, n, (float)k / (float)kCdfGuide);
  }
}

void buildCdfGuideDevice(const float* cdf, int n, size_t stride, int rows, int* guide,
                         cudaStream_t st) {
  const int total = rows * (kCdfGuide + 1);
  const int grid = std::max(1, std::min((total + 255) / 256, 148 * 8));
  cdfGuide<<<grid, 256, 0, st>>>(cdf, n, stride, rows, guide);
  cudaCheck(cudaGetLastError(), "CDF guide launch");
}

void buildEnvCdfDevice(const float4* texels, int w, int h, float* marg, float* cond,
                       bool& degenerate, cudaStream_t st) {
  std::vector<float> sinT(h);
  for (int row = 0; row < h; row++) sinT[row] = sinf(kPi * (row + 0.5f) / h);
  DevBuf dSin, dRow, dDeg;
  dSin.upload(sinT.data(), sinT.size() * sizeof(float));
  dRow.alloc((size_t)h * sizeof(double));
  dDeg.alloc(sizeof(int));
  envRowCdf<<<h, kScanThreads, 0, st>>>(texels, w, (const float*)dSin.ptr, cond,
                                        (double*)dRow.ptr);
  cudaCheck(cudaGetLastError(), "env row CDF launch");
  envMarginalCdf<<<1, kScanThreads, 0, st>>>((const double*)dRow.ptr, h, marg, (int*)dDeg.ptr);
  cudaCheck(cudaGetLastError(), "env marginal CDF launch");
  int deg = 0;
  cudaCheck(cudaMemcpyAsync(&deg, dDeg.ptr, sizeof deg, cudaMemcpyDeviceToHost, st), "env CDF");
  cudaCheck(cudaStreamSynchronize(st), "env CDF");
  degenerate = deg != 0;
}

double buildMeshLightCdfDevice(const float3* pos, int numVerts, const uint3* idx, int numTris,
                               const Xform& xf, float3* worldPos, float* cdf, cudaStream_t st) {
  int grid = (numVerts + 255) / 256;
  if (grid > 1184) grid = 1184;
  if (grid < 1) grid = 1;
  meshLightWorld<<<grid, 256, 0, st>>>(pos, numVerts, xf, worldPos);
  cudaCheck(cudaGetLastError(), "mesh light transform launch");
  DevBuf dTot;
  dTot.alloc(sizeof(double));
  meshLightCdf<<<1, kScanThreads, 0, st>>>(worldPos, idx, numTris, cdf, (double*)dTot.ptr);
  cudaCheck(cudaGetLastError(), "mesh light CDF launch");
  double total = 0.0;
  cudaCheck(cudaMemcpyAsync(&total, dTot.ptr, sizeof total, cudaMemcpyDeviceToHost, st),
            "mesh light CDF");
  cudaCheck(cudaStreamSynchronize(st), "mesh light CDF");
  return total;
}

}  // namespace sdb
