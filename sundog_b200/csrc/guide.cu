// Learned path guiding: the network's training and inference kernels and the
// online schedule that interleaves them with rendering.
//
// Network (guide_net.h): 48 inputs -> 3 x 64 ReLU -> 48 outputs describing an
// 8-lobe von Mises-Fisher mixture over incident directions. Weights are BF16,
// every product accumulates in FP32 on the tensor cores (tcgen05.mma kind::f16
// for inference, mma.m16n8k16.bf16 in the fused training step).
//
// guideTrainKernel: one fused forward + backward pass over a batch of
//   training records. A warp owns 16 records; the activations of all three
//   hidden layers stay in registers as MMA fragments (the accumulator layout
//   of two adjacent 16x8 tiles is the operand layout of the next 16x16 step,
//   so a layer's output feeds the next layer without leaving registers).
//   The loss gradient of each record's mixture is computed by one lane. The
//   backward chain dH = dZ W runs in registers the same way; the weight
//   gradients dW = dZ^T H reduce over the CTA's 128 records with MMAs on
//   transposed copies in shared memory and are accumulated in shared memory
//   across the CTA's tiles, then added to the global gradient once per CTA.
// guideForwardTc: the forward pass alone on tcgen05 tensor cores (TMEM
//   accumulators, one elected thread issuing the MMAs), for the mixture-table
//   bake (one row per grid cell and normal direction) and the raw-output
//   check. The fused training kernel keeps warp-level MMAs: its backward
//   pass reduces weight gradients over records with transposed operands that
//   live in registers between layers, and at 64-wide layers its time goes to
//   barriers and the per-record loss head, not to the MMA rate.
// guideAdamKernel: Adam on the FP32 master parameters; refreshes the BF16
//   weight copy.
//
// Loss: the KL divergence from the normalised target F (the luminance of the
// incident radiance times |cos| to the normal) to the mixture q, estimated from samples drawn with
// density p: L = -(1/B) sum_i c_i log q(w_i | x_i, n_i), c_i = (F_i / p_i) /
// mean(F / p), c_i clamped at kWeightClamp (Mueller et al., "Neural
// Importance Sampling", 2019, eq. 6).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "../../include/sundog_api.h"
#include "abi_util.h"
#include "guide.h"
#include "guide_net.h"
#include "kernels.h"
#include "render_session.h"
#include "sd_guide.cuh"

namespace sdb {

typedef __nv_bfloat16 bf16;

namespace {

constexpr int kWarps = 8;
constexpr int kThreads = 32 * kWarps;
constexpr int kTileRows = 16 * kWarps;  // records per CTA tile
constexpr int kS48 = 56;                // padded shared-memory row strides
constexpr int kS64 = 72;                //   (elements), conflict-free for
constexpr int kST = kTileRows + 8;      //   the fragment loads below
constexpr int kOutStride = 49;
constexpr float kWeightClamp = 100.0f;

// Shared-memory carve-up of the training kernel (bytes): weights, biases and
// output tiles first, then the backward pass's transposes and accumulators.
constexpr int oSW0 = 0;
constexpr int oSW1 = oSW0 + kNetHid * kS48 * 2;
constexpr int oSW2 = oSW1 + kNetHid * kS64 * 2;
constexpr int oSW3 = oSW2 + kNetHid * kS64 * 2;
constexpr int oSBias = oSW3 + kNetOut * kS64 * 2;
constexpr int oSOut = oSBias + (kNetParams - kNetWeights) * 4;
constexpr int kSmemForward = oSOut + kWarps * 16 * kOutStride * 4;
constexpr int oSW1T = kSmemForward;
constexpr int oSW2T = oSW1T + kNetHid * kS64 * 2;
constexpr int oSW3T = oSW2T + kNetHid * kS64 * 2;
constexpr int oSZT = oSW3T + kNetHid * kS48 * 2;
constexpr int oSHT = oSZT + kNetHid * kST * 2;
constexpr int oSdW = oSHT + kNetHid * kST * 2;
constexpr int kSmemTrain = oSdW + kNetParams * 4;
static_assert(kSmemTrain <= 227 * 1024, "training kernel shared memory");
static_assert(oSBias % 16 == 0 && oSOut % 16 == 0 && oSZT % 16 == 0 && oSdW % 16 == 0, "align");

__device__ __forceinline__ void mma16816(float (&c)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ bool bfPositive(uint32_t bits16) {
  return (bits16 & 0x8000u) == 0 && (bits16 & 0x7FFFu) != 0;
}
__device__ __forceinline__ uint32_t ld32(const bf16* p) {
  return *reinterpret_cast<const uint32_t*>(p);
}

// Copies the BF16 weights into padded shared-memory matrices (and, for
// training, their transposes) and the FP32 biases.
__device__ void loadNet(unsigned char* sm, const bf16* wb, const float* params, bool transposes) {
  bf16* sW0 = (bf16*)(sm + oSW0);
  bf16* sW1 = (bf16*)(sm + oSW1);
  bf16* sW2 = (bf16*)(sm + oSW2);
  bf16* sW3 = (bf16*)(sm + oSW3);
  bf16* sW1T = (bf16*)(sm + oSW1T);
  bf16* sW2T = (bf16*)(sm + oSW2T);
  bf16* sW3T = (bf16*)(sm + oSW3T);
  float* sB = (float*)(sm + oSBias);
  for (int i = threadIdx.x; i < kNetWeights; i += blockDim.x) {
    bf16 w = wb[i];
    if (i < kOffW1) {
      int o = i / kNetIn, c = i % kNetIn;
      sW0[o * kS48 + c] = w;
    } else if (i < kOffW2) {
      int j = i - kOffW1, o = j / kNetHid, c = j % kNetHid;
      sW1[o * kS64 + c] = w;
      if (transposes) sW1T[c * kS64 + o] = w;
    } else if (i < kOffW3) {
      int j = i - kOffW2, o = j / kNetHid, c = j % kNetHid;
      sW2[o * kS64 + c] = w;
      if (transposes) sW2T[c * kS64 + o] = w;
    } else {
      int j = i - kOffW3, o = j / kNetHid, c = j % kNetHid;
      sW3[o * kS64 + c] = w;
      if (transposes) sW3T[c * kS48 + o] = w;
    }
  }
  for (int i = threadIdx.x; i < kNetParams - kNetWeights; i += blockDim.x)
    sB[i] = params[kNetWeights + i];
}

// acc[NT] = A[KC] x B (+ bias): B[k][n] = W[n][k] read from a [n][k] matrix
// with row stride `stride`; 16 rows per warp, NT x 8 columns.
template <int KC, int NT>
__device__ __forceinline__ void warpGemm(const uint32_t (&A)[KC][4], const bf16* sW, int stride,
                                         const float* bias, float (&acc)[NT][4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < NT; nt++) {
    float b0 = bias ? bias[8 * nt + 2 * t] : 0.0f;
    float b1 = bias ? bias[8 * nt + 2 * t + 1] : 0.0f;
    acc[nt][0] = b0;
    acc[nt][1] = b1;
    acc[nt][2] = b0;
    acc[nt][3] = b1;
  }
#pragma unroll
  for (int kc = 0; kc < KC; kc++) {
#pragma unroll
    for (int nt = 0; nt < NT; nt++) {
      const bf16* w = sW + (8 * nt + g) * stride + 16 * kc + 2 * t;
      mma16816(acc[nt], A[kc], ld32(w), ld32(w + 8));
    }
  }
}

// Accumulators of 2 KC column tiles -> operand fragments (ReLU, BF16).
template <int KC>
__device__ __forceinline__ void packRelu(const float (&acc)[2 * KC][4], uint32_t (&A)[KC][4]) {
#pragma unroll
  for (int kc = 0; kc < KC; kc++) {
    A[kc][0] = pack2(fmaxf(acc[2 * kc][0], 0.0f), fmaxf(acc[2 * kc][1], 0.0f));
    A[kc][1] = pack2(fmaxf(acc[2 * kc][2], 0.0f), fmaxf(acc[2 * kc][3], 0.0f));
    A[kc][2] = pack2(fmaxf(acc[2 * kc + 1][0], 0.0f), fmaxf(acc[2 * kc + 1][1], 0.0f));
    A[kc][3] = pack2(fmaxf(acc[2 * kc + 1][2], 0.0f), fmaxf(acc[2 * kc + 1][3], 0.0f));
  }
}

// dZ = dH where the layer's output H is positive (ReLU derivative), as
// operand fragments.
template <int KC>
__device__ __forceinline__ void maskPack(const float (&acc)[2 * KC][4], const uint32_t (&H)[KC][4],
                                         uint32_t (&D)[KC][4]) {
#pragma unroll
  for (int kc = 0; kc < KC; kc++) {
#pragma unroll
    for (int reg = 0; reg < 4; reg++) {
      const int nt = 2 * kc + (reg >> 1), pr = reg & 1;
      uint32_t h = H[kc][reg];
      float lo = bfPositive(h & 0xFFFFu) ? acc[nt][2 * pr] : 0.0f;
      float hi = bfPositive(h >> 16) ? acc[nt][2 * pr + 1] : 0.0f;
      D[kc][reg] = pack2(lo, hi);
    }
  }
}

// Writes a warp's 16 x (16 KC) fragment matrix transposed into dst[col][row]
// (row stride kST) at rows rowBase..rowBase+15.
template <int KC>
__device__ __forceinline__ void storeT(const uint32_t (&F)[KC][4], bf16* dst, int rowBase) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  unsigned short* d = reinterpret_cast<unsigned short*>(dst);
#pragma unroll
  for (int kc = 0; kc < KC; kc++) {
#pragma unroll
    for (int reg = 0; reg < 4; reg++) {
      int row = rowBase + g + (reg & 1) * 8;
      int col = 16 * kc + 2 * t + (reg >> 1) * 8;
      d[col * kST + row] = (unsigned short)(F[kc][reg] & 0xFFFFu);
      d[(col + 1) * kST + row] = (unsigned short)(F[kc][reg] >> 16);
    }
  }
}

// dW[M x N] += ZT[M x 128] x HT[N x 128]^T and db[M] += row sums of ZT,
// over the CTA's 128 records (shared-memory operands, FP32 accumulation).
template <int M, int N>
__device__ __forceinline__ void weightGrad(const bf16* sZT, const bf16* sHT, float* dW, float* db) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  constexpr int NTL = N / 8, tiles = (M / 16) * NTL;
  for (int tile = warp; tile < tiles; tile += kWarps) {
    const int m0 = (tile / NTL) * 16, n0 = (tile % NTL) * 8;
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int kc = 0; kc < kTileRows / 16; kc++) {
      const bf16* za = sZT + (m0 + g) * kST + 16 * kc + 2 * t;
      uint32_t a[4] = {ld32(za), ld32(za + 8 * kST), ld32(za + 8), ld32(za + 8 * kST + 8)};
      const bf16* hb = sHT + (n0 + g) * kST + 16 * kc + 2 * t;
      mma16816(acc, a, ld32(hb), ld32(hb + 8));
    }
    dW[(m0 + g) * N + n0 + 2 * t] += acc[0];
    dW[(m0 + g) * N + n0 + 2 * t + 1] += acc[1];
    dW[(m0 + g + 8) * N + n0 + 2 * t] += acc[2];
    dW[(m0 + g + 8) * N + n0 + 2 * t + 1] += acc[3];
  }
  for (int o = threadIdx.x; o < M; o += blockDim.x) {
    float s = 0.0f;
    const __nv_bfloat162* z = reinterpret_cast<const __nv_bfloat162*>(sZT + o * kST);
    for (int r = 0; r < kTileRows / 2; r++) {
      float2 f = __bfloat1622float2(z[r]);
      s += f.x + f.y;
    }
    db[o] += s;
  }
}

// Input fragments for the warp's rows g and g+8 (positions normalised to
// [0,1]^3). Column pairs are (sin, cos) of one frequency, or two normal
// components, or zero.
__device__ __forceinline__ uint32_t featurePair(float3 p, float3 n, int col) {
  if (col < 2 * 3 * kNetFreqs) {
    int i = col / (2 * kNetFreqs), j = (col % (2 * kNetFreqs)) >> 1;
    float s, c;
    sincospif(comp(p, i) * (float)(1 << j), &s, &c);
    return pack2(s, c);
  }
  if (col == 32) return pack2(n.x, n.y);
  if (col == 34) return pack2(n.z, 0.0f);
  return 0u;
}

__device__ __forceinline__ void inputFrags(float3 p0, float3 n0, float3 p1, float3 n1,
                                           uint32_t (&X)[3][4]) {
  const int t = threadIdx.x & 3;
#pragma unroll
  for (int kc = 0; kc < 3; kc++) {
#pragma unroll
    for (int reg = 0; reg < 4; reg++) {
      int col = 16 * kc + 2 * t + (reg >> 1) * 8;
      X[kc][reg] = (reg & 1) ? featurePair(p1, n1, col) : featurePair(p0, n0, col);
    }
  }
}

struct Acts {
  uint32_t x[3][4], h0[4][4], h1[4][4], h2[4][4];
};

// Forward pass of the warp's 16 rows; the 48 outputs go to sOut[16][kOutStride].
__device__ __forceinline__ void forwardWarp(const unsigned char* sm, Acts& a, float* sOut) {
  const bf16* sW0 = (const bf16*)(sm + oSW0);
  const bf16* sW1 = (const bf16*)(sm + oSW1);
  const bf16* sW2 = (const bf16*)(sm + oSW2);
  const bf16* sW3 = (const bf16*)(sm + oSW3);
  const float* sB = (const float*)(sm + oSBias);
  float acc[8][4];
  warpGemm<3, 8>(a.x, sW0, kS48, sB + (kOffB0 - kNetWeights), acc);
  packRelu<4>(acc, a.h0);
  warpGemm<4, 8>(a.h0, sW1, kS64, sB + (kOffB1 - kNetWeights), acc);
  packRelu<4>(acc, a.h1);
  warpGemm<4, 8>(a.h1, sW2, kS64, sB + (kOffB2 - kNetWeights), acc);
  packRelu<4>(acc, a.h2);
  float out[6][4];
  warpGemm<4, 6>(a.h2, sW3, kS64, sB + (kOffB3 - kNetWeights), out);
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < 6; nt++) {
    sOut[g * kOutStride + 8 * nt + 2 * t] = out[nt][0];
    sOut[g * kOutStride + 8 * nt + 2 * t + 1] = out[nt][1];
    sOut[(g + 8) * kOutStride + 8 * nt + 2 * t] = out[nt][2];
    sOut[(g + 8) * kOutStride + 8 * nt + 2 * t + 1] = out[nt][3];
  }
}

struct Lobe {
  float3 mu;
  float kappa, logw, rn, dKappa;  // dKappa: d kappa / d s (0 where clamped)
};

__device__ __forceinline__ void decodeLobes(const float* o, Lobe (&L)[kGuideLobes]) {
  float zmax = -1e30f;
#pragma unroll
  for (int k = 0; k < kGuideLobes; k++) zmax = fmaxf(zmax, o[5 * k + 4]);
  float zs = 0.0f;
#pragma unroll
  for (int k = 0; k < kGuideLobes; k++) zs += expf(o[5 * k + 4] - zmax);
  float lse = zmax + logf(zs);
#pragma unroll
  for (int k = 0; k < kGuideLobes; k++) {
    float3 r = v3(o[5 * k], o[5 * k + 1], o[5 * k + 2]);
    float rn = fmaxf(len(r), 1e-4f);
    L[k].mu = r * (1.0f / rn);
    L[k].rn = rn;
    float s = o[5 * k + 3];
    float sp = s > 15.0f ? s : log1pf(expf(s));
    float kap = sp + kKappaMin;
    float sig = 1.0f / (1.0f + expf(-s));
    if (kap > kKappaMax) {
      kap = kKappaMax;
      sig = 0.0f;
    }
    L[k].kappa = kap;
    L[k].dKappa = sig;
    L[k].logw = o[5 * k + 4] - lse;
  }
}

// log of the vMF normalisation kappa / (2 pi (1 - e^-2kappa)).
__device__ __forceinline__ float vmfLogNorm(float kappa) {
  return logf(kappa) - 1.8378770664f - log1pf(-expf(-2.0f * kappa));
}

// Loss -c log q(w) of one record and its gradient d[40] w.r.t. the outputs.
__device__ float headLossGrad(const float* o, float3 w, float c, float* d) {
  Lobe L[kGuideLobes];
  decodeLobes(o, L);
  float lq[kGuideLobes], cosm[kGuideLobes];
  float lmax = -1e30f;
#pragma unroll
  for (int k = 0; k < kGuideLobes; k++) {
    cosm[k] = dot(L[k].mu, w);
    lq[k] = L[k].logw + vmfLogNorm(L[k].kappa) + L[k].kappa * (cosm[k] - 1.0f);
    lmax = fmaxf(lmax, lq[k]);
  }
  float sum = 0.0f;
#pragma unroll
  for (int k = 0; k < kGuideLobes; k++) sum += expf(lq[k] - lmax);
  float logq = lmax + logf(sum);
#pragma unroll
  for (int k = 0; k < kGuideLobes; k++) {
    float gam = expf(lq[k] - logq);
    float wk = expf(L[k].logw);
    float kap = L[k].kappa;
    d[5 * k + 4] = -c * (gam - wk);
    float dlk = 1.0f / kap - 2.0f / expm1f(2.0f * kap) + (cosm[k] - 1.0f);
    d[5 * k + 3] = -c * gam * dlk * L[k].dKappa;
    float3 dr = (w - cosm[k] * L[k].mu) * (-c * gam * kap / L[k].rn);
    d[5 * k] = dr.x;
    d[5 * k + 1] = dr.y;
    d[5 * k + 2] = dr.z;
  }
  return -c * logq;
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

struct TrainArgs {
  const bf16* wb;
  const float* params;
  float* grads;
  float* loss;
  const float4* records;
  const unsigned long long* count;  // records written (may exceed cap)
  unsigned long long cap;
  const float* sumF;                // sum of F / p over the records
  int batch;
  int sequential;                   // row i uses record i (gradient check)
  unsigned long long seed;
  int step;
  float3 lo, invExt;
};

__device__ __forceinline__ float3 normPos(float3 x, float3 lo, float3 invExt) {
  float3 p = (x - lo) * invExt;
  return v3(clamp01(p.x), clamp01(p.y), clamp01(p.z));
}

__global__ void __launch_bounds__(kThreads, 1) guideTrainKernel(TrainArgs a) {
  extern __shared__ __align__(16) unsigned char sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2;
  float* sdW = (float*)(sm + oSdW);
  for (int i = threadIdx.x; i < kNetParams; i += blockDim.x) sdW[i] = 0.0f;
  loadNet(sm, a.wb, a.params, true);
  __syncthreads();

  unsigned long long n = *a.count;
  if (n > a.cap) n = a.cap;
  const float meanF = n ? *a.sumF / (float)n : 1.0f;
  const int tiles = (a.batch + kTileRows - 1) / kTileRows;
  float* sOut = (float*)(sm + oSOut) + warp * 16 * kOutStride;
  bf16* sZT = (bf16*)(sm + oSZT);
  bf16* sHT = (bf16*)(sm + oSHT);
  const bf16* sW1T = (const bf16*)(sm + oSW1T);
  const bf16* sW2T = (const bf16*)(sm + oSW2T);
  const bf16* sW3T = (const bf16*)(sm + oSW3T);
  float lossAcc = 0.0f;

  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int rowBase = tile * kTileRows + warp * 16;
    auto recordOf = [&](int row) -> unsigned long long {
      if (n == 0) return 0ull;
      if (a.sequential) return (unsigned long long)min((unsigned long long)row, n - 1);
      return mix64(a.seed ^ ((unsigned long long)a.step << 32) ^ (unsigned long long)row) % n;
    };
    Acts act;
    {
      // Rows past the batch take a fixed finite input (their loss weight is
      // zero, and finite activations keep 0 x activation = 0 in dW).
      float3 p[2] = {v3(0.5f), v3(0.5f)}, nn[2] = {v3(0.0f, 0.0f, 1.0f), v3(0.0f, 0.0f, 1.0f)};
#pragma unroll
      for (int h = 0; h < 2; h++) {
        int row = rowBase + g + 8 * h;
        if (row < a.batch && n > 0) {
          unsigned long long r = recordOf(row);
          float4 x = a.records[3 * r], nr = a.records[3 * r + 1];
          p[h] = normPos(v3(x.x, x.y, x.z), a.lo, a.invExt);
          nn[h] = v3(nr.x, nr.y, nr.z);
        }
      }
      inputFrags(p[0], nn[0], p[1], nn[1], act.x);
    }
    forwardWarp(sm, act, sOut);
    __syncwarp();
    if (lane < 16) {
      int row = rowBase + lane;
      float c = 0.0f;  // rows past the batch (or no records) carry no loss
      float3 w = v3(0.0f, 0.0f, 1.0f);
      if (row < a.batch && n > 0) {
        unsigned long long r = recordOf(row);
        float4 x = a.records[3 * r], wi = a.records[3 * r + 2];
        w = v3(wi.x, wi.y, wi.z);
        c = fminf(x.w / meanF, kWeightClamp) / (float)a.batch;
      }
      float o[kNetLobeOut], d[kNetLobeOut];
      for (int j = 0; j < kNetLobeOut; j++) o[j] = sOut[lane * kOutStride + j];
      if (c > 0.0f) {
        lossAcc += headLossGrad(o, w, c, d);
      } else {
        for (int j = 0; j < kNetLobeOut; j++) d[j] = 0.0f;
      }
      for (int j = 0; j < kNetLobeOut; j++) sOut[lane * kOutStride + j] = d[j];
      for (int j = kNetLobeOut; j < kNetOut; j++) sOut[lane * kOutStride + j] = 0.0f;
    }
    __syncwarp();
    uint32_t dO[3][4];
    {
      const int t = lane & 3;
#pragma unroll
      for (int kc = 0; kc < 3; kc++) {
#pragma unroll
        for (int reg = 0; reg < 4; reg++) {
          int row = g + (reg & 1) * 8, col = 16 * kc + 2 * t + (reg >> 1) * 8;
          dO[kc][reg] = pack2(sOut[row * kOutStride + col], sOut[row * kOutStride + col + 1]);
        }
      }
    }
    const int cr = warp * 16;  // this warp's rows within the CTA tile
    float acc[8][4];
    uint32_t dZ[4][4], dZb[4][4];
    // Output layer.
    storeT<3>(dO, sZT, cr);
    storeT<4>(act.h2, sHT, cr);
    warpGemm<3, 8>(dO, sW3T, kS48, nullptr, acc);
    maskPack<4>(acc, act.h2, dZ);
    __syncthreads();
    weightGrad<kNetOut, kNetHid>(sZT, sHT, sdW + kOffW3, sdW + kOffB3);
    __syncthreads();
    // Hidden layer 2.
    storeT<4>(dZ, sZT, cr);
    storeT<4>(act.h1, sHT, cr);
    warpGemm<4, 8>(dZ, sW2T, kS64, nullptr, acc);
    maskPack<4>(acc, act.h1, dZb);
    __syncthreads();
    weightGrad<kNetHid, kNetHid>(sZT, sHT, sdW + kOffW2, sdW + kOffB2);
    __syncthreads();
    // Hidden layer 1.
    storeT<4>(dZb, sZT, cr);
    storeT<4>(act.h0, sHT, cr);
    warpGemm<4, 8>(dZb, sW1T, kS64, nullptr, acc);
    maskPack<4>(acc, act.h0, dZ);
    __syncthreads();
    weightGrad<kNetHid, kNetHid>(sZT, sHT, sdW + kOffW1, sdW + kOffB1);
    __syncthreads();
    // Input layer.
    storeT<4>(dZ, sZT, cr);
    storeT<3>(act.x, sHT, cr);
    __syncthreads();
    weightGrad<kNetHid, kNetIn>(sZT, sHT, sdW + kOffW0, sdW + kOffB0);
    __syncthreads();
  }
  for (int off = 16; off > 0; off >>= 1) lossAcc += __shfl_down_sync(0xFFFFFFFFu, lossAcc, off);
  if (lane == 0 && lossAcc != 0.0f) atomicAdd(a.loss, lossAcc);
  if (blockIdx.x < tiles)
    for (int i = threadIdx.x; i < kNetParams; i += blockDim.x)
      if (sdW[i] != 0.0f) atomicAdd(a.grads + i, sdW[i]);
}

struct ForwardArgs {
  const bf16* wb;
  const float* params;
  int rows;
  const float* queries;  // raw-output mode: rows x 6 (position in [0,1]^3, normal)
  float* outputs;        // raw-output mode: rows x 40
  float4* lobes;         // bake mode: [cell][8]
  float* cdf;            // bake mode: [cell][8]
};

// Bake mode (queries == nullptr): row = grid cell x normal direction, with
// the cell centre as position, and the kernel writes the cache entries
// sd_guide.cuh reads; otherwise raw outputs for the queries.
// ---- forward pass on tcgen05 (5th-generation tensor cores, TMEM accumulators) --
//
// One CTA of 128 threads runs 128 rows through the network, one row per
// thread: thread t builds row t's input features and, after each layer, reads
// row t of the accumulator from tensor memory (TMEM lane t). A layer is K/16
// tcgen05.mma steps of M=128 x N x K=16 issued by one thread, BF16 operands
// from shared memory, FP32 accumulators in TMEM, completion signalled through
// an mbarrier. Operands use the canonical K-major layout without swizzle:
// core matrices of 8 rows x 16 bytes, the two 8-element K halves of a step
// 128 bytes apart (leading offset), 8-row groups K*16 bytes apart (stride
// offset). The activations between layers go TMEM -> registers (bias, ReLU,
// BF16) -> shared memory, never to global memory.
namespace tc {

constexpr int kRows = 128;
constexpr int kCtaThreads = 128;
constexpr int oW0 = 0;                               // 64 x 48
constexpr int oW1 = oW0 + kNetHid * kNetIn * 2;      // 64 x 64
constexpr int oW2 = oW1 + kNetHid * kNetHid * 2;     // 64 x 64
constexpr int oW3 = oW2 + kNetHid * kNetHid * 2;     // 48 x 64
constexpr int oA = oW3 + kNetOut * kNetHid * 2;      // 128 x 64 activations
constexpr int oBias = oA + kRows * kNetHid * 2;
constexpr int oBar = oBias + (kNetParams - kNetWeights) * 4;
constexpr int oTmem = oBar + 8;
constexpr int kSmem = oTmem + 8;
constexpr uint32_t kTmemCols = 64;                   // N <= 64 FP32 accumulators
constexpr unsigned kWaitLimit = 1u << 24;            // mbarrier polls before giving up
static_assert(oA % 128 == 0 && oBar % 8 == 0, "tcgen05 shared-memory layout");

// Byte offset of element (r, k) of a K-major matrix with K columns.
__device__ __forceinline__ uint32_t coreOff(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor: start address, leading byte offset 128,
// stride byte offset K*16, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smemDesc(uint32_t saddr, int K) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) |
         ((uint64_t)((((uint32_t)K * 16u) >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N and M encoded as N/8 and M/16.
__device__ __forceinline__ uint32_t instrDesc(int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(kRows >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t dTmem, uint64_t a, uint64_t b, uint32_t idesc,
                                    uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(dTmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(bar)
               : "memory");
}

__device__ __forceinline__ bool tryWait(uint32_t bar, uint32_t phase) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(done)
      : "r"(bar), "r"(phase)
      : "memory");
  return done != 0;
}

// 16 FP32 accumulator columns [col, col+16) of this thread's TMEM lane.
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}

}  // namespace tc

__device__ int g_tcTimeout;  // set when an mbarrier wait hit its limit

__global__ void __launch_bounds__(tc::kCtaThreads, 4) guideForwardTc(ForwardArgs a) {
  using namespace tc;
  extern __shared__ __align__(1024) unsigned char sm[];
  const int t = threadIdx.x, warp = t >> 5;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
  const uint32_t bar = sbase + oBar;
  float* sB = (float*)(sm + oBias);

  // Weights in the canonical layout, biases, barrier, TMEM.
  for (int i = t; i < kNetWeights; i += kCtaThreads) {
    unsigned short w = reinterpret_cast<const unsigned short*>(a.wb)[i];
    uint32_t off;
    if (i < kOffW1) off = oW0 + coreOff(i / kNetIn, i % kNetIn, kNetIn);
    else if (i < kOffW2) off = oW1 + coreOff((i - kOffW1) / kNetHid, (i - kOffW1) % kNetHid, kNetHid);
    else if (i < kOffW3) off = oW2 + coreOff((i - kOffW2) / kNetHid, (i - kOffW2) % kNetHid, kNetHid);
    else off = oW3 + coreOff((i - kOffW3) / kNetHid, (i - kOffW3) % kNetHid, kNetHid);
    *reinterpret_cast<unsigned short*>(sm + off) = w;
  }
  for (int i = t; i < kNetParams - kNetWeights; i += kCtaThreads) sB[i] = a.params[kNetWeights + i];
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     sbase + oTmem),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + oTmem);
  const uint32_t myLane = tmem + ((uint32_t)(warp * 32) << 16);

  const int layerK[4] = {kNetIn, kNetHid, kNetHid, kNetHid};
  const int layerN[4] = {kNetHid, kNetHid, kNetHid, kNetOut};
  const int layerW[4] = {oW0, oW1, oW2, oW3};
  const int layerB[4] = {kOffB0 - kNetWeights, kOffB1 - kNetWeights, kOffB2 - kNetWeights,
                         kOffB3 - kNetWeights};
  uint32_t phase = 0;
  bool failed = false;
  const int tiles = (a.rows + kRows - 1) / kRows;
  for (int tile = blockIdx.x; tile < tiles && !failed; tile += gridDim.x) {
    const int row = tile * kRows + t;
    // Input features of this thread's row (same definition as featurePair).
    {
      int r = min(row, a.rows - 1);
      float3 p, n;
      if (a.queries) {
        const float* q = a.queries + 6 * (size_t)r;
        p = v3(q[0], q[1], q[2]);
        n = v3(q[3], q[4], q[5]);
      } else {
        int bin = r % kGuideNormals, cell = r / kGuideNormals;
        int iz = cell % kGuideGrid, iy = (cell / kGuideGrid) % kGuideGrid,
            ix = cell / (kGuideGrid * kGuideGrid);
        const float inv = 1.0f / kGuideGrid;
        p = v3((ix + 0.5f) * inv, (iy + 0.5f) * inv, (iz + 0.5f) * inv);
        float sgn = (bin & 1) ? -1.0f : 1.0f;
        n = v3(bin >> 1 == 0 ? sgn : 0.0f, bin >> 1 == 1 ? sgn : 0.0f, bin >> 1 == 2 ? sgn : 0.0f);
      }
      for (int col = 0; col < kNetIn; col += 2) {
        uint32_t pr = featurePair(p, n, col);
        *reinterpret_cast<uint32_t*>(sm + oA + coreOff(t, col, kNetIn)) = pr;
      }
    }
    float out[kNetOut];
    for (int l = 0; l < 4 && !failed; l++) {
      const int K = layerK[l], N = layerN[l];
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (t == 0) {
        const uint32_t idesc = instrDesc(N);
        for (int kk = 0; kk < K / 16; kk++)
          mma(tmem, smemDesc(sbase + oA + kk * 256, K), smemDesc(sbase + layerW[l] + kk * 256, K),
              idesc, kk > 0 ? 1u : 0u);
        commit(bar);
      }
      unsigned polls = 0;
      bool timedOut = false;
      while (!tryWait(bar, phase)) {
        if (++polls >= kWaitLimit) {
          timedOut = true;
          break;
        }
      }
      phase ^= 1u;
      // One decision for the whole block, so no thread is left at a barrier.
      failed = __syncthreads_or(timedOut) != 0;
      if (failed) {
        if (t == 0) atomicExch(&g_tcTimeout, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      float acc[64];
      for (int c = 0; c < N; c += 16) {
        float v[16];
        tc::ld16(myLane + (uint32_t)c, v);
#pragma unroll
        for (int j = 0; j < 16; j++) acc[c + j] = v[j];
      }
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      const float* bias = sB + layerB[l];
      if (l < 3) {
        // Next layer's operand: this row, 64 BF16 values after bias + ReLU.
        for (int c = 0; c < kNetHid; c += 2) {
          uint32_t pr = pack2(fmaxf(acc[c] + bias[c], 0.0f), fmaxf(acc[c + 1] + bias[c + 1], 0.0f));
          *reinterpret_cast<uint32_t*>(sm + oA + coreOff(t, c, kNetHid)) = pr;
        }
      } else {
        for (int c = 0; c < kNetOut; c++) out[c] = acc[c] + bias[c];
      }
    }
    if (failed) break;
    if (row < a.rows) {
      if (a.queries) {
        for (int j = 0; j < kNetLobeOut; j++) a.outputs[(size_t)row * kNetLobeOut + j] = out[j];
      } else {
        Lobe L[kGuideLobes];
        decodeLobes(out, L);
        float accw = 0.0f;
        for (int k = 0; k < kGuideLobes; k++) {
          float kap = L[k].kappa;
          float3 km = L[k].mu * kap;
          a.lobes[(size_t)row * kGuideLobes + k] =
              make_float4(km.x, km.y, km.z, L[k].logw + vmfLogNorm(kap) - kap);
          accw += expf(L[k].logw);
          a.cdf[(size_t)row * kGuideLobes + k] = accw;
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
}

int smCount();

// Runs guideForwardTc over f.rows rows; throws if a completion wait timed out.
void runForwardTc(const ForwardArgs& f, cudaStream_t st) {
  int zero = 0;
  cudaCheck(cudaMemcpyToSymbolAsync(g_tcTimeout, &zero, sizeof zero, 0, cudaMemcpyHostToDevice, st),
            "tcgen05 flag");
  int tiles = (f.rows + tc::kRows - 1) / tc::kRows;
  guideForwardTc<<<std::min(tiles, smCount() * 4), tc::kCtaThreads, tc::kSmem, st>>>(f);
  cudaCheck(cudaGetLastError(), "guide forward (tcgen05)");
  int flag = 0;
  cudaCheck(cudaMemcpyFromSymbolAsync(&flag, g_tcTimeout, sizeof flag, 0, cudaMemcpyDeviceToHost, st),
            "tcgen05 flag");
  cudaCheck(cudaStreamSynchronize(st), "guide forward (tcgen05)");
  if (flag) throw std::runtime_error("guide forward: tensor-core completion wait timed out");
}

__global__ void guideAdamKernel(float* P, float* G, float* M, float* V, bf16* wb, float lr,
                                float c1, float c2) {
  const float b1 = 0.9f, b2 = 0.99f, eps = 1e-8f;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kNetParams) return;
  float g = G[i];
  G[i] = 0.0f;
  float m = b1 * M[i] + (1.0f - b1) * g;
  float v = b2 * V[i] + (1.0f - b2) * g * g;
  M[i] = m;
  V[i] = v;
  float p = P[i] - lr * (m * c1) / (sqrtf(v * c2) + eps);
  P[i] = p;
  if (i < kNetWeights) wb[i] = __float2bfloat16_rn(p);
}

__global__ void guideToBf16Kernel(const float* P, bf16* wb) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kNetWeights) wb[i] = __float2bfloat16_rn(P[i]);
}

__global__ void guideSumKernel(const float4* rec, const unsigned long long* count,
                               unsigned long long cap, float* sum) {
  unsigned long long n = *count;
  if (n > cap) n = cap;
  float s = 0.0f;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x)
    s += rec[3 * i].w;
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, off);
  if ((threadIdx.x & 31) == 0 && s != 0.0f) atomicAdd(sum, s);
}

int smCount() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 1;
}

void enableSmem() {
  static unsigned long long done = 0;  // one bit per device
  int dev = 0;
  cudaCheck(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 64 && (done >> dev & 1ull)) return;
  cudaCheck(cudaFuncSetAttribute(guideTrainKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kSmemTrain),
            "guide train smem");

  if (dev < 64) done |= 1ull << dev;
}

unsigned long long splitmix(unsigned long long& s) {
  unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

// ---- host: network state and schedule -----------------------------------------

void guideInitParams(unsigned long long seed, float* p) {
  unsigned long long s = seed * 0x2545F4914F6CDD1Dull + 1;
  auto gauss = [&]() {
    double u1 = ((splitmix(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    double u2 = ((splitmix(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    return (float)(std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
  };
  std::memset(p, 0, sizeof(float) * kNetParams);
  for (int i = kOffW0; i < kOffW1; i++) p[i] = gauss() * std::sqrt(2.0f / 35.0f);
  for (int i = kOffW1; i < kOffW3; i++) p[i] = gauss() * std::sqrt(2.0f / kNetHid);
  for (int i = kOffW3; i < kNetWeights; i++) p[i] = gauss() * 0.01f;
  // Output biases: lobes toward the 8 cube corners, kappa 2, equal weights.
  const float sInit = std::log(std::exp(2.0f - kKappaMin) - 1.0f);
  for (int k = 0; k < kGuideLobes; k++) {
    float d = 1.0f / std::sqrt(3.0f);
    p[kOffB3 + 5 * k] = (k & 1) ? d : -d;
    p[kOffB3 + 5 * k + 1] = (k & 2) ? d : -d;
    p[kOffB3 + 5 * k + 2] = (k & 4) ? d : -d;
    p[kOffB3 + 5 * k + 3] = sInit;
    p[kOffB3 + 5 * k + 4] = 0.0f;
  }
}

sundog_guiding_config guideDefaults() {
  sundog_guiding_config c;
  std::memset(&c, 0, sizeof c);
  c.train_spp = 32;
  c.pass_spp = 8;
  c.steps_per_pass = 64;
  c.batch = 16384;
  c.learning_rate = 5e-3f;
  c.mix = 0.7f;
  c.seed = 1;
  c.record_cap = 1ull << 22;
  return c;
}

void GuideState::configure(const sundog_guiding_config& c) {
  if (c.train_spp < 0 || c.pass_spp <= 0 || c.steps_per_pass < 0 || c.batch <= 0 ||
      !(c.learning_rate > 0.0f) || !(c.mix >= 0.0f && c.mix < 1.0f) || c.record_cap == 0)
    throw std::runtime_error("guiding: invalid configuration");
  cfg = c;
  params.alloc(kNetParams * sizeof(float));
  grads.alloc(kNetParams * sizeof(float));
  adamM.alloc(kNetParams * sizeof(float));
  adamV.alloc(kNetParams * sizeof(float));
  wbf.alloc(kNetWeights * sizeof(bf16));
  scal.alloc(4 * sizeof(float));
  counter.alloc(sizeof(unsigned long long));
  records.alloc((size_t)c.record_cap * kGuideRecordFloats * sizeof(float));
  lobes.alloc((size_t)kGuideCells * kGuideLobes * sizeof(float4));
  cdf.alloc((size_t)kGuideCells * kGuideLobes * sizeof(float));
  cudaCheck(cudaEventCreate(&e0), "event");
  cudaCheck(cudaEventCreate(&e1), "event");
  reset();
}

GuideState::~GuideState() {
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
}

void GuideState::reset() {
  std::vector<float> p(kNetParams);
  guideInitParams(cfg.seed, p.data());
  cudaCheck(cudaMemcpy(params.ptr, p.data(), p.size() * sizeof(float), cudaMemcpyHostToDevice),
            "guide params");
  cudaCheck(cudaMemset(grads.ptr, 0, grads.bytes), "guide reset");
  cudaCheck(cudaMemset(adamM.ptr, 0, adamM.bytes), "guide reset");
  cudaCheck(cudaMemset(adamV.ptr, 0, adamV.bytes), "guide reset");
  guideToBf16Kernel<<<(kNetWeights + 255) / 256, 256>>>((const float*)params.ptr, (bf16*)wbf.ptr);
  cudaCheck(cudaGetLastError(), "guide bf16");
  cudaCheck(cudaDeviceSynchronize(), "guide reset");
  trainedSpp = 0;
  adamStep = 0;
  haveBox = false;
  baked = false;
  std::memset(&stats, 0, sizeof stats);
}

int GuideState::kernelMode() const {
  int mode = baked ? kGuideSample : 0;
  if (training()) mode |= kGuideRecord;
  return mode;
}

void GuideState::beginPass(SdLaunch& lp, cudaStream_t st) {
  cudaCheck(cudaMemsetAsync(counter.ptr, 0, sizeof(unsigned long long), st), "guide counter");
  lp.guideTrain = (float4*)records.ptr;
  lp.guideTrainCount = (unsigned long long*)counter.ptr;
  lp.guideTrainCap = cfg.record_cap;
}

// Guide box: the 0.5th..99.5th percentile of the first pass's record
// positions per axis, padded by 2% of its extent.
void GuideState::computeBox(cudaStream_t st) {
  unsigned long long n = 0;
  cudaCheck(cudaMemcpyAsync(&n, counter.ptr, sizeof n, cudaMemcpyDeviceToHost, st), "guide count");
  cudaCheck(cudaStreamSynchronize(st), "guide count");
  n = std::min<unsigned long long>(n, cfg.record_cap);
  float3 lo = v3(-1.0f), hi = v3(1.0f);
  if (n > 0) {
    const unsigned long long want = 65536;
    unsigned long long stride = std::max<unsigned long long>(1, n / want);
    unsigned long long m = (n + stride - 1) / stride;
    std::vector<float4> xs(m);
    // One strided copy: the first float4 of every stride-th record.
    cudaCheck(cudaMemcpy2DAsync(xs.data(), sizeof(float4), records.ptr,
                                stride * 3 * sizeof(float4), sizeof(float4), m,
                                cudaMemcpyDeviceToHost, st),
              "guide sample");
    cudaCheck(cudaStreamSynchronize(st), "guide sample");
    std::vector<float> v(m);
    for (int axis = 0; axis < 3; axis++) {
      for (unsigned long long i = 0; i < m; i++) v[i] = comp(v3(xs[i].x, xs[i].y, xs[i].z), axis);
      size_t a = (size_t)(0.005 * (m - 1)), b = (size_t)(0.995 * (m - 1));
      std::nth_element(v.begin(), v.begin() + a, v.end());
      float va = v[a];
      std::nth_element(v.begin(), v.begin() + b, v.end());
      float vb = v[b];
      float pad = 0.02f * std::max(vb - va, 1e-3f);
      if (axis == 0) { lo.x = va - pad; hi.x = vb + pad; }
      if (axis == 1) { lo.y = va - pad; hi.y = vb + pad; }
      if (axis == 2) { lo.z = va - pad; hi.z = vb + pad; }
    }
  }
  boxLo = lo;
  boxHi = hi;
  haveBox = true;
}

void GuideState::trainAndBake(SdLaunch& lp, cudaStream_t st, int samplesInPass) {
  enableSmem();
  if (!haveBox) computeBox(st);
  float3 ext = boxHi - boxLo;
  float3 invExt = v3(1.0f / ext.x, 1.0f / ext.y, 1.0f / ext.z);
  cudaCheck(cudaEventRecord(e0, st), "event");
  cudaCheck(cudaMemsetAsync(scal.ptr, 0, scal.bytes, st), "guide scalars");
  float* sumF = (float*)scal.ptr;
  float* loss = (float*)scal.ptr + 1;
  guideSumKernel<<<smCount() * 4, 256, 0, st>>>((const float4*)records.ptr,
                                                (const unsigned long long*)counter.ptr,
                                                cfg.record_cap, sumF);
  cudaCheck(cudaGetLastError(), "guide sum");
  const int tiles = (cfg.batch + kTileRows - 1) / kTileRows;
  const int grid = std::min(tiles, smCount());
  for (int s = 0; s < cfg.steps_per_pass; s++) {
    TrainArgs a;
    a.wb = (const bf16*)wbf.ptr;
    a.params = (const float*)params.ptr;
    a.grads = (float*)grads.ptr;
    a.loss = loss;
    a.records = (const float4*)records.ptr;
    a.count = (const unsigned long long*)counter.ptr;
    a.cap = cfg.record_cap;
    a.sumF = sumF;
    a.batch = cfg.batch;
    a.sequential = 0;
    a.seed = cfg.seed * 0x9E3779B97F4A7C15ull + 17;
    a.step = adamStep;
    a.lo = boxLo;
    a.invExt = invExt;
    guideTrainKernel<<<grid, kThreads, kSmemTrain, st>>>(a);
    cudaCheck(cudaGetLastError(), "guide train");
    adamStep++;
    float c1 = 1.0f / (1.0f - std::pow(0.9f, (float)adamStep));
    float c2 = 1.0f / (1.0f - std::pow(0.99f, (float)adamStep));
    guideAdamKernel<<<(kNetParams + 255) / 256, 256, 0, st>>>(
        (float*)params.ptr, (float*)grads.ptr, (float*)adamM.ptr, (float*)adamV.ptr,
        (bf16*)wbf.ptr, cfg.learning_rate, c1, c2);
    cudaCheck(cudaGetLastError(), "guide adam");
  }
  cudaCheck(cudaEventRecord(e1, st), "event");
  bake(st);
  float lossSum = 0.0f;
  unsigned long long n = 0;
  cudaCheck(cudaMemcpyAsync(&lossSum, loss, sizeof lossSum, cudaMemcpyDeviceToHost, st), "loss");
  cudaCheck(cudaMemcpyAsync(&n, counter.ptr, sizeof n, cudaMemcpyDeviceToHost, st), "count");
  cudaCheck(cudaStreamSynchronize(st), "guide training");
  float tms = 0.0f;
  cudaCheck(cudaEventElapsedTime(&tms, e0, e1), "event time");
  stats.train_ms += tms;
  stats.train_steps += cfg.steps_per_pass;
  stats.passes++;
  stats.records = n;
  stats.last_loss = cfg.steps_per_pass > 0 ? lossSum / cfg.steps_per_pass : 0.0;
  stats.box_lo[0] = boxLo.x;
  stats.box_lo[1] = boxLo.y;
  stats.box_lo[2] = boxLo.z;
  stats.box_hi[0] = boxHi.x;
  stats.box_hi[1] = boxHi.y;
  stats.box_hi[2] = boxHi.z;
  trainedSpp += samplesInPass;
  lp.guideLobes = (const float4*)lobes.ptr;
  lp.guideCdf = (const float*)cdf.ptr;
  lp.guideLo = boxLo;
  lp.guideInvExtent = invExt;
  lp.guideMix = cfg.mix;
}

void GuideState::bake(cudaStream_t st) {
  enableSmem();
  cudaEvent_t b0 = nullptr, b1 = nullptr;
  cudaCheck(cudaEventCreate(&b0), "event");
  cudaCheck(cudaEventCreate(&b1), "event");
  cudaCheck(cudaEventRecord(b0, st), "event");
  ForwardArgs f;
  f.wb = (const bf16*)wbf.ptr;
  f.params = (const float*)params.ptr;
  f.rows = kGuideCells;
  f.queries = nullptr;
  f.outputs = nullptr;
  f.lobes = (float4*)lobes.ptr;
  f.cdf = (float*)cdf.ptr;
  runForwardTc(f, st);
  cudaCheck(cudaEventRecord(b1, st), "event");
  cudaCheck(cudaEventSynchronize(b1), "guide bake");
  float ms = 0.0f;
  cudaCheck(cudaEventElapsedTime(&ms, b0, b1), "event time");
  stats.bake_ms += ms;
  cudaEventDestroy(b0);
  cudaEventDestroy(b1);
  baked = true;
}

}  // namespace sdb

using namespace sdb;

namespace {

struct TmpNet {
  DevBuf params, wbf;
  explicit TmpNet(const float* p) {
    params.alloc(kNetParams * sizeof(float));
    cudaCheck(cudaMemcpy(params.ptr, p, kNetParams * sizeof(float), cudaMemcpyHostToDevice),
              "params");
    wbf.alloc(kNetWeights * sizeof(bf16));
    guideToBf16Kernel<<<(kNetWeights + 255) / 256, 256>>>((const float*)params.ptr, (bf16*)wbf.ptr);
    cudaCheck(cudaGetLastError(), "bf16");
  }
};

}  // namespace

extern "C" int sundog_guide_gradients(const float* params, const float* records, int n,
                                      const float* box, float* grads, float* loss) {
  SDB_TRY
  if (!params || !records || !box || !grads || n <= 0) throw std::runtime_error("guide: bad arguments");
  enableSmem();
  TmpNet net(params);
  DevBuf rec, g, scal, cnt;
  rec.upload(records, (size_t)n * kGuideRecordFloats * sizeof(float));
  g.alloc(kNetParams * sizeof(float));
  cudaCheck(cudaMemset(g.ptr, 0, g.bytes), "grads");
  scal.alloc(2 * sizeof(float));
  double sum = 0.0;
  for (int i = 0; i < n; i++) sum += records[(size_t)i * kGuideRecordFloats + 3];
  float h[2] = {(float)sum, 0.0f};
  cudaCheck(cudaMemcpy(scal.ptr, h, sizeof h, cudaMemcpyHostToDevice), "scalars");
  unsigned long long cn = (unsigned long long)n;
  cnt.upload(&cn, sizeof cn);
  TrainArgs a;
  a.wb = (const bf16*)net.wbf.ptr;
  a.params = (const float*)net.params.ptr;
  a.grads = (float*)g.ptr;
  a.loss = (float*)scal.ptr + 1;
  a.records = (const float4*)rec.ptr;
  a.count = (const unsigned long long*)cnt.ptr;
  a.cap = cn;
  a.sumF = (const float*)scal.ptr;
  a.batch = n;
  a.sequential = 1;
  a.seed = 0;
  a.step = 0;
  a.lo = v3(box[0], box[1], box[2]);
  a.invExt = v3(box[3], box[4], box[5]);
  int tiles = (n + kTileRows - 1) / kTileRows;
  guideTrainKernel<<<std::min(tiles, smCount()), kThreads, kSmemTrain>>>(a);
  cudaCheck(cudaGetLastError(), "guide train");
  cudaCheck(cudaDeviceSynchronize(), "guide train");
  cudaCheck(cudaMemcpy(grads, g.ptr, kNetParams * sizeof(float), cudaMemcpyDeviceToHost), "grads");
  if (loss) {
    cudaCheck(cudaMemcpy(h, scal.ptr, sizeof h, cudaMemcpyDeviceToHost), "loss");
    *loss = h[1];
  }
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_guide_outputs(const float* params, const float* queries, int n,
                                    float* outputs) {
  SDB_TRY
  if (!params || !queries || !outputs || n <= 0) throw std::runtime_error("guide: bad arguments");
  enableSmem();
  TmpNet net(params);
  DevBuf q, o;
  q.upload(queries, (size_t)n * 6 * sizeof(float));
  o.alloc((size_t)n * kNetLobeOut * sizeof(float));
  ForwardArgs f;
  f.wb = (const bf16*)net.wbf.ptr;
  f.params = (const float*)net.params.ptr;
  f.rows = n;
  f.queries = (const float*)q.ptr;
  f.outputs = (float*)o.ptr;
  f.lobes = nullptr;
  f.cdf = nullptr;
  runForwardTc(f, nullptr);
  cudaCheck(cudaMemcpy(outputs, o.ptr, o.bytes, cudaMemcpyDeviceToHost), "outputs");
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_session_guide_params(sundog_session* sh, float* params) {
  SDB_TRY
  if (!sh || !params) throw std::runtime_error("session: null argument");
  const RenderSession* s = reinterpret_cast<RenderSession*>(sh);
  if (!s->guide) throw std::runtime_error("session: guiding is not enabled");
  cudaCheck(cudaDeviceSynchronize(), "guide params");
  cudaCheck(cudaMemcpy(params, s->guide->params.ptr, kNetParams * sizeof(float),
                       cudaMemcpyDeviceToHost),
            "guide params");
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_session_guide_records(sundog_session* sh, float* out, uint64_t max_records,
                                            uint64_t* count) {
  SDB_TRY
  if (!sh) throw std::runtime_error("session: null handle");
  const RenderSession* s = reinterpret_cast<RenderSession*>(sh);
  if (!s->guide) throw std::runtime_error("session: guiding is not enabled");
  cudaCheck(cudaDeviceSynchronize(), "guide records");
  unsigned long long n = 0;
  cudaCheck(cudaMemcpy(&n, s->guide->counter.ptr, sizeof n, cudaMemcpyDeviceToHost), "count");
  n = std::min<unsigned long long>(n, s->guide->cfg.record_cap);
  if (count) *count = n;
  unsigned long long m = std::min<unsigned long long>(n, max_records);
  if (out && m)
    cudaCheck(cudaMemcpy(out, s->guide->records.ptr, m * kGuideRecordFloats * sizeof(float),
                         cudaMemcpyDeviceToHost),
              "records");
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_guide_init_params(uint64_t seed, float* params) {
  SDB_TRY
  if (!params) throw std::runtime_error("guide: null params");
  guideInitParams(seed, params);
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}
