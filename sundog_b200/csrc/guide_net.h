// Guiding network shape and parameter layout, shared by host and device.
//
//   input  48 = 30 frequency features of the position (sin, cos of
//               2^j pi p_i, j = 0..4, i = x, y, z; p normalised to the guide
//               box) + 2 zero + the normal (3) + 13 zero
//   hidden 3 x 64, ReLU
//   output 48 = 8 lobes x (r.xyz, s, z) + 8 unused:
//               mu = r / |r|, kappa = softplus(s) + kKappaMin (at most
//               kKappaMax), weight = softmax(z)
//
// Parameters live in one FP32 array: the weight matrices row-major
// [out][in] (W0 64x48, W1 64x64, W2 64x64, W3 48x64), then the biases. The
// kernels read the weights as BF16 copies and the biases in FP32.
#pragma once

namespace sdb {

constexpr int kNetIn = 48;
constexpr int kNetHid = 64;
constexpr int kNetOut = 48;
constexpr int kNetLobeOut = 40;  // used outputs
constexpr int kNetFreqs = 5;
constexpr float kKappaMin = 0.05f;
constexpr float kKappaMax = 500.0f;

constexpr int kOffW0 = 0;
constexpr int kOffW1 = kOffW0 + kNetHid * kNetIn;
constexpr int kOffW2 = kOffW1 + kNetHid * kNetHid;
constexpr int kOffW3 = kOffW2 + kNetHid * kNetHid;
constexpr int kNetWeights = kOffW3 + kNetOut * kNetHid;  // 14336
constexpr int kOffB0 = kNetWeights;
constexpr int kOffB1 = kOffB0 + kNetHid;
constexpr int kOffB2 = kOffB1 + kNetHid;
constexpr int kOffB3 = kOffB2 + kNetHid;
constexpr int kNetParams = kOffB3 + kNetOut;  // 14576

// A training record: 3 float4 = (x, F / pdf), (n, 0), (wi, 0).
constexpr int kGuideRecordFloats = 12;

// Mixture table: a 32^3 grid over the guide box times 6 normal directions
// (+x, -x, +y, -y, +z, -z), 8 lobes per entry.
constexpr int kGuideLobes = 8;
constexpr int kGuideGrid = 32;
constexpr int kGuideNormals = 6;
constexpr int kGuideCells = kGuideGrid * kGuideGrid * kGuideGrid * kGuideNormals;

// Path-kernel variants: bit 0 samples by MIS with the guide, bit 1 records
// training samples.
constexpr int kGuideSample = 1;
constexpr int kGuideRecord = 2;

}  // namespace sdb
