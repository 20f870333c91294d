// Learned path guiding hooks used by the path kernel. The plain kernel
// (SdLaunch::guiding == 0) never calls into this header.
#pragma once

#include "sd_bsdf.cuh"
#include "sd_types.h"

namespace sdb {

__device__ __forceinline__ bool guideEligible(const SdMaterial& m) {
  return !isDeltaMaterial(m) && m.kind != MT_EMISSIVE;
}

__device__ __forceinline__ float guideMixPdf(const SdLaunch&, float3, float3, float3, float pdfB,
                                             const SdMaterial&) {
  return pdfB;
}

__device__ __forceinline__ BsdfDraw guidedDraw(const SdLaunch&, const SdMaterial& m, float3 albedo,
                                               float3 d, float3 ns, bool front, float etaExt,
                                               float, float3, Pcg& rng) {
  return bsdfDraw(m, albedo, d, ns, front, etaExt, rng);
}

__device__ __forceinline__ void guideRecord(const SdLaunch&, int, float3, float3, float3, float3,
                                            float3) {}

}  // namespace sdb
