// Host side of learned path guiding: the network's device state and the
// training schedule a guided render follows (guide.cu).
//
// A guided render traces its first train_spp samples in passes of pass_spp
// samples. Every pass records training samples; after it the network takes
// steps_per_pass Adam steps on them and the mixture table is re-baked, and
// the next pass samples by MIS with the updated guide. The remaining samples
// use the final guide without recording. Every sample of every pass goes to
// the film: each is an unbiased estimate whatever the guide is.
#pragma once

#include <cuda_runtime.h>

#include "../../include/sundog_api.h"
#include "guide_net.h"
#include "render_session.h"
#include "sd_types.h"

namespace sdb {

sundog_guiding_config guideDefaults();
void guideInitParams(unsigned long long seed, float* params);

struct GuideState {
  sundog_guiding_config cfg{};
  DevBuf params, grads, adamM, adamV, wbf, scal, counter, records, lobes, cdf;
  float3 boxLo{}, boxHi{};
  bool haveBox = false;
  bool baked = false;
  int trainedSpp = 0;
  int adamStep = 0;
  sundog_guiding_stats stats{};
  cudaEvent_t e0 = nullptr, e1 = nullptr;

  GuideState() = default;
  GuideState(const GuideState&) = delete;
  GuideState& operator=(const GuideState&) = delete;
  ~GuideState();

  void configure(const sundog_guiding_config& c);
  void reset();  // fresh network, untrained
  bool training() const { return trainedSpp < cfg.train_spp; }
  // Kernel variant for the next launch (kGuideSample / kGuideRecord bits).
  int kernelMode() const;
  void beginPass(SdLaunch& lp, cudaStream_t st);
  void trainAndBake(SdLaunch& lp, cudaStream_t st, int samplesInPass);
  void bake(cudaStream_t st);

 private:
  void computeBox(cudaStream_t st);
};

}  // namespace sdb
