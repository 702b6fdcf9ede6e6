// fkd_plan.h -- host-side planning of a (batched) build (see fkd_plan.cu).
#pragma once
#include <string.h>

#include <vector>

#include "fkd_internal.h"

namespace fkd {

struct PlanLevel {
  std::vector<uint2> segs, htiles, ptiles;
  std::vector<uint32_t> child;  // per segment: index of its left child in the next level's list (~0u: none)
  uint32_t hts = HIST_STEP;
  uint32_t maxlen = 0;  // longest segment of the level
};

struct PlanHost {
  std::vector<EvDesc> evs;
  std::vector<PlanLevel> levels;
  std::vector<uint2> subs;
  uint32_t maxseg = 1;
};

// The device copy of a plan (one allocation) and the host-side LevelPlan
// array pointing into it.
struct PlanDev {
  void* dev = nullptr;
  size_t cap = 0;
  std::vector<uint32_t> host;
  const EvDesc* evs = nullptr;
  uint32_t nev = 0;
  const uint2* subs = nullptr;
  uint32_t nsub = 0;
  std::vector<LevelPlan> levels;
  uint32_t maxseg = 1;
  // On failure the plan is left empty (clear()); the caller must re-upload.
  cudaError_t upload(const PlanHost& h, cudaStream_t stream);
  void clear();
  ~PlanDev();
};

// Plans the build of nev events of n_ev[e] points whose records start at
// base_ev[e] of the concatenated arrays; hist_ctas is the number of
// digit-pass CTAs to aim for per level.
void plan_build(const uint32_t* n_ev, const uint32_t* base_ev, uint32_t nev, int dim, uint32_t hist_ctas,
                PlanHost& out, int subn = 0);

}  // namespace fkd
