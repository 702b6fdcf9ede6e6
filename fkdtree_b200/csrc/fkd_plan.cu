// fkd_plan.cu -- host-side planning of a (batched) build.
//
// A build is a set of independent events (one tree each).  Because every
// interval of a complete heap tree is a closed-form function of (n, depth,
// index-in-level), the whole work decomposition is known from the event sizes
// alone: for each global level the (event, segment) pairs that level splits,
// the CTA -> (segment, tile) maps of the digit-pass and partition kernels, and
// the (event, subtree) roots of the shared-memory subtree kernel.  The plan is
// built once per set of sizes, uploaded in one copy, and reused by every
// build (and every CUDA-graph replay) with those sizes.
#include <algorithm>

#include "fkd_plan.h"

namespace fkd {

void plan_build(const uint32_t* n_ev, const uint32_t* base_ev, uint32_t nev, int dim, uint32_t hist_ctas,
                PlanHost& out, int subn) {
  out.evs.assign(nev, EvDesc{});
  out.levels.clear();
  out.subs.clear();
  out.maxseg = 1;
  uint32_t maxd0 = 0;
  for (uint32_t e = 0; e < nev; ++e) {
    EvDesc& d = out.evs[e];
    d.g = make_geom(n_ev[e]);
    d.base = base_ev[e];
    d.d0 = build_global_levels(n_ev[e], dim, subn);
    if (n_ev[e] && d.d0 > maxd0) maxd0 = d.d0;
  }
  out.levels.resize(maxd0);
  // first[L][e]: index of event e's first segment in level L's list
  std::vector<std::vector<uint32_t>> first(maxd0 + 1, std::vector<uint32_t>(nev, ~0u));
  for (uint32_t L = 0; L < maxd0; ++L) {
    uint32_t k = 0;
    for (uint32_t e = 0; e < nev; ++e) {
      const EvDesc& d = out.evs[e];
      if (d.g.n == 0 || d.d0 <= L) continue;
      first[L][e] = k;
      k += 1u << L;
    }
  }
  for (uint32_t L = 0; L < maxd0; ++L) {
    PlanLevel& lv = out.levels[L];
    uint64_t total = 0;
    for (uint32_t e = 0; e < nev; ++e) {
      const EvDesc& d = out.evs[e];
      if (d.g.n == 0 || d.d0 <= L) continue;
      for (uint32_t t = 0; t < (1u << L); ++t) {
        lv.segs.push_back(make_uint2(e, t));
        lv.child.push_back(d.d0 > L + 1 ? first[L + 1][e] + 2u * t : ~0u);
        total += seg_len(d.g, L, t);
        lv.maxlen = std::max<uint32_t>(lv.maxlen, seg_len(d.g, L, t));
      }
    }
    out.maxseg = std::max<uint32_t>(out.maxseg, (uint32_t)lv.segs.size());
    // digit passes: about hist_ctas CTAs for the level, tiles a multiple of HIST_STEP
    const uint64_t want = (total + hist_ctas - 1) / std::max<uint32_t>(hist_ctas, 1u);
    lv.hts = (uint32_t)std::max<uint64_t>(HIST_STEP, ((want + HIST_STEP - 1) / HIST_STEP) * HIST_STEP);
    for (uint32_t s = 0; s < lv.segs.size(); ++s) {
      const EvDesc& d = out.evs[lv.segs[s].x];
      const uint32_t len = seg_len(d.g, L, lv.segs[s].y);
      const uint32_t nh = (len + lv.hts - 1) / lv.hts;
      for (uint32_t t = 0; t < nh; ++t) lv.htiles.push_back(make_uint2(s, t));
      const uint32_t np = (len + PART_TILE - 1) / PART_TILE;
      for (uint32_t t = 0; t < np; ++t) lv.ptiles.push_back(make_uint2(s, t));
    }
  }
  for (uint32_t e = 0; e < nev; ++e) {
    const EvDesc& d = out.evs[e];
    if (d.g.n == 0) continue;
    for (uint32_t s = 0; s < (1u << d.d0); ++s) out.subs.push_back(make_uint2(e, s));
  }
}

// Forgets the uploaded plan: after a failed upload nothing may point into a
// freed or half-written device copy.
void PlanDev::clear() {
  evs = nullptr;
  nev = 0;
  subs = nullptr;
  nsub = 0;
  levels.clear();
  maxseg = 1;
}

cudaError_t PlanDev::upload(const PlanHost& h, cudaStream_t stream) {
  clear();
  // every array starts on a 16-byte boundary (uint2 / EvDesc loads need 8)
  size_t words = h.evs.size() * (sizeof(EvDesc) / 4) + 2 * h.subs.size() + 8;
  for (const PlanLevel& lv : h.levels)
    words += 2 * (lv.segs.size() + lv.htiles.size() + lv.ptiles.size()) + lv.child.size() + 16;
  host.assign(words + 16, 0u);
  size_t pos = 0;
  auto put = [&](const void* src, size_t bytes) {
    const size_t at = pos;
    if (bytes) memcpy(host.data() + pos, src, bytes);
    pos += ((bytes + 15) / 16) * 4;
    return at;
  };
  const size_t evs_at = put(h.evs.data(), h.evs.size() * sizeof(EvDesc));
  const size_t subs_at = put(h.subs.data(), h.subs.size() * sizeof(uint2));
  std::vector<size_t> at(h.levels.size() * 4);
  for (size_t L = 0; L < h.levels.size(); ++L) {
    at[4 * L] = put(h.levels[L].segs.data(), h.levels[L].segs.size() * sizeof(uint2));
    at[4 * L + 1] = put(h.levels[L].htiles.data(), h.levels[L].htiles.size() * sizeof(uint2));
    at[4 * L + 2] = put(h.levels[L].ptiles.data(), h.levels[L].ptiles.size() * sizeof(uint2));
    at[4 * L + 3] = put(h.levels[L].child.data(), h.levels[L].child.size() * sizeof(uint32_t));
  }
  const size_t bytes = pos * 4 + 16;
  if (bytes > cap) {
    if (dev) cudaFree(dev);
    dev = nullptr;
    cap = 0;
    cudaError_t e = device_alloc(&dev, bytes);
    if (e != cudaSuccess) return e;
    cap = bytes;
  }
  cudaError_t e = cudaMemcpyAsync(dev, host.data(), pos * 4, cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) return e;
  uint32_t* d = (uint32_t*)dev;
  evs = (const EvDesc*)(d + evs_at);
  nev = (uint32_t)h.evs.size();
  subs = (const uint2*)(d + subs_at);
  nsub = (uint32_t)h.subs.size();
  levels.resize(h.levels.size());
  for (size_t L = 0; L < h.levels.size(); ++L) {
    LevelPlan& lp = levels[L];
    lp.segs = (const uint2*)(d + at[4 * L]);
    lp.nseg = (uint32_t)h.levels[L].segs.size();
    lp.htiles = (const uint2*)(d + at[4 * L + 1]);
    lp.nhtile = (uint32_t)h.levels[L].htiles.size();
    lp.hts = h.levels[L].hts;
    lp.ptiles = (const uint2*)(d + at[4 * L + 2]);
    lp.nptile = (uint32_t)h.levels[L].ptiles.size();
    lp.child = (const uint32_t*)(d + at[4 * L + 3]);
    lp.maxlen = h.levels[L].maxlen;
  }
  maxseg = h.maxseg;
  return cudaSuccess;
}

PlanDev::~PlanDev() {
  if (dev) cudaFree(dev);
}

}  // namespace fkd
