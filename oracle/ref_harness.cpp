// ref_harness.cpp -- C entry points over the UNMODIFIED reference CPU tree.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file against the
// reference's own headers (FKDTree_cpu.h, FKDTree.h, FKDPoint.h, FQueue.h,
// found through -I on the reference checkout) into oracle/_ref/libfkdref.so.
// Nothing of the reference is copied here: this file only constructs
// FKDTree_CPU<float, D>, calls its public methods and moves data in and out.
// It serves two purposes:
//   * pinning the C restatement (fkd_oracle.c) and generating the golden
//     fixtures under tests/golden/ (tests/golden/make_golden.py);
//   * the CPU baseline timed by bench.py: the reference build (serial by
//     design, FKDTree_cpu.h:221-277) and its searches under an OpenMP
//     parallel-for over boxes, the reference driver's `-p <threads>` loop
//     (main.cpp:369-381) with OpenMP standing in for TBB as in test.cpp:71-76;
//   * the reference's other CPU tree, the "vanilla" CMSSW KDTreeLinkerAlgo
//     (KDTreeLinkerAlgoT.h), built and searched the way main.cpp:558-612
//     does it (serially: its search keeps the result list in a member), as an
//     extra baseline column.
//
// It is compiled WITHOUT -DNDEBUG, so a FQueue overflow (FQueue.h:158) aborts
// loudly rather than corrupting results; callers only run the level-order,
// BFS and branchless variants on boxes whose frontier the C restatement has
// shown to fit in FQueue's 1024 slots.
#include <omp.h>
#include <stdint.h>

#include <chrono>
#include <cstring>
#include <memory>
#include <vector>

#include "FKDTree_cpu.h"
#include "KDTreeLinkerAlgoT.h"

namespace {

struct HandleBase {
  virtual ~HandleBase() {}
  virtual int dim() const = 0;
  virtual uint32_t size() const = 0;
  virtual double build() = 0;
  virtual void tables(float* tab_soa, uint32_t* ids) = 0;
  virtual void search(int variant, uint64_t nq, const float* mins, const float* maxs, uint32_t* counts,
                      const uint64_t* offsets, uint32_t* out, int threads, double* seconds) = 0;
  // search_in_the_box_recursive of boxes [j0, j1) (bounds SoA with row
  // stride `stride`): count and digest of its ids, serially
  virtual void digest(uint64_t j0, uint64_t j1, uint64_t stride, const float* mins, const float* maxs,
                      uint32_t* counts, uint64_t* digests) = 0;
};

inline uint64_t mix_id(uint32_t id) {
  uint64_t z = (uint64_t)id + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

template <int D>
struct Handle : HandleBase {
  std::vector<FKDPoint<float, D>> pts;
  std::unique_ptr<FKDTree_CPU<float, D>> tree;

  Handle(uint32_t n, const float* coords_soa, const uint32_t* ids) : pts(n) {
    for (uint32_t i = 0; i < n; ++i) {
      for (int c = 0; c < D; ++c) pts[i].setDimension(c, coords_soa[(size_t)c * n + i]);
      pts[i].setId(ids[i]);
    }
  }
  int dim() const override { return D; }
  uint32_t size() const override { return (uint32_t)pts.size(); }

  // Construction + build, the span main.cpp:201-207 times.
  double build() override {
    auto t0 = std::chrono::steady_clock::now();
    tree.reset(new FKDTree_CPU<float, D>(pts));
    tree->build();
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
  }

  void tables(float* tab_soa, uint32_t* ids) override {
    const size_t n = pts.size();
    for (int c = 0; c < D; ++c) {
      const std::vector<float>& v = tree->getDimensionVector(c);
      std::memcpy(tab_soa + (size_t)c * n, v.data(), n * sizeof(float));
    }
    const std::vector<unsigned int>& id = tree->getIdVector();
    std::memcpy(ids, id.data(), n * sizeof(uint32_t));
  }

  std::vector<unsigned int> one(int variant, const FKDPoint<float, D>& lo, const FKDPoint<float, D>& hi) {
    switch (variant) {
      case 0: return tree->search_in_the_box(lo, hi);
      case 1: return tree->search_in_the_box_BFS(lo, hi);
      case 2: return tree->search_in_the_box_branchless(lo, hi);
      default: {
        std::vector<unsigned int> r;
        tree->search_in_the_box_recursive(lo, hi, r);
        return r;
      }
    }
  }

  void digest(uint64_t j0, uint64_t j1, uint64_t stride, const float* mins, const float* maxs, uint32_t* counts,
              uint64_t* digests) override {
    FKDPoint<float, D> lo, hi;
    for (uint64_t j = j0; j < j1; ++j) {
      for (int c = 0; c < D; ++c) {
        lo.setDimension(c, mins[(size_t)c * stride + j]);
        hi.setDimension(c, maxs[(size_t)c * stride + j]);
      }
      std::vector<unsigned int> r;
      tree->search_in_the_box_recursive(lo, hi, r);
      uint64_t dg = 0;
      for (unsigned int id : r) dg += mix_id(id);
      counts[j] = (uint32_t)r.size();
      digests[j] = dg;
    }
  }

  void search(int variant, uint64_t nq, const float* mins, const float* maxs, uint32_t* counts,
              const uint64_t* offsets, uint32_t* out, int threads, double* seconds) override {
    std::vector<FKDPoint<float, D>> lo(nq), hi(nq);
    for (uint64_t j = 0; j < nq; ++j)
      for (int c = 0; c < D; ++c) {
        lo[j].setDimension(c, mins[(size_t)c * nq + j]);
        hi[j].setDimension(c, maxs[(size_t)c * nq + j]);
      }
    if (threads > 0) omp_set_num_threads(threads);
    auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t j = 0; j < (int64_t)nq; ++j) {
      std::vector<unsigned int> r = one(variant, lo[j], hi[j]);
      if (counts) counts[j] = (uint32_t)r.size();
      if (offsets && out && !r.empty()) std::memcpy(out + offsets[j], r.data(), r.size() * sizeof(uint32_t));
    }
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  }
};

}  // namespace

extern "C" {

// Creates a reference tree over n points (coords_soa[c*n + i], ids[i]).
void* fkdref_create(int dim, uint32_t n, const float* coords_soa, const uint32_t* ids) {
  switch (dim) {
    case 1: return new Handle<1>(n, coords_soa, ids);
    case 2: return new Handle<2>(n, coords_soa, ids);
    case 3: return new Handle<3>(n, coords_soa, ids);
    case 4: return new Handle<4>(n, coords_soa, ids);
    default: return nullptr;
  }
}

void fkdref_destroy(void* h) { delete static_cast<HandleBase*>(h); }

// FKDTree_CPU ctor + build(); returns the elapsed seconds (n must be > 0:
// the reference build writes theIntervalMin[0] even for an empty input).
double fkdref_build(void* h) { return static_cast<HandleBase*>(h)->build(); }

// getDimensionVector(c) for every c, then getIdVector().
void fkdref_tables(void* h, float* tab_soa, uint32_t* ids) { static_cast<HandleBase*>(h)->tables(tab_soa, ids); }

// variant: 0 search_in_the_box, 1 _BFS, 2 _branchless, 3 _recursive.
// counts may be null; ids are written to out[offsets[j]...] when both given.
void fkdref_search(void* h, int variant, uint64_t nq, const float* mins_soa, const float* maxs_soa,
                   uint32_t* counts, const uint64_t* offsets, uint32_t* out, int threads, double* seconds) {
  static_cast<HandleBase*>(h)->search(variant, nq, mins_soa, maxs_soa, counts, offsets, out, threads, seconds);
}

int fkdref_max_threads(void) { return omp_get_max_threads(); }

// search_in_the_box_recursive of every box under an OpenMP parallel-for over
// boxes (main.cpp:351-359's loop), reducing each box's id list to its count
// and digest (the one fkdref_batch reports).  Returns the elapsed seconds.
double fkdref_search_digest(void* h, uint64_t nq, const float* mins_soa, const float* maxs_soa, uint32_t* counts,
                            uint64_t* digests, int threads) {
  HandleBase* b = static_cast<HandleBase*>(h);
  if (threads > 0) omp_set_num_threads(threads);
  const int64_t chunk = 64;
  auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t j = 0; j < (int64_t)nq; j += chunk) {
    const uint64_t j1 = (uint64_t)j + chunk < nq ? (uint64_t)j + chunk : nq;
    b->digest((uint64_t)j, j1, nq, mins_soa, maxs_soa, counts, digests);
  }
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

// Batched events, the reference way (OpenMP over events; each event a serial
// FKDTree_CPU build and a serial search_in_the_box_recursive of its boxes):
// per box the result count and the digest (wrap-around sum over the result
// ids of the splitmix64 finaliser of id + 0x9E3779B97F4A7C15, the digest the
// GPU library reports).  Event e owns points [pt_off[e], pt_off[e+1]) with
// coordinates SoA at coords[coord_off[e] + c*n + i] and boxes [q_off[e],
// q_off[e+1]) with bounds SoA at mins/maxs[qcoord_off[e] + c*q + j].
// Returns the elapsed seconds.
double fkdref_batch(uint32_t nev, const uint32_t* dims, const uint64_t* pt_off, const uint64_t* coord_off,
                    const float* coords, const uint32_t* ids, const uint64_t* q_off, const uint64_t* qcoord_off,
                    const float* mins, const float* maxs, uint32_t* counts, uint64_t* digests, int threads) {
  if (threads > 0) omp_set_num_threads(threads);
  auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t e = 0; e < (int64_t)nev; ++e) {
    const uint32_t n = (uint32_t)(pt_off[e + 1] - pt_off[e]);
    const uint64_t q = q_off[e + 1] - q_off[e];
    if (n == 0) {
      for (uint64_t j = 0; j < q; ++j) {
        counts[q_off[e] + j] = 0;
        digests[q_off[e] + j] = 0;
      }
      continue;
    }
    std::unique_ptr<HandleBase> h;
    switch (dims[e]) {
      case 1: h.reset(new Handle<1>(n, coords + coord_off[e], ids + pt_off[e])); break;
      case 2: h.reset(new Handle<2>(n, coords + coord_off[e], ids + pt_off[e])); break;
      case 3: h.reset(new Handle<3>(n, coords + coord_off[e], ids + pt_off[e])); break;
      default: h.reset(new Handle<4>(n, coords + coord_off[e], ids + pt_off[e])); break;
    }
    h->build();
    h->digest(0, q, q, mins + qcoord_off[e], maxs + qcoord_off[e], counts + q_off[e], digests + q_off[e]);
  }
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

// The vanilla CMSSW tree over n 3D points (coords_soa[c*n + i], data = i),
// region = the points' bounding box, as main.cpp:558-590 builds it; then one
// serial search per box (main.cpp:596-605).  counts[j] receives the number of
// points found for box j.  Returns the build seconds (filling the node list
// included, as main.cpp times it); *search_seconds the search loop.
double fkdref_cmssw(uint32_t n, const float* coords_soa, uint64_t nq, const float* mins, const float* maxs,
                    uint32_t* counts, double* search_seconds) {
  auto t0 = std::chrono::steady_clock::now();
  KDTreeLinkerAlgo<unsigned, 3> tree;
  std::vector<KDTreeNodeInfoT<unsigned, 3>> nodes;
  nodes.reserve(n);
  float lo[3] = {0.f, 0.f, 0.f}, hi[3] = {0.f, 0.f, 0.f};
  for (uint32_t i = 0; i < n; ++i) {
    const float x = coords_soa[i], y = coords_soa[(size_t)n + i], z = coords_soa[2 * (size_t)n + i];
    nodes.emplace_back(i, x, y, z);
    const float p[3] = {x, y, z};
    for (int c = 0; c < 3; ++c) {
      if (i == 0 || p[c] < lo[c]) lo[c] = p[c];
      if (i == 0 || p[c] > hi[c]) hi[c] = p[c];
    }
  }
  KDTreeCube bounds(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]);
  tree.build(nodes, bounds);
  auto t1 = std::chrono::steady_clock::now();
  std::vector<KDTreeNodeInfoT<unsigned, 3>> found;
  for (uint64_t j = 0; j < nq; ++j) {
    KDTreeCube box(mins[j], maxs[j], mins[nq + j], maxs[nq + j], mins[2 * nq + j], maxs[2 * nq + j]);
    tree.search(box, found);
    counts[j] = (uint32_t)found.size();
    found.clear();
  }
  auto t2 = std::chrono::steady_clock::now();
  *search_seconds = std::chrono::duration<double>(t2 - t1).count();
  return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
