// fkd_internal.h -- declarations shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fkd_common.cuh"

namespace fkd {

// Process-wide count of kernel launches issued by this library (telemetry for
// benchmarks: how many of the library's own kernels ran in a timed region).
void count_launches(uint64_t k);
uint64_t launches_total();

// Per-segment state of the global-level radix select (one per node of the
// level being split).
struct SegSel {
  unsigned long long prefix;  // the known top `bits` bits of the pivot key
  uint32_t bits;              // 0..64
  uint32_t krem;              // rank of the pivot among keys matching prefix
  uint32_t cnt;               // number of keys matching prefix
  uint32_t done;              // the pivot key is determined
  uint32_t tiles_done;        // CTAs of the current pass that finished
  uint32_t curL, curR, curE;  // partition cursors
  uint32_t pad;
};

struct BuildCtx {
  Geom g;
  CSoA input;     // the points to build from (device)
  SoA work[2];    // ping-pong working records
  SegSel* sel;    // >= 2^(d0-1) entries
  uint32_t* ghist;
  uint32_t* pending;  // one word per digit pass (+1): does that pass have work
  Table tab;
  uint32_t* err;
  cudaStream_t stream;
};

// Number of levels split by the global kernels (the first level whose
// intervals all fit the shared-memory subtree kernel).
uint32_t build_global_levels(uint32_t n, int dim);
size_t build_ghist_words(uint32_t n, int dim);
int sub_capacity(int dim);
cudaError_t launch_build(BuildCtx& bc, int dim);

// ------------------------------------------------------------------ search

struct Boxes {
  const float* lo;  // lo[c*stride + j]
  const float* hi;
  uint64_t stride;
  uint64_t q;
};

enum SearchMode { SEARCH_COUNT = 0, SEARCH_WRITE = 1, SEARCH_DIGEST = 2 };

struct SearchCtx {
  Geom g;
  Table tab;
  Boxes boxes;
  const uint32_t* order;   // optional processing order of the boxes (null: 0..q-1)
  uint32_t* counts;        // SEARCH_COUNT / SEARCH_DIGEST
  const uint64_t* offsets; // SEARCH_WRITE
  uint32_t* out;           // SEARCH_WRITE (heap indices when `heap_out`)
  uint64_t capacity;       // ids the output can hold
  unsigned long long* digests;  // SEARCH_DIGEST
  uint32_t* qcounter;      // work counter (zeroed by the launcher)
  uint32_t* err;
  int heap_out;            // write heap indices instead of ids
  cudaStream_t stream;
};

cudaError_t launch_search(SearchCtx& sc, int dim, int mode);
// Sorts every box's result slice by heap index and maps it to ids.
cudaError_t launch_order_results(const Geom& g, const Table& tab, const uint64_t* offsets, uint64_t q, uint32_t* out,
                                 uint32_t* tmp, uint32_t* err, cudaStream_t stream);
// Processing order of the boxes (see fkd_search.cu); scratch holds
// box_order_words(q) words; *order_out points into it.
size_t box_order_words(uint64_t q);
cudaError_t launch_box_order(const Geom& g, const Table& tab, const Boxes& b, int dim, uint32_t* scratch,
                             uint32_t** order_out, cudaStream_t stream);
// Exclusive prefix sum of q uint32 counts into q+1 uint64 offsets.
cudaError_t launch_scan_counts(const uint32_t* counts, uint64_t q, uint64_t* offsets, unsigned long long* partials,
                               cudaStream_t stream);
size_t scan_partials_words(uint64_t q);

}  // namespace fkd
