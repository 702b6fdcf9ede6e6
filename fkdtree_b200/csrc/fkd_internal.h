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
// cudaMalloc with the allocation-failure injection of fkd_debug_fail_alloc
cudaError_t device_alloc(void** p, size_t bytes);

// Per-segment state of the global-level select (one per node of the level
// being split).  The digit passes (k_hist) narrow an interval [klo, khi] of
// 64-bit order keys (mono(coordinate) << 32 | id) that holds the pivot: the
// candidates are the segment's points whose key lies in it, krem the pivot's
// rank among them and cnt their number.  While the interval spans several
// coordinate values its id part is the full range and a pass bins the value
// (linearly in the float value for the first pass of a segment whose value
// range is known, `lin`; else the key bits); once the value is fixed a pass
// bins the id.  The select is done when one candidate is left, when the
// interval is one key (repeated keys), or when at most SMALL_CAP candidates
// are left (`small`): the partition then parks them and k_small_fix orders
// them by key.  k_select_small and the learned bracket also keep the prefix
// form (prefix / bits) of the levels they serve.
struct SegSel {
  unsigned long long prefix;  // k_select_small: the known top `bits` bits of the pivot key
  uint32_t bits;              // 0..64
  uint32_t krem;              // rank of the pivot among the candidates
  uint32_t cnt;               // number of candidates
  uint32_t done;              // the pivot is determined (or `small`)
  uint32_t tiles_done;        // CTAs of the current pass that finished
  uint32_t curL, curR, curE;  // partition cursors
  uint32_t verify;            // 1: [klo, khi] is a predicted block, the next pass verifies it
  uint32_t below;             // verify pass: points whose key lies below the block
  uint32_t kfull;             // the pivot rank within the segment (fallback restart)
  uint32_t bits0;             // the common prefix every key of the segment shares
  unsigned long long prefix0;
  uint32_t small;             // done with cnt <= SMALL_CAP candidates: the partition parks them
  uint32_t lin;               // the next pass bins the value linearly: bin = floor((v - vmin) * scale)
  unsigned long long klo, khi;    // the candidate key interval
  unsigned long long klo0, khi0;  // the segment's own interval (fallback restart)
  float vmin, scale;              // linear binning of the next pass
  float vmin0, scale0;            // ... of the segment's own range (restart)
  uint32_t lin0;
  uint32_t cmin, cmax;            // the pass's smallest / largest candidate value key (id once the
                                  // value is fixed): the next interval is clipped to them
};
// Candidates a select may leave for the partition to order itself (one warp
// sorts them); more are narrowed by further digit passes.
constexpr uint32_t SMALL_CAP = 32;

constexpr int FKD_MLP_FEATURES = 40;  // node summary width (== FKD_MLP_IN of the C ABI)

// Learned-split state of a build (all null / zero for the plain build).
struct LearnCtx {
  const float* params;  // MLP parameters (null: plain radix select)
  float delta;          // bracket half-width, in units of the sample range
  float* feat;          // >= maxseg * 40 features
  float* yhat;          // >= maxseg predictions
  float2* range;        // >= maxseg sample ranges (min, max) along the split dimension
  unsigned long long* stats;  // [0] brackets tried, [1] verified, [2] fell back
  // recording mode (training data): targets of every global segment
  float* rec_x;         // features of recorded segments (rows of 40)
  float* rec_t;         // their targets
  unsigned long long* rec_n;  // running count
  uint64_t rec_cap;
};

// One event (one independent tree) of a build: its geometry, the position of
// its first point in the concatenated working arrays / node tables, the number
// of levels the global kernels split (d0), and where its boxes are.
struct EvDesc {
  Geom g;
  uint32_t base;     // first point / node of the event
  uint32_t d0;       // global levels of this event
  uint32_t nq;       // boxes of the event
  uint64_t qbase;    // index of the event's first box in the launch's box space
  uint64_t qcbase;   // offset of the event's box coordinates (SoA slice: [c*nq + j])
  uint64_t qout;     // index of the event's first box in the caller's output arrays
};

// Device-side plan of a (batched) build: per global level the list of
// (event, segment) pairs and the CTA -> (segment, tile) maps of the digit and
// partition kernels; the list of (event, subtree) roots of the subtree kernel.
struct LevelPlan {
  const uint2* segs;    // (event, index-in-level)
  uint32_t nseg;
  const uint2* htiles;  // digit-pass CTA -> (segment, tile)
  uint32_t nhtile;
  uint32_t hts;         // digit-pass tile length
  const uint2* ptiles;  // partition CTA -> (segment, tile)
  uint32_t nptile;
  const uint32_t* child;  // per segment: its left child's index in the next level (~0u: not a global segment)
  uint32_t maxlen;        // longest segment of the level
};

struct BuildCtx {
  const EvDesc* evs;
  uint32_t nlevels;
  const LevelPlan* levels;  // host array of nlevels
  const uint2* subs;        // (event, subtree index at the event's d0)
  uint32_t nsub;
  CSoA input;     // the points to build from (device, SoA with stride = total points)
  SoA work[2];    // ping-pong working records
  SegSel* sel;    // >= max segments of a level
  uint32_t* ghist;
  uint32_t* pending;  // one word per digit pass (+1): does that pass have work
  uint32_t* tiebuf = nullptr;  // >= max segments * SMALL_CAP * (dim + 1) words: the candidates a select
                               // leaves to the partition (null: every select narrows to one key)
  uint2* bnd = nullptr;    // 2 x bnd_stride: per-segment (min, max) of the split coordinate's
                           // order bits, written by the previous level's partition (null: unused)
  uint32_t bnd_stride = 0; // >= max segments of a level
  Table tab;
  uint32_t* err;
  cudaStream_t stream;
  LearnCtx learn;
  cudaEvent_t ev_sub = nullptr;  // optional: recorded right before the subtree kernel
  int subtree = 0;               // shared-memory subtree kernel: 0 auto, 1 radix select, 2 presorted lists
  bool small_select = true;      // levels of small segments select with one CTA per segment
  bool lin = true;               // a segment's first digit pass bins its value range linearly
  int subn = 0;                  // presorted subtree size the plan was made for (0: 1,024)
};

// Number of levels split by the global kernels (the first level whose
// intervals all fit the shared-memory subtree kernel).
// subn: the presorted-list kernel's subtree size (512 or 1,024; 0 = 1,024).
uint32_t build_global_levels(uint32_t n, int dim, int subn = 0);
int sub_capacity(int dim);
int sorted_sub_capacity(int subn = 0);  // largest subtree of the presorted-list kernel (dims 1-3)
constexpr uint32_t HIST_BINS = 2048;  // global digit histogram per segment
#ifndef FKD_PART_PIPT
#define FKD_PART_PIPT 4
#endif
constexpr uint32_t PART_TILE = 256 * FKD_PART_PIPT;  // records per partition CTA
constexpr uint32_t HIST_STEP = 2048;  // digit-pass tile granularity
cudaError_t launch_build(BuildCtx& bc, int dim);
// fkd_subtree_sort.cu: the subtree kernel by presorted lists (dims 1-3)
cudaError_t launch_subtree_sorted(const EvDesc* evs, const uint2* subs, uint32_t nsub, CSoA in, CSoA b0, CSoA b1,
                                  Table tab, uint32_t* err, int dim, int subn, cudaStream_t stream);
// The shared-memory subtree kernel alone, for events whose d0 is 0 (reads
// every event from `src`).
cudaError_t launch_subtree_direct(const EvDesc* evs, const uint2* subs, uint32_t nsub, CSoA src, Table tab,
                                  uint32_t* err, int dim, cudaStream_t stream);
// fkd_features.cu: node summaries, bracket initialisation, target recording
cudaError_t launch_features(uint32_t d, const EvDesc* evs, const uint2* segs, uint32_t nseg, CSoA src, int dim,
                            float* feat, float2* range, cudaStream_t stream);
cudaError_t launch_bracket(uint32_t d, const EvDesc* evs, const uint2* segs, uint32_t nseg, const float* yhat,
                           const float2* range, float delta, SegSel* sel, unsigned long long* stats,
                           cudaStream_t stream);
cudaError_t launch_record(uint32_t d, const EvDesc* evs, const uint2* segs, uint32_t nseg, int dim, Table tab,
                          const float* feat, const float2* range, float* rec_x, float* rec_t,
                          unsigned long long* rec_n, uint64_t rec_cap, cudaStream_t stream);

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
  const EvDesc* evs;       // batched search: per-event geometry / bases (null: one event, g + tab)
  uint32_t nev;
  const uint32_t* order;   // optional processing order of the boxes (null: 0..q-1)
  uint32_t* counts;        // SEARCH_COUNT / SEARCH_DIGEST
  const uint64_t* offsets; // SEARCH_WRITE
  uint32_t* out;           // SEARCH_WRITE (heap indices when `heap_out`)
  uint64_t capacity;       // ids the output can hold
  unsigned long long* digests;  // SEARCH_DIGEST
  uint32_t* qcounter;      // work counter (zeroed by the launcher)
  uint32_t* err;
  int heap_out;            // write heap indices instead of ids
  uint32_t lanes;          // count / digest: lanes per box (1, 2, 4, 8, 16; 0 or 32: one warp per box)
  const uint32_t* evsel;   // batched search over a subset of the events (null: all boxes in order)
  const uint64_t* evsel_q; // exclusive prefix of the subset's box counts (nsel + 1 entries)
  uint32_t nsel;
  // count pass with a run pool: every box's result recorded as runs of the
  // in-order table, in chunks that k_expand writes out (null pool: no record)
  uint32_t* pool_st;             // in-order start of every run
  uint32_t* pool_len;            // its length
  uint32_t* pool_s;              // in-order position of every single (in-box node without a contained child)
  unsigned long long* pool_ctr;  // [0] runs, [1] singles reserved (zeroed by the caller; count past the caps)
  uint64_t pool_cap;             // runs
  uint64_t pool_cap_s;           // singles
  uint4* brec;                   // two uint4 per chunk: (box, offset within the box, singles position,
                                 // singles), (runs position, runs, 0, 0)
  unsigned long long* brec_ctr;  // chunks reserved (zeroed by the caller; counts past brec_cap)
  uint64_t brec_cap;
  uint32_t* flags;               // boxes whose runs did not fit (the write pass traverses them)
  uint32_t* flag_ctr;            // (zeroed by the caller)
  int rec_ids;                   // the singles pool holds ids, not in-order positions (unordered writes)
  int bucket_runs;               // recording with ids: leaf-bucket hits at consecutive positions still become runs
  unsigned long long* work_ctr;  // k_expand: records handed out (zeroed by the caller)
  // leaf buckets (needs tab.ipts): visited subtrees of height <= bucket are
  // scanned in in-order layout instead of walked (0: walk every level)
  uint32_t bucket;
  uint32_t bucket_grp;           // the same for the searches with fewer than 32 lanes per box (one lane
                                 // scans a bucket of at most 2^(h+1)-1 points)
  cudaStream_t stream;
};

cudaError_t launch_search(SearchCtx& sc, int dim, int mode);
// One box searched by one warp, level by level (no count pass): out[0] the
// result count, out[1] a frontier overflow flag, out[4 ..] the first cap ids
// in ascending heap order.
struct OneBox {
  float lo[4], hi[4];
};
cudaError_t launch_one(const Table& tab, uint32_t n, int dim, const OneBox& bx, uint32_t* out, uint32_t cap,
                       cudaStream_t stream);
// Writes the results of the runs a recording count pass stored (no-op without a pool).
cudaError_t launch_expand(const SearchCtx& sc);
// Fills tab.dids / tab.dnode (in-order tables; required by SEARCH_WRITE) and,
// when tab.ipts is set, the in-order node copy the leaf-bucket scan reads.
cudaError_t launch_inorder(const Geom& g, Table tab, cudaStream_t stream);
// The same for every event of a batch: ipts, and dids where tab.dids is set.
cudaError_t launch_inorder_events(const EvDesc* evs, uint32_t nev, uint32_t max_n, Table tab, cudaStream_t stream);
// Largest leaf-bucket height the searches accept (subtrees of up to 2^(h+1)-1 points).
constexpr uint32_t BUCKET_MAX = 6;
// Fills tab.sdig (subtree digests) for every event; required by SEARCH_DIGEST.
cudaError_t launch_subtree_digests(const EvDesc* evs, uint32_t nev, uint32_t max_n, Table tab, cudaStream_t stream);
// Sorts every box's result slice by heap index and maps it to ids.
cudaError_t launch_order_results(const Geom& g, const Table& tab, const uint64_t* offsets, uint64_t q, uint32_t* out,
                                 uint32_t* tmp, uint32_t* err, cudaStream_t stream);
// Processing order of the boxes (see fkd_search.cu); scratch holds
// box_order_words(q) words; *order_out points into it.
size_t box_order_words(uint64_t q);
cudaError_t launch_box_order(const Geom& g, const Table& tab, const Boxes& b, int dim, uint32_t* scratch,
                             uint32_t** order_out, cudaStream_t stream);
// fkd_nn.cu: radius search (a warp per query) and k-nearest-neighbour search
// (a thread per query); ctr is the SoA centre array of stride q.  launch_radius counts into
// `counts` when `out` is null, else writes heap indices (heap_out) or ids at
// `offsets`.
constexpr uint32_t KNN_MAX = 64;
cudaError_t launch_radius(const Geom& g, const Table& tab, const float* ctr, const float* rad, uint64_t q,
                          const uint32_t* order, uint32_t* counts, const uint64_t* offsets, uint32_t* out,
                          int heap_out, uint32_t* err, int dim, cudaStream_t stream);
cudaError_t launch_knn(const Geom& g, const Table& tab, const float* ctr, uint64_t q, const uint32_t* order,
                       uint32_t k, uint32_t* ids, float* d2, uint32_t* err, int dim, cudaStream_t stream);
// Exclusive prefix sum of q uint32 counts into q+1 uint64 offsets.
cudaError_t launch_scan_counts(const uint32_t* counts, uint64_t q, uint64_t* offsets, unsigned long long* partials,
                               cudaStream_t stream);
size_t scan_partials_words(uint64_t q);

}  // namespace fkd
