// fkd_batch.cu -- building and searching many independent events at once.
//
// No reference counterpart: the reference builds one FKDTree_CPU per event
// (FKDTree_cpu.h:19-23, :221-277).  Here thousands of uneven events are built
// by the same kernels as a single tree (fkd_build.cu, driven by the plan of
// fkd_plan.cu, which lists every (event, segment) of every global level) and
// searched by the same warp-per-box kernel (fkd_search.cu) with a per-box
// event lookup.  Events are grouped by dimension ("parts"); each part has its
// own working records and node tables.  fkd_batch_run captures gather, build
// and search into one CUDA graph and replays it for later calls with the same
// buffers.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/fkdtree_b200.h"
#include "fkd_internal.h"
#include "fkd_plan.h"
#include "fkd_mlp.h"

using namespace fkd;

namespace fkd {
fkd_status capi_fail(fkd_status s, const std::string& msg);
fkd_status capi_status_from_err(uint32_t e, const char* what);
}  // namespace fkd

namespace {

#define BCUDA(call)                                                                                      \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess)                                                                               \
      return capi_fail(e_ == cudaErrorMemoryAllocation ? FKD_ERR_NOMEM : FKD_ERR_CUDA,                   \
                       std::string(#call) + ": " + cudaGetErrorString(e_));                              \
  } while (0)

struct Buf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t want) {
    if (want <= bytes && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    if (want == 0) want = 16;
    cudaError_t e = device_alloc(&p, want);
    if (e == cudaSuccess) bytes = want;
    return e;
  }
  ~Buf() {
    if (p) cudaFree(p);
  }
  template <class T>
  T* as() const {
    return (T*)p;
  }
};

// Where an event's points live in the caller's arrays and in the part.
struct EvIO {
  uint64_t coord_off;  // caller: coordinates of the event, SoA slice [c*n + i]
  uint64_t pt_off;     // caller: ids of the event
  uint32_t base;       // part: first point
  uint32_t n;
};

constexpr uint32_t GATHER_CHUNK = 2048;

template <int DIM>
__global__ void k_gather(const EvIO* __restrict__ io, const uint2* __restrict__ chunks, const float* __restrict__ coords,
                         const uint32_t* __restrict__ ids, SoA work) {
  const uint2 ch = chunks[blockIdx.x];
  const EvIO e = io[ch.x];
  const uint32_t i0 = ch.y * GATHER_CHUNK;
  const uint32_t i1 = min(e.n, i0 + GATHER_CHUNK);
  for (uint32_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
#pragma unroll
    for (int c = 0; c < DIM; ++c)
      work.base[(uint64_t)c * work.stride + e.base + i] = __float_as_uint(coords[e.coord_off + (uint64_t)c * e.n + i]);
    work.ids[e.base + i] = ids[e.pt_off + i];
  }
}

template <int DIM>
__global__ void k_tables_scatter(const EvIO* __restrict__ io, const uint2* __restrict__ chunks,
                                 const uint4* __restrict__ nodes, const uint32_t* __restrict__ nids,
                                 float* __restrict__ tab, uint32_t* __restrict__ tab_ids) {
  const uint2 ch = chunks[blockIdx.x];
  const EvIO e = io[ch.x];
  const uint32_t i0 = ch.y * GATHER_CHUNK;
  const uint32_t i1 = min(e.n, i0 + GATHER_CHUNK);
  for (uint32_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const uint4 v = nodes[e.base + i];
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
    if (tab) {
#pragma unroll
      for (int c = 0; c < DIM; ++c) tab[e.coord_off + (uint64_t)c * e.n + i] = __uint_as_float(w[c]);
    }
    if (tab_ids) tab_ids[e.pt_off + i] = nids[e.base + i];
  }
}

struct Part {
  int dim = 3;
  std::vector<uint32_t> events;  // global indices
  uint64_t npts = 0, nq = 0;
  uint32_t maxn = 0;  // largest event (sizes the search stack)
  PlanDev plan;
  Buf io, chunks, work0, work1, nodes, ids, sel, ghist, lfeat, lyhat, lrange, sdig, bnd, tiebuf, ipts, dids;
  uint32_t nchunks = 0;
  std::vector<uint32_t> ev_n;  // points of every (local) event
  // digest search split by event size (knob search_big_n): [0] smaller events, [1] the others
  Buf evsel[2], evsel_q[2];
  uint32_t nsel[2] = {0, 0};
  uint64_t selq[2] = {0, 0};
};

}  // namespace

struct fkd_batch_s {
  uint32_t nev = 0;
  std::vector<uint32_t> dims;
  std::vector<uint64_t> pt_off, coord_off, q_off, qcoord_off;
  std::vector<std::unique_ptr<Part>> parts;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  uint32_t flags = 0;
  int device = 0;
  Buf err, qctr, passflags, stage_coords, stage_ids, stage_lo, stage_hi, stage_counts, stage_dig;
  uint32_t* herr = nullptr;
  bool built = false;
  bool planned = false;  // false after a failed (re-)plan: builds are refused until one succeeds
  // tuning knobs (fkd_batch_set_param)
  uint32_t hist_ctas = 0;
  uint32_t search_lanes = 0;
  uint32_t search_lanes_big = 0;  // lanes per box for events of at least search_big_n points (0: search_lanes)
  uint32_t search_big_n = 0;      // 0: one launch for every event
  int subtree = 0;
  int subtree_size = 0;   // presorted subtree size (0: 1,024)
  bool small_fix = true;  // selects stop at SMALL_CAP candidates, the partition orders them
  bool lin_pass = true;   // a segment's first digit pass bins its value range linearly
  uint32_t search_bucket = 5;  // leaf-bucket height of the warp-per-box digest search (0: walk every level)
  uint32_t search_bucket_grp = 0;  // ... of the digest search with fewer than 32 lanes per box
  // learned split
  fkd_mlp mlp = nullptr;
  float mlp_delta = 0.f;
  Buf lstats;
  // recording of training targets (fkd_batch_record)
  float* rec_x = nullptr;
  float* rec_t = nullptr;
  unsigned long long* rec_n = nullptr;
  uint64_t rec_cap = 0;
  // captured build+search graph and the pointers it was captured with
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  const void* gkey[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};

  ~fkd_batch_s() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    if (herr) cudaFreeHost(herr);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
};

namespace {

fkd_status batch_plan(fkd_batch b) {
  b->planned = false;
  b->built = false;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  const uint32_t hist_ctas = b->hist_ctas ? b->hist_ctas : 4u * (uint32_t)sms;
  for (auto& pp : b->parts) {
    Part& p = *pp;
    std::vector<uint32_t> n_ev, base_ev;
    std::vector<EvIO> io;
    std::vector<uint2> chunks;
    uint64_t base = 0, qb = 0;
    for (uint32_t le = 0; le < p.events.size(); ++le) {
      const uint32_t e = p.events[le];
      const uint32_t n = (uint32_t)(b->pt_off[e + 1] - b->pt_off[e]);
      n_ev.push_back(n);
      base_ev.push_back((uint32_t)base);
      p.maxn = std::max(p.maxn, n);
      io.push_back(EvIO{b->coord_off[e], b->pt_off[e], (uint32_t)base, n});
      for (uint32_t c = 0; c * GATHER_CHUNK < n; ++c) chunks.push_back(make_uint2(le, c));
      base += n;
    }
    p.npts = base;
    p.ev_n = n_ev;
    PlanHost ph;
    plan_build(n_ev.data(), base_ev.data(), (uint32_t)n_ev.size(), p.dim, hist_ctas, ph, b->subtree_size);
    for (uint32_t le = 0; le < p.events.size(); ++le) {
      const uint32_t e = p.events[le];
      EvDesc& d = ph.evs[le];
      d.nq = (uint32_t)(b->q_off[e + 1] - b->q_off[e]);
      d.qbase = qb;
      d.qcbase = b->qcoord_off[e];
      d.qout = b->q_off[e];
      qb += d.nq;
    }
    p.nq = qb;
    BCUDA(p.plan.upload(ph, b->stream));
    BCUDA(p.io.ensure(io.size() * sizeof(EvIO)));
    BCUDA(p.chunks.ensure(chunks.size() * sizeof(uint2)));
    if (!io.empty()) BCUDA(cudaMemcpy(p.io.p, io.data(), io.size() * sizeof(EvIO), cudaMemcpyHostToDevice));
    if (!chunks.empty())
      BCUDA(cudaMemcpy(p.chunks.p, chunks.data(), chunks.size() * sizeof(uint2), cudaMemcpyHostToDevice));
    p.nchunks = (uint32_t)chunks.size();
    const size_t rec = (size_t)(p.dim + 1) * p.npts * 4;
    BCUDA(p.work0.ensure(rec));
    BCUDA(p.work1.ensure(rec));
    BCUDA(p.nodes.ensure(p.npts * sizeof(uint4)));
    BCUDA(p.ids.ensure(p.npts * 4));
    BCUDA(p.sel.ensure(sizeof(SegSel) * (size_t)p.plan.maxseg));
    BCUDA(p.bnd.ensure(2 * sizeof(uint2) * (size_t)p.plan.maxseg));
    BCUDA(p.tiebuf.ensure((size_t)p.plan.maxseg * SMALL_CAP * (p.dim + 1) * 4));
    // leaf-bucket tables (in-order node copy; ids too in 4-D): allocated here,
    // never while a graph is being captured
    BCUDA(p.ipts.ensure(p.npts * sizeof(uint4)));
    if (p.dim > 3) BCUDA(p.dids.ensure(p.npts * sizeof(uint32_t)));
    BCUDA(p.ghist.ensure((size_t)p.plan.maxseg * HIST_BINS * 4));
    BCUDA(p.sdig.ensure(p.npts * sizeof(unsigned long long)));
    BCUDA(p.lfeat.ensure((size_t)p.plan.maxseg * FKD_MLP_FEATURES * 4));
    BCUDA(p.lyhat.ensure((size_t)p.plan.maxseg * 4));
    BCUDA(p.lrange.ensure((size_t)p.plan.maxseg * sizeof(float2)));
  }
  BCUDA(b->lstats.ensure(64));
  BCUDA(cudaStreamSynchronize(b->stream));
  b->planned = true;
  return FKD_OK;
}

template <int DIM>
void launch_gather(Part& p, const float* coords, const uint32_t* ids, cudaStream_t s) {
  SoA w{p.work1.as<uint32_t>(), p.work1.as<uint32_t>() + (size_t)DIM * p.npts, p.npts};
  if (p.nchunks) {
    k_gather<DIM><<<p.nchunks, 256, 0, s>>>(p.io.as<EvIO>(), p.chunks.as<uint2>(), coords, ids, w);
    count_launches(1);
  }
}

// gather + build of every part (stream-ordered, capturable)
fkd_status enqueue_build(fkd_batch b, const float* coords, const uint32_t* ids) {
  for (auto& pp : b->parts) {
    Part& p = *pp;
    if (p.npts == 0) continue;
    switch (p.dim) {
      case 1: launch_gather<1>(p, coords, ids, b->stream); break;
      case 2: launch_gather<2>(p, coords, ids, b->stream); break;
      case 3: launch_gather<3>(p, coords, ids, b->stream); break;
      default: launch_gather<4>(p, coords, ids, b->stream); break;
    }
    BCUDA(cudaGetLastError());
    BCUDA(cudaMemsetAsync(p.ghist.p, 0, (size_t)p.plan.maxseg * HIST_BINS * 4, b->stream));
    BuildCtx bc;
    uint32_t* w0 = p.work0.as<uint32_t>();
    uint32_t* w1 = p.work1.as<uint32_t>();
    bc.input = CSoA{w1, w1 + (size_t)p.dim * p.npts, p.npts};
    bc.work[0] = SoA{w0, w0 + (size_t)p.dim * p.npts, p.npts};
    bc.work[1] = SoA{w1, w1 + (size_t)p.dim * p.npts, p.npts};
    bc.evs = p.plan.evs;
    bc.nlevels = (uint32_t)p.plan.levels.size();
    bc.levels = p.plan.levels.data();
    bc.subs = p.plan.subs;
    bc.nsub = p.plan.nsub;
    bc.sel = p.sel.as<SegSel>();
    bc.ghist = p.ghist.as<uint32_t>();
    bc.tab = Table{p.nodes.as<uint4>(), p.ids.as<uint32_t>()};
    bc.err = b->err.as<uint32_t>();
    bc.pending = b->passflags.as<uint32_t>();
    bc.bnd = p.bnd.as<uint2>();
    bc.bnd_stride = p.plan.maxseg;
    bc.tiebuf = b->small_fix ? p.tiebuf.as<uint32_t>() : nullptr;
    bc.lin = b->lin_pass;
    bc.subtree = b->subtree;
    bc.subn = b->subtree_size;
    bc.stream = b->stream;
    memset(&bc.learn, 0, sizeof bc.learn);
    bc.learn.stats = b->lstats.as<unsigned long long>();  // [3] counts the digit passes
    if (b->mlp || b->rec_x) {
      bc.learn.feat = p.lfeat.as<float>();
      bc.learn.yhat = p.lyhat.as<float>();
      bc.learn.range = p.lrange.as<float2>();
      bc.learn.stats = b->lstats.as<unsigned long long>();
    }
    if (b->mlp) {
      bc.learn.params = mlp_params(b->mlp);
      bc.learn.delta = b->mlp_delta;
    }
    if (b->rec_x) {
      bc.learn.rec_x = b->rec_x;
      bc.learn.rec_t = b->rec_t;
      bc.learn.rec_n = b->rec_n;
      bc.learn.rec_cap = b->rec_cap;
    }
    BCUDA(launch_build(bc, p.dim));
  }
  return FKD_OK;
}

// The event subsets of a size-split digest search: events with boxes, below
// search_big_n points in [0], the others in [1] (uploaded once per knob value).
fkd_status batch_search_sets(fkd_batch b) {
  for (auto& pp : b->parts) {
    Part& p = *pp;
    std::vector<uint32_t> sel[2];
    std::vector<uint64_t> q[2];
    q[0].push_back(0);
    q[1].push_back(0);
    for (uint32_t le = 0; le < p.ev_n.size(); ++le) {
      const uint32_t e = p.events[le];
      const uint64_t nq = b->q_off[e + 1] - b->q_off[e];
      if (nq == 0) continue;
      const int k = (b->search_big_n && p.ev_n[le] >= b->search_big_n) ? 1 : 0;
      sel[k].push_back(le);
      q[k].push_back(q[k].back() + nq);
    }
    for (int k = 0; k < 2; ++k) {
      p.nsel[k] = (uint32_t)sel[k].size();
      p.selq[k] = q[k].back();
      if (sel[k].empty()) continue;
      BCUDA(p.evsel[k].ensure(sel[k].size() * sizeof(uint32_t)));
      BCUDA(p.evsel_q[k].ensure(q[k].size() * sizeof(uint64_t)));
      BCUDA(cudaMemcpy(p.evsel[k].p, sel[k].data(), sel[k].size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
      BCUDA(cudaMemcpy(p.evsel_q[k].p, q[k].data(), q[k].size() * sizeof(uint64_t), cudaMemcpyHostToDevice));
    }
  }
  return FKD_OK;
}

fkd_status enqueue_digest(fkd_batch b, const float* mins, const float* maxs, uint32_t* counts, uint64_t* digests) {
  for (auto& pp : b->parts) {
    Part& p = *pp;
    if (p.nq == 0) continue;
    Table tab{p.nodes.as<uint4>(), p.ids.as<uint32_t>(), p.sdig.as<unsigned long long>()};
    BCUDA(launch_subtree_digests(p.plan.evs, p.plan.nev, p.maxn, tab, b->stream));
    // leaf buckets (in-order node copy per event), when a search that scans them runs
    const bool full_warp = b->search_lanes == 0 || b->search_lanes == 32 ||
                           (b->search_big_n && (b->search_lanes_big == 0 || b->search_lanes_big == 32));
    if ((b->search_bucket && full_warp) || b->search_bucket_grp) {
      tab.ipts = p.ipts.as<uint4>();
      tab.dids = p.dim > 3 ? p.dids.as<uint32_t>() : nullptr;
      BCUDA(launch_inorder_events(p.plan.evs, p.plan.nev, p.maxn, tab, b->stream));
    }
    SearchCtx sc;
    memset(&sc, 0, sizeof sc);
    sc.g = make_geom(p.maxn);  // per-box geometry comes from the event; this sizes the stack
    sc.tab = tab;
    sc.boxes = Boxes{mins, maxs, 0, p.nq};
    sc.evs = p.plan.evs;
    sc.nev = p.plan.nev;
    sc.counts = counts;
    sc.digests = (unsigned long long*)digests;
    sc.qcounter = b->qctr.as<uint32_t>();
    sc.err = b->err.as<uint32_t>();
    sc.capacity = ~0ull;
    sc.lanes = b->search_lanes;
    sc.bucket = tab.ipts ? b->search_bucket : 0u;
    sc.bucket_grp = tab.ipts ? b->search_bucket_grp : 0u;
    sc.stream = b->stream;
    if (b->search_big_n == 0) {
      BCUDA(launch_search(sc, p.dim, SEARCH_DIGEST));
      continue;
    }
    // small and large events with their own lanes per box
    for (int k = 0; k < 2; ++k) {
      if (p.nsel[k] == 0) continue;
      SearchCtx s2 = sc;
      s2.boxes.q = p.selq[k];
      s2.evsel = p.evsel[k].as<uint32_t>();
      s2.evsel_q = p.evsel_q[k].as<uint64_t>();
      s2.nsel = p.nsel[k];
      if (k == 1 && b->search_lanes_big) s2.lanes = b->search_lanes_big;
      BCUDA(launch_search(s2, p.dim, SEARCH_DIGEST));
    }
  }
  return FKD_OK;
}

fkd_status batch_finish(fkd_batch b, const char* what, int mem) {
  if (mem == FKD_MEM_DEVICE && (b->flags & FKD_FLAG_ASYNC)) return FKD_OK;
  BCUDA(cudaMemcpyAsync(b->herr, b->err.p, 4, cudaMemcpyDeviceToHost, b->stream));
  BCUDA(cudaStreamSynchronize(b->stream));
  return capi_status_from_err(*b->herr, what);
}

uint64_t coords_total(fkd_batch b) { return b->coord_off[b->nev]; }
uint64_t boxes_total(fkd_batch b) { return b->qcoord_off[b->nev]; }

}  // namespace

extern "C" {

fkd_status fkd_batch_create(uint32_t n_events, const uint32_t* dims, const uint64_t* pt_off, const uint64_t* q_off,
                            uint32_t flags, void* stream, fkd_batch* out) {
  if (!out) return capi_fail(FKD_ERR_ARG, "null output handle pointer");
  *out = nullptr;
  if (n_events == 0 || !dims || !pt_off || !q_off) return capi_fail(FKD_ERR_ARG, "empty batch or null arrays");
  std::unique_ptr<fkd_batch_s> b(new (std::nothrow) fkd_batch_s());
  if (!b) return capi_fail(FKD_ERR_NOMEM, "host allocation failed");
  b->nev = n_events;
  b->flags = flags;
  b->dims.assign(dims, dims + n_events);
  b->pt_off.assign(pt_off, pt_off + n_events + 1);
  b->q_off.assign(q_off, q_off + n_events + 1);
  b->coord_off.assign(n_events + 1, 0);
  b->qcoord_off.assign(n_events + 1, 0);
  std::map<int, Part*> bydim;
  for (uint32_t e = 0; e < n_events; ++e) {
    if (dims[e] < 1 || dims[e] > 4) return capi_fail(FKD_ERR_ARG, "event dims must be 1..4");
    if (pt_off[e + 1] < pt_off[e] || q_off[e + 1] < q_off[e]) return capi_fail(FKD_ERR_ARG, "offsets must not decrease");
    const uint64_t n = pt_off[e + 1] - pt_off[e];
    if (n >= (1ull << 31)) return capi_fail(FKD_ERR_ARG, "at most 2^31-1 points per event");
    b->coord_off[e + 1] = b->coord_off[e] + dims[e] * n;
    b->qcoord_off[e + 1] = b->qcoord_off[e] + dims[e] * (q_off[e + 1] - q_off[e]);
    Part*& p = bydim[(int)dims[e]];
    if (!p) {
      b->parts.emplace_back(new Part());
      p = b->parts.back().get();
      p->dim = (int)dims[e];
    }
    p->events.push_back(e);
  }
  for (auto& p : b->parts) {
    uint64_t tot = 0;
    for (uint32_t e : p->events) tot += pt_off[e + 1] - pt_off[e];
    if (tot >= (1ull << 32)) return capi_fail(FKD_ERR_ARG, "at most 2^32-1 points per dimension class");
  }
  BCUDA(cudaGetDevice(&b->device));
  if (stream) {
    b->stream = (cudaStream_t)stream;
  } else {
    BCUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->own_stream = true;
  }
  BCUDA(b->err.ensure(16));
  BCUDA(b->qctr.ensure(16));
  BCUDA(b->passflags.ensure(256));
  BCUDA(cudaMallocHost((void**)&b->herr, 16));
  BCUDA(cudaMemsetAsync(b->err.p, 0, 4, b->stream));
  fkd_status s = batch_plan(b.get());
  if (s != FKD_OK) return s;
  *out = b.release();
  return FKD_OK;
}

fkd_status fkd_batch_destroy(fkd_batch b) {
  if (!b) return FKD_OK;
  cudaStreamSynchronize(b->stream);
  delete b;
  return FKD_OK;
}

fkd_status fkd_batch_set_param(fkd_batch b, const char* name, int64_t value) {
  if (!b || !name) return capi_fail(FKD_ERR_ARG, "null argument");
  auto drop_graph = [b]() {
    if (b->gexec) {
      cudaGraphExecDestroy(b->gexec);
      b->gexec = nullptr;
    }
    if (b->graph) {
      cudaGraphDestroy(b->graph);
      b->graph = nullptr;
    }
  };
  if (strcmp(name, "hist_ctas") == 0) {
    if (value < 0 || value > (1 << 20)) return capi_fail(FKD_ERR_ARG, "hist_ctas out of range");
    b->hist_ctas = (uint32_t)value;
    drop_graph();
    return batch_plan(b);
  }
  if (strcmp(name, "subtree") == 0) {
    if (value < 0 || value > 2) return capi_fail(FKD_ERR_ARG, "subtree must be 0, 1 or 2");
    b->subtree = (int)value;
    drop_graph();
    return FKD_OK;
  }
  if (strcmp(name, "subtree_size") == 0) {
    if (value != 0 && value != 512 && value != 1024)
      return capi_fail(FKD_ERR_ARG, "subtree_size must be 0, 512 or 1024");
    b->subtree_size = (int)value;
    drop_graph();
    return batch_plan(b);
  }
  if (strcmp(name, "small_fix") == 0) {
    if (value != 0 && value != 1) return capi_fail(FKD_ERR_ARG, "small_fix must be 0 or 1");
    b->small_fix = value != 0;
    drop_graph();
    return FKD_OK;
  }
  if (strcmp(name, "lin_pass") == 0) {
    if (value != 0 && value != 1) return capi_fail(FKD_ERR_ARG, "lin_pass must be 0 or 1");
    b->lin_pass = value != 0;
    drop_graph();
    return FKD_OK;
  }
  if (strcmp(name, "search_bucket") == 0) {
    if (value < 0 || value > (int64_t)BUCKET_MAX) return capi_fail(FKD_ERR_ARG, "search_bucket must be 0..6");
    b->search_bucket = (uint32_t)value;
    drop_graph();
    return FKD_OK;
  }
  if (strcmp(name, "search_bucket_lanes") == 0) {
    if (value < 0 || value > 3) return capi_fail(FKD_ERR_ARG, "search_bucket_lanes must be 0..3");
    b->search_bucket_grp = (uint32_t)value;
    drop_graph();
    return FKD_OK;
  }
  if (strcmp(name, "search_lanes_big") == 0) {
    if (value != 0 && value != 1 && value != 2 && value != 4 && value != 8 && value != 16 && value != 32)
      return capi_fail(FKD_ERR_ARG, "search_lanes_big must be 0, 1, 2, 4, 8, 16 or 32");
    b->search_lanes_big = (uint32_t)value;
    drop_graph();
    return FKD_OK;
  }
  if (strcmp(name, "search_big_n") == 0) {
    if (value < 0 || value > 0x7fffffffll) return capi_fail(FKD_ERR_ARG, "search_big_n out of range");
    b->search_big_n = (uint32_t)value;
    drop_graph();
    return batch_search_sets(b);
  }
  if (strcmp(name, "search_lanes") == 0) {
    if (value != 0 && value != 1 && value != 2 && value != 4 && value != 8 && value != 16 && value != 32)
      return capi_fail(FKD_ERR_ARG, "search_lanes must be 0, 1, 2, 4, 8, 16 or 32");
    b->search_lanes = (uint32_t)value;
    drop_graph();
    return FKD_OK;
  }
  return capi_fail(FKD_ERR_ARG, std::string("unknown parameter ") + name);
}

fkd_status fkd_batch_build(fkd_batch b, const float* coords, const uint32_t* ids, int mem) {
  if (!b) return capi_fail(FKD_ERR_ARG, "null handle");
  if (mem != FKD_MEM_HOST && mem != FKD_MEM_DEVICE) return capi_fail(FKD_ERR_ARG, "bad mem");
  const uint64_t nc = coords_total(b), np = b->pt_off[b->nev];
  if (np && (!coords || !ids)) return capi_fail(FKD_ERR_ARG, "null coords or ids");
  if (!b->planned) return capi_fail(FKD_ERR_STATE, "the batch has no build plan (a re-plan failed); set hist_ctas again");
  b->built = false;
  if (mem == FKD_MEM_HOST && np) {
    BCUDA(b->stage_coords.ensure(nc * 4));
    BCUDA(b->stage_ids.ensure(np * 4));
    BCUDA(cudaMemcpyAsync(b->stage_coords.p, coords, nc * 4, cudaMemcpyHostToDevice, b->stream));
    BCUDA(cudaMemcpyAsync(b->stage_ids.p, ids, np * 4, cudaMemcpyHostToDevice, b->stream));
    coords = b->stage_coords.as<float>();
    ids = b->stage_ids.as<uint32_t>();
  }
  BCUDA(cudaMemsetAsync(b->err.p, 0, 4, b->stream));
  fkd_status s = enqueue_build(b, coords, ids);
  if (s != FKD_OK) return s;
  b->built = true;
  s = batch_finish(b, "fkd_batch_build", mem);
  if (s != FKD_OK) b->built = false;
  return s;
}

fkd_status fkd_batch_get_tables(fkd_batch b, float* tab, uint32_t* tab_ids, int mem) {
  if (!b) return capi_fail(FKD_ERR_ARG, "null handle");
  if (!b->built) return capi_fail(FKD_ERR_STATE, "tables requested before build");
  const uint64_t nc = coords_total(b), np = b->pt_off[b->nev];
  float* dt = tab;
  uint32_t* di = tab_ids;
  if (mem == FKD_MEM_HOST) {
    BCUDA(b->stage_coords.ensure(nc * 4));
    BCUDA(b->stage_ids.ensure(np * 4));
    dt = tab ? b->stage_coords.as<float>() : nullptr;
    di = tab_ids ? b->stage_ids.as<uint32_t>() : nullptr;
  }
  for (auto& pp : b->parts) {
    Part& p = *pp;
    if (!p.nchunks) continue;
    switch (p.dim) {
      case 1: k_tables_scatter<1><<<p.nchunks, 256, 0, b->stream>>>(p.io.as<EvIO>(), p.chunks.as<uint2>(), p.nodes.as<uint4>(), p.ids.as<uint32_t>(), dt, di); break;
      case 2: k_tables_scatter<2><<<p.nchunks, 256, 0, b->stream>>>(p.io.as<EvIO>(), p.chunks.as<uint2>(), p.nodes.as<uint4>(), p.ids.as<uint32_t>(), dt, di); break;
      case 3: k_tables_scatter<3><<<p.nchunks, 256, 0, b->stream>>>(p.io.as<EvIO>(), p.chunks.as<uint2>(), p.nodes.as<uint4>(), p.ids.as<uint32_t>(), dt, di); break;
      default: k_tables_scatter<4><<<p.nchunks, 256, 0, b->stream>>>(p.io.as<EvIO>(), p.chunks.as<uint2>(), p.nodes.as<uint4>(), p.ids.as<uint32_t>(), dt, di); break;
    }
    count_launches(1);
    BCUDA(cudaGetLastError());
  }
  if (mem == FKD_MEM_HOST) {
    if (tab) BCUDA(cudaMemcpyAsync(tab, dt, nc * 4, cudaMemcpyDeviceToHost, b->stream));
    if (tab_ids) BCUDA(cudaMemcpyAsync(tab_ids, di, np * 4, cudaMemcpyDeviceToHost, b->stream));
  }
  BCUDA(cudaStreamSynchronize(b->stream));
  return FKD_OK;
}

static fkd_status stage_batch_boxes(fkd_batch b, const float** mins, const float** maxs, int mem) {
  if (mem != FKD_MEM_HOST) return FKD_OK;
  const uint64_t nb = boxes_total(b);
  BCUDA(b->stage_lo.ensure(nb * 4));
  BCUDA(b->stage_hi.ensure(nb * 4));
  if (nb) {
    BCUDA(cudaMemcpyAsync(b->stage_lo.p, *mins, nb * 4, cudaMemcpyHostToDevice, b->stream));
    BCUDA(cudaMemcpyAsync(b->stage_hi.p, *maxs, nb * 4, cudaMemcpyHostToDevice, b->stream));
  }
  *mins = b->stage_lo.as<float>();
  *maxs = b->stage_hi.as<float>();
  return FKD_OK;
}

fkd_status fkd_batch_search_digest(fkd_batch b, const float* mins, const float* maxs, uint32_t* counts,
                                   uint64_t* digests, int mem) {
  if (!b) return capi_fail(FKD_ERR_ARG, "null handle");
  if (!b->built) return capi_fail(FKD_ERR_STATE, "search before build");
  const uint64_t q = b->q_off[b->nev];
  if (q && (!mins || !maxs || !counts || !digests)) return capi_fail(FKD_ERR_ARG, "null boxes or outputs");
  fkd_status s = stage_batch_boxes(b, &mins, &maxs, mem);
  if (s != FKD_OK) return s;
  uint32_t* dc = counts;
  uint64_t* dd = digests;
  if (mem == FKD_MEM_HOST) {
    BCUDA(b->stage_counts.ensure(q * 4));
    BCUDA(b->stage_dig.ensure(q * 8));
    dc = b->stage_counts.as<uint32_t>();
    dd = b->stage_dig.as<uint64_t>();
  }
  BCUDA(cudaMemsetAsync(b->err.p, 0, 4, b->stream));
  if ((s = enqueue_digest(b, mins, maxs, dc, dd)) != FKD_OK) return s;
  if (mem == FKD_MEM_HOST && q) {
    BCUDA(cudaMemcpyAsync(counts, dc, q * 4, cudaMemcpyDeviceToHost, b->stream));
    BCUDA(cudaMemcpyAsync(digests, dd, q * 8, cudaMemcpyDeviceToHost, b->stream));
  }
  return batch_finish(b, "fkd_batch_search_digest", mem);
}

fkd_status fkd_batch_run(fkd_batch b, const float* coords, const uint32_t* ids, const float* mins, const float* maxs,
                         uint32_t* counts, uint64_t* digests) {
  if (!b) return capi_fail(FKD_ERR_ARG, "null handle");
  const uint64_t q = b->q_off[b->nev], np = b->pt_off[b->nev];
  if ((np && (!coords || !ids)) || (q && (!mins || !maxs || !counts || !digests)))
    return capi_fail(FKD_ERR_ARG, "null device buffer");
  if (!b->planned) return capi_fail(FKD_ERR_STATE, "the batch has no build plan (a re-plan failed); set hist_ctas again");
  const void* key[6] = {coords, ids, mins, maxs, counts, digests};
  if (!b->gexec || memcmp(key, b->gkey, sizeof key) != 0) {
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
    BCUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    fkd_status s = FKD_OK;
    if (cudaMemsetAsync(b->err.p, 0, 4, b->stream) != cudaSuccess) s = FKD_ERR_CUDA;
    if (s == FKD_OK) s = enqueue_build(b, coords, ids);
    if (s == FKD_OK) s = enqueue_digest(b, mins, maxs, counts, digests);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
    if (s != FKD_OK) {
      if (g) cudaGraphDestroy(g);
      return s;
    }
    BCUDA(ce);
    b->graph = g;
    BCUDA(cudaGraphInstantiate(&b->gexec, g, 0));
    memcpy(b->gkey, key, sizeof key);
  }
  BCUDA(cudaGraphLaunch(b->gexec, b->stream));
  b->built = true;
  return batch_finish(b, "fkd_batch_run", FKD_MEM_DEVICE);
}

fkd_status fkd_batch_set_mlp(fkd_batch b, fkd_mlp m, float delta) {
  if (!b) return capi_fail(FKD_ERR_ARG, "null handle");
  if (m && !(delta > 0.f)) return capi_fail(FKD_ERR_ARG, "delta must be positive");
  b->mlp = m;
  b->mlp_delta = delta;
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->gexec = nullptr;
  b->graph = nullptr;
  BCUDA(cudaMemsetAsync(b->lstats.p, 0, 32, b->stream));
  BCUDA(cudaStreamSynchronize(b->stream));
  return FKD_OK;
}

fkd_status fkd_batch_learn_stats(fkd_batch b, uint64_t* stats, int reset) {
  if (!b || !stats) return capi_fail(FKD_ERR_ARG, "null argument");
  BCUDA(cudaMemcpyAsync(stats, b->lstats.p, 4 * sizeof(uint64_t), cudaMemcpyDeviceToHost, b->stream));
  if (reset) BCUDA(cudaMemsetAsync(b->lstats.p, 0, 32, b->stream));
  BCUDA(cudaStreamSynchronize(b->stream));
  return FKD_OK;
}

fkd_status fkd_batch_record(fkd_batch b, const float* coords, const uint32_t* ids, float* x_out, float* t_out,
                            uint64_t cap, uint64_t* n_out, int mem) {
  if (!b || !n_out || (cap && (!x_out || !t_out))) return capi_fail(FKD_ERR_ARG, "null argument");
  Buf dx, dt, dn;
  BCUDA(dx.ensure((cap ? cap : 1) * FKD_MLP_FEATURES * 4));
  BCUDA(dt.ensure((cap ? cap : 1) * 4));
  BCUDA(dn.ensure(8));
  BCUDA(cudaMemsetAsync(dn.p, 0, 8, b->stream));
  fkd_mlp saved = b->mlp;
  b->mlp = nullptr;  // recording needs the plain (exact, unpredicted) select
  b->rec_x = dx.as<float>();
  b->rec_t = dt.as<float>();
  b->rec_n = dn.as<unsigned long long>();
  b->rec_cap = cap;
  fkd_status s = fkd_batch_build(b, coords, ids, mem);
  b->mlp = saved;
  b->rec_x = b->rec_t = nullptr;
  b->rec_n = nullptr;
  b->rec_cap = 0;
  if (s != FKD_OK) return s;
  unsigned long long n = 0;
  BCUDA(cudaMemcpy(&n, dn.p, 8, cudaMemcpyDeviceToHost));
  *n_out = n;
  const uint64_t m = n < cap ? n : cap;
  if (m) {
    BCUDA(cudaMemcpy(x_out, dx.p, m * FKD_MLP_FEATURES * 4, cudaMemcpyDeviceToHost));
    BCUDA(cudaMemcpy(t_out, dt.p, m * 4, cudaMemcpyDeviceToHost));
  }
  return FKD_OK;
}

fkd_status fkd_batch_sync(fkd_batch b) {
  if (!b) return capi_fail(FKD_ERR_ARG, "null handle");
  return batch_finish(b, "fkd_batch_sync", FKD_MEM_HOST);
}

}  // extern "C"
