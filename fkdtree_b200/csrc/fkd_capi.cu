// fkd_capi.cu -- the C ABI (include/fkdtree_b200.h) over the build and search
// kernels: handle lifetime, device buffers, host staging and error latching.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <mutex>
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
static unsigned long long g_launches = 0;
void count_launches(uint64_t k) { __atomic_fetch_add(&g_launches, (unsigned long long)k, __ATOMIC_RELAXED); }
uint64_t launches_total() { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

// Allocation failure injection (fkd_debug_fail_alloc): >= 0 counts down the
// device allocations left before one fails; -1 (the default) is off.
static int g_fail_alloc = -1;
cudaError_t device_alloc(void** p, size_t bytes) {
  int v = __atomic_load_n(&g_fail_alloc, __ATOMIC_RELAXED);
  while (v >= 0) {
    if (__atomic_compare_exchange_n(&g_fail_alloc, &v, v - 1, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
      if (v == 0) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
      }
      break;
    }
  }
  return cudaMalloc(p, bytes);
}
}  // namespace fkd

namespace {

thread_local std::string g_last_error;

fkd_status fail(fkd_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

#define FKD_CUDA(call)                                                                                    \
  do {                                                                                                    \
    cudaError_t e_ = (call);                                                                              \
    if (e_ != cudaSuccess)                                                                                \
      return fail(e_ == cudaErrorMemoryAllocation ? FKD_ERR_NOMEM : FKD_ERR_CUDA,                         \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                                    \
  } while (0)

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t want) {
    if (want <= bytes && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    if (want == 0) return cudaSuccess;
    cudaError_t e = device_alloc(&p, want);
    if (e == cudaSuccess) bytes = want;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T>
  T* as() const {
    return (T*)p;
  }
};

}  // namespace

// Per-call scratch of the searches.  Every search call leases one slot from
// its handle's pool for its duration, so searches on one built tree may run
// from several host threads at once (the reference's TBB loop over one tree,
// main.cpp:351-359): each has its own staging buffers, error word and -- for
// host-memory calls -- its own stream; the tree tables are only read.
struct SearchSlot {
  DevBuf qlo, qhi, counts, offsets, partials, out, tmp, digests, qorder;
  DevBuf pool_st, pool_len, pool_s, brec, jctr, rflags, err, qctr, one;
  uint32_t* herr = nullptr;      // pinned: [0] error word, [2..3] total, [4..11] pool demand
  uint32_t* hone = nullptr;      // pinned: the single-box search's count, flag and first ids
  cudaStream_t own = nullptr;    // stream of host-memory calls
  cudaEvent_t done = nullptr;    // the slot's last work (waited on by its next lease)
  // run pool of fkd_search, sized by the previous call's demand
  uint64_t pool_want = 0, pool_s_want = 0, brec_want = 0;
  ~SearchSlot() {
    DevBuf* all[] = {&qlo, &qhi, &counts, &offsets, &partials, &out, &tmp, &digests, &qorder,
                     &pool_st, &pool_len, &pool_s, &brec, &jctr, &rflags, &err, &qctr, &one};
    if (own) cudaStreamSynchronize(own);
    for (DevBuf* b : all) b->release();
    if (herr) cudaFreeHost(herr);
    if (hone) cudaFreeHost(hone);
    if (done) cudaEventDestroy(done);
    if (own) cudaStreamDestroy(own);
  }
};

struct fkd_tree_s {
  int dim = 3;
  uint32_t flags = 0;
  cudaStream_t stream = nullptr;
  int device = 0;
  uint64_t n = 0;
  bool built = false;
  DevBuf nodes, ids, work0, work1, sel, ghist, err, qctr, passflags, tmp;
  uint32_t* herr = nullptr;  // pinned mirror of err
  PlanDev plan;              // build plan of the last size built
  uint64_t plan_n = ~0ull;
  uint32_t hist_ctas = 0;    // digit-pass CTAs per level (0: four per SM)
  uint32_t search_lanes = 0; // count / digest lanes per box (0: one warp)
  int subtree = 0;           // subtree kernel: 0 auto, 1 radix select, 2 presorted lists
  int subtree_size = 0;      // presorted subtree size: 0 (1,024), 512 or 1,024 ("subtree_size")
  bool small_select = true;  // one CTA per segment on levels of small segments
  bool box_order = true;     // search boxes in the spatial order of their centres
  fkd_mlp mlp = nullptr;     // learned split (null: plain radix select)
  float mlp_delta = 0.f;
  DevBuf lfeat, lyhat, lrange, lstats, sdig, dids, dnode, ipts, bnd, tiebuf;
  bool small_fix = true;        // selects stop at SMALL_CAP candidates, the partition orders them ("small_fix")
  bool lin_pass = true;         // a segment's first digit pass bins its value range linearly ("lin_pass")
  uint32_t search_bucket = 5;   // leaf-bucket height of the searches ("search_bucket"; 0: walk every level)
  uint32_t search_bucket_grp = 0;  // ... of the searches with fewer than 32 lanes per box ("search_bucket_lanes")
  bool bucket_runs = true;      // unordered recorded searches merge consecutive bucket hits into runs ("bucket_runs")
  bool search_record = true;    // fkd_search records runs in the count pass ("search_record")
  bool search_one = true;       // fkd_search of one host-memory box: one level-order warp ("search_one")
  uint64_t search_pool = 0;     // fixed pool entries ("search_pool"; 0: sized by demand)
  // tables derived from the tree on first use (in-order ids / heap indices /
  // nodes, subtree digests), built once under tree_mu; the events mark them ready
  bool sdig_valid = false;
  bool inorder_valid = false;
  bool ipts_valid = false;
  std::mutex tree_mu;
  cudaEvent_t built_ev = nullptr, inorder_ev = nullptr, sdig_ev = nullptr;
  // search slots (SearchSlot): all of them, and the ones not leased
  std::mutex slot_mu;
  std::vector<std::unique_ptr<SearchSlot>> slots;
  std::vector<SearchSlot*> free_slots;
  std::mutex tab_mu;  // fkd_get_tables stages through work0
  // optional per-kernel timing (fkd_set_param "kernel_events"): a ring of
  // KEV_RING event sets, one per build / search call
  static constexpr uint32_t KEV_RING = 64;
  std::vector<cudaEvent_t> kev;  // [slot * 7 + k]: 0 count start, 1 count end, 2 write start, 3 write end,
                                 //                  4 build start, 5 subtree start, 6 build end
  uint64_t kev_builds = 0, kev_searches = 0;

  ~fkd_tree_s() {
    slots.clear();
    DevBuf* all[] = {&nodes, &ids, &work0, &work1, &sel, &ghist, &err, &qctr, &passflags, &tmp,
                     &lfeat, &lyhat, &lrange, &lstats, &sdig, &dids, &dnode, &ipts, &bnd, &tiebuf};
    for (DevBuf* b : all) b->release();
    if (herr) cudaFreeHost(herr);
    for (cudaEvent_t e : kev) cudaEventDestroy(e);
    for (cudaEvent_t e : {built_ev, inorder_ev, sdig_ev})
      if (e) cudaEventDestroy(e);
  }
  cudaEvent_t kev_at(uint64_t call, int k) { return kev[(size_t)(call % KEV_RING) * 7 + k]; }
};

namespace {

fkd_status status_from_err(uint32_t e, const char* what) {
  if (e == 0) return FKD_OK;
  char buf[160];
  if (e & ERRB_NAN) {
    snprintf(buf, sizeof buf, "%s: input coordinates contain NaN", what);
    return fail(FKD_ERR_NAN, buf);
  }
  if (e & ERRB_CAPACITY) {
    snprintf(buf, sizeof buf, "%s: a result or frontier capacity was exceeded", what);
    return fail(FKD_ERR_CAPACITY, buf);
  }
  if (e & ERRB_TIMEOUT) {
    snprintf(buf, sizeof buf, "%s: a bounded device wait gave up", what);
    return fail(FKD_ERR_TIMEOUT, buf);
  }
  snprintf(buf, sizeof buf, "%s: device consistency check failed (0x%x)", what, e);
  return fail(FKD_ERR_INTERNAL, buf);
}

// Reads the handle's (build) error word and clears it.
fkd_status check_err_word(fkd_tree h, const char* what) {
  FKD_CUDA(cudaMemcpyAsync(h->herr, h->err.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  FKD_CUDA(cudaMemsetAsync(h->err.p, 0, sizeof(uint32_t), h->stream));
  FKD_CUDA(cudaStreamSynchronize(h->stream));
  return status_from_err(*h->herr, what);
}

fkd_status finish(fkd_tree h, const char* what, int mem) {
  if (mem == FKD_MEM_DEVICE && (h->flags & FKD_FLAG_ASYNC)) return FKD_OK;
  return check_err_word(h, what);
}

Table table_of(fkd_tree h) { return Table{h->nodes.as<uint4>(), h->ids.as<uint32_t>()}; }

// Makes the calling thread's current device the handle's for one call.
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess || prev == dev) prev = -1;
    else cudaSetDevice(dev);
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// One search call's slot and stream.  Device-memory calls run on the
// handle's stream (stream-ordered with the caller's work); host-memory calls
// are synchronous and run on the slot's own stream, so concurrent ones
// overlap on the GPU.  Every lease first waits for the slot's previous work
// and for the last build; release records the slot's completion event and
// returns it to the pool.
struct Lease {
  fkd_tree h = nullptr;
  SearchSlot* s = nullptr;
  cudaStream_t st = nullptr;
  ~Lease() {
    if (!s) return;
    cudaEventRecord(s->done, st);
    std::lock_guard<std::mutex> g(h->slot_mu);
    h->free_slots.push_back(s);
  }
};

fkd_status lease_slot(fkd_tree h, int mem, Lease* L) {
  SearchSlot* s = nullptr;
  {
    std::lock_guard<std::mutex> g(h->slot_mu);
    if (!h->free_slots.empty()) {
      s = h->free_slots.back();
      h->free_slots.pop_back();
    }
  }
  if (!s) {
    std::unique_ptr<SearchSlot> ns(new (std::nothrow) SearchSlot());
    if (!ns) return fail(FKD_ERR_NOMEM, "host allocation failed");
    FKD_CUDA(cudaStreamCreateWithFlags(&ns->own, cudaStreamNonBlocking));
    FKD_CUDA(cudaEventCreateWithFlags(&ns->done, cudaEventDisableTiming));
    FKD_CUDA(ns->err.ensure(sizeof(uint32_t) * 4));
    FKD_CUDA(ns->qctr.ensure(sizeof(uint32_t) * 4));
    FKD_CUDA(cudaMallocHost((void**)&ns->herr, sizeof(uint32_t) * 16));
    FKD_CUDA(cudaMemsetAsync(ns->err.p, 0, sizeof(uint32_t) * 4, ns->own));
    FKD_CUDA(cudaEventRecord(ns->done, ns->own));
    s = ns.get();
    std::lock_guard<std::mutex> g(h->slot_mu);
    h->slots.push_back(std::move(ns));
  }
  L->h = h;
  L->s = s;
  L->st = mem == FKD_MEM_DEVICE ? h->stream : s->own;
  FKD_CUDA(cudaStreamWaitEvent(L->st, s->done, 0));
  if (L->st != h->stream) FKD_CUDA(cudaStreamWaitEvent(L->st, h->built_ev, 0));
  return FKD_OK;
}

// Reads the slot's error word and clears it (an error latched by an earlier
// asynchronous call that used the slot is reported here too).
fkd_status check_slot_err(const Lease& L, const char* what) {
  FKD_CUDA(cudaMemcpyAsync(L.s->herr, L.s->err.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, L.st));
  FKD_CUDA(cudaMemsetAsync(L.s->err.p, 0, sizeof(uint32_t), L.st));
  FKD_CUDA(cudaStreamSynchronize(L.st));
  return status_from_err(*L.s->herr, what);
}

fkd_status finish_search(fkd_tree h, const Lease& L, const char* what, int mem) {
  if (mem == FKD_MEM_DEVICE && (h->flags & FKD_FLAG_ASYNC)) return FKD_OK;
  return check_slot_err(L, what);
}

__global__ void k_tables_out(uint32_t n, int dim, const uint4* __restrict__ nodes, float* __restrict__ tab) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint4 v = nodes[i];
  const uint32_t w[4] = {v.x, v.y, v.z, v.w};
  for (int c = 0; c < dim; ++c) tab[(uint64_t)c * n + i] = __uint_as_float(w[c]);
}

// Stages host boxes (or aliases device boxes).
fkd_status stage_boxes(fkd_tree h, const Lease& L, const float* mins, const float* maxs, uint64_t q, int mem,
                       Boxes* b) {
  b->q = q;
  b->stride = q;
  if (mem == FKD_MEM_DEVICE) {
    b->lo = mins;
    b->hi = maxs;
    return FKD_OK;
  }
  SearchSlot* s = L.s;
  const size_t bytes = (size_t)h->dim * q * sizeof(float);
  FKD_CUDA(s->qlo.ensure(bytes ? bytes : 4));
  FKD_CUDA(s->qhi.ensure(bytes ? bytes : 4));
  if (bytes) {
    FKD_CUDA(cudaMemcpyAsync(s->qlo.p, mins, bytes, cudaMemcpyHostToDevice, L.st));
    FKD_CUDA(cudaMemcpyAsync(s->qhi.p, maxs, bytes, cudaMemcpyHostToDevice, L.st));
  }
  b->lo = s->qlo.as<float>();
  b->hi = s->qhi.as<float>();
  return FKD_OK;
}

SearchCtx search_ctx(fkd_tree h, const Lease& L, const Boxes& b) {
  SearchCtx sc;
  memset(&sc, 0, sizeof sc);
  sc.g = make_geom((uint32_t)h->n);
  sc.tab = table_of(h);
  if ((h->search_bucket || h->search_bucket_grp) && h->ipts_valid) {
    sc.tab.ipts = h->ipts.as<uint4>();
    sc.tab.dids = h->dids.as<uint32_t>();
    sc.tab.dnode = h->dnode.as<uint32_t>();
    sc.bucket = h->search_bucket;
    sc.bucket_grp = h->search_bucket_grp;
  }
  sc.boxes = b;
  sc.qcounter = L.s->qctr.as<uint32_t>();
  sc.err = L.s->err.as<uint32_t>();
  sc.stream = L.st;
  sc.capacity = ~0ull;
  sc.lanes = h->search_lanes;
  return sc;
}

fkd_status check_search_args(fkd_tree h, const float* mins, const float* maxs, uint64_t q, int mem) {
  if (!h) return fail(FKD_ERR_ARG, "null handle");
  if (!h->built) return fail(FKD_ERR_STATE, "search before build");
  if (mem != FKD_MEM_HOST && mem != FKD_MEM_DEVICE) return fail(FKD_ERR_ARG, "mem must be FKD_MEM_HOST or FKD_MEM_DEVICE");
  if (q > 0xffffffffull) return fail(FKD_ERR_ARG, "at most 2^32-1 boxes per call");
  if (q && (!mins || !maxs)) return fail(FKD_ERR_ARG, "null box bounds");
  return FKD_OK;
}

// Boxes below this count are searched in the caller's order: a spatial order
// only pays when many boxes share the tree's cache lines.
constexpr uint64_t BOX_ORDER_MIN = 4096;

// Spatial processing order of the boxes (fkd_search.cu: launch_box_order).
fkd_status box_order(fkd_tree h, const Lease& L, const Boxes& b, const uint32_t** order) {
  *order = nullptr;
  if (!h->box_order || b.q < BOX_ORDER_MIN) return FKD_OK;
  FKD_CUDA(L.s->qorder.ensure(box_order_words(b.q) * sizeof(uint32_t)));
  uint32_t* o = nullptr;
  FKD_CUDA(launch_box_order(make_geom((uint32_t)h->n), table_of(h), b, h->dim, L.s->qorder.as<uint32_t>(), &o,
                            L.st));
  *order = o;
  return FKD_OK;
}

// count pass into dcounts (device)
// rec (optional): the run pool fields of a recording count pass
fkd_status count_pass(fkd_tree h, const Lease& L, const Boxes& b, uint32_t* dcounts, const uint32_t* order,
                      const SearchCtx* rec = nullptr) {
  SearchCtx sc = search_ctx(h, L, b);
  sc.counts = dcounts;
  sc.order = order;
  if (rec) {
    sc.pool_st = rec->pool_st;
    sc.pool_len = rec->pool_len;
    sc.pool_s = rec->pool_s;
    sc.pool_ctr = rec->pool_ctr;
    sc.pool_cap = rec->pool_cap;
    sc.pool_cap_s = rec->pool_cap_s;
    sc.brec = rec->brec;
    sc.brec_ctr = rec->brec_ctr;
    sc.brec_cap = rec->brec_cap;
    sc.flags = rec->flags;
    sc.flag_ctr = rec->flag_ctr;
    sc.rec_ids = rec->rec_ids;
    sc.bucket_runs = rec->bucket_runs;
  }
  FKD_CUDA(launch_search(sc, h->dim, SEARCH_COUNT));
  return FKD_OK;
}

// In-order id / heap-index tables of the current tree -- and, with leaf
// buckets on, the in-order copy of the nodes -- built once per tree by the
// first search that needs them; every caller's stream then waits for them.
fkd_status ensure_inorder(fkd_tree h, cudaStream_t st) {
  if (h->n == 0) return FKD_OK;
  {
    std::lock_guard<std::mutex> g(h->tree_mu);
    const bool want_ipts = h->search_bucket != 0 || h->search_bucket_grp != 0;
    if (!h->inorder_valid || (want_ipts && !h->ipts_valid)) {
      FKD_CUDA(h->dids.ensure(h->n * sizeof(uint32_t)));
      FKD_CUDA(h->dnode.ensure(h->n * sizeof(uint32_t)));
      Table t = table_of(h);
      t.dids = h->dids.as<uint32_t>();
      t.dnode = h->dnode.as<uint32_t>();
      if (want_ipts) {
        FKD_CUDA(h->ipts.ensure(h->n * sizeof(uint4)));
        t.ipts = h->ipts.as<uint4>();
      }
      FKD_CUDA(launch_inorder(make_geom((uint32_t)h->n), t, st));
      FKD_CUDA(cudaEventRecord(h->inorder_ev, st));
      h->inorder_valid = true;
      h->ipts_valid = want_ipts;
    }
  }
  FKD_CUDA(cudaStreamWaitEvent(st, h->inorder_ev, 0));
  return FKD_OK;
}

// The leaf-bucket scan's in-order tables, when it is on.
fkd_status ensure_buckets(fkd_tree h, cudaStream_t st) {
  return (h->search_bucket || h->search_bucket_grp) ? ensure_inorder(h, st) : FKD_OK;
}

// Subtree digests of the current tree (digest search), built once per tree.
fkd_status ensure_sdig(fkd_tree h, cudaStream_t st) {
  if (h->n == 0) return FKD_OK;
  {
    std::lock_guard<std::mutex> g(h->tree_mu);
    if (!h->sdig_valid) {
      FKD_CUDA(h->sdig.ensure(h->n * sizeof(unsigned long long)));
      Table t = table_of(h);
      t.sdig = h->sdig.as<unsigned long long>();
      FKD_CUDA(launch_subtree_digests(h->plan.evs, 1, (uint32_t)h->n, t, st));
      FKD_CUDA(cudaEventRecord(h->sdig_ev, st));
      h->sdig_valid = true;
    }
  }
  FKD_CUDA(cudaStreamWaitEvent(st, h->sdig_ev, 0));
  return FKD_OK;
}

}  // namespace

namespace fkd {
fkd_status capi_fail(fkd_status s, const std::string& msg) { return fail(s, msg); }
fkd_status capi_status_from_err(uint32_t e, const char* what) { return status_from_err(e, what); }
}  // namespace fkd

extern "C" {

const char* fkd_version(void) { return "fkdtree_b200 0.1 (sm_100a)"; }

uint64_t fkd_kernel_launches(void) { return launches_total(); }

const char* fkd_last_error(void) { return g_last_error.c_str(); }

void fkd_debug_fail_alloc(int32_t after) { __atomic_store_n(&fkd::g_fail_alloc, after < 0 ? -1 : after, __ATOMIC_RELAXED); }

fkd_status fkd_create(int dim, uint32_t flags, void* stream, fkd_tree* out) {
  if (!out) return fail(FKD_ERR_ARG, "null output handle pointer");
  *out = nullptr;
  if (dim < 1 || dim > 4) return fail(FKD_ERR_ARG, "dim must be 1..4");
  fkd_tree h = new (std::nothrow) fkd_tree_s();
  if (!h) return fail(FKD_ERR_NOMEM, "host allocation failed");
  h->dim = dim;
  h->flags = flags;
  h->stream = (cudaStream_t)stream;
  cudaError_t e = cudaGetDevice(&h->device);
  if (e == cudaSuccess) e = h->err.ensure(sizeof(uint32_t) * 4);
  if (e == cudaSuccess) e = h->qctr.ensure(sizeof(uint32_t) * 4);
  if (e == cudaSuccess) e = h->passflags.ensure(sizeof(uint32_t) * 64);
  if (e == cudaSuccess) e = h->lstats.ensure(4 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemsetAsync(h->lstats.p, 0, 4 * sizeof(unsigned long long), h->stream);
  if (e == cudaSuccess) e = cudaMallocHost((void**)&h->herr, sizeof(uint32_t) * 16);
  for (cudaEvent_t* ev : {&h->built_ev, &h->inorder_ev, &h->sdig_ev})
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->err.p, 0, sizeof(uint32_t), h->stream);
  if (e == cudaSuccess) e = cudaEventRecord(h->built_ev, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    delete h;
    return fail(e == cudaErrorMemoryAllocation ? FKD_ERR_NOMEM : FKD_ERR_CUDA,
                std::string("fkd_create: ") + cudaGetErrorString(e));
  }
  *out = h;
  g_last_error.clear();
  return FKD_OK;
}

fkd_status fkd_destroy(fkd_tree h) {
  if (!h) return FKD_OK;
  DeviceScope ds(h->device);
  cudaStreamSynchronize(h->stream);
  delete h;
  return FKD_OK;
}

fkd_status fkd_set_stream(fkd_tree h, void* stream) {
  if (!h) return fail(FKD_ERR_ARG, "null handle");
  h->stream = (cudaStream_t)stream;
  return FKD_OK;
}

}  // extern "C"

namespace {

// Points in the reference's FKDPoint<float, dim> layout (FKDPoint.h:102-103:
// dim coordinates then the id, (dim + 1) words per point) to the SoA records
// of the build (coordinate c of point i at soa[c*n + i], ids at soa[dim*n + i]).
__global__ void k_points_to_soa(const uint32_t* __restrict__ pts, uint64_t n, int dim, uint32_t* __restrict__ soa) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t* p = pts + i * (uint64_t)(dim + 1);
  for (int w = 0; w <= dim; ++w) soa[(uint64_t)w * n + i] = __ldg(p + w);
}

// fkd_build (coords + ids SoA) and fkd_build_points (AoS points) share this.
fkd_status build_impl(fkd_tree h, const float* coords, const uint32_t* ids, const void* points, uint64_t n,
                             int mem) {
  if (!h) return fail(FKD_ERR_ARG, "null handle");
  if (mem != FKD_MEM_HOST && mem != FKD_MEM_DEVICE) return fail(FKD_ERR_ARG, "mem must be FKD_MEM_HOST or FKD_MEM_DEVICE");
  if (n >= (1ull << 31)) return fail(FKD_ERR_ARG, "at most 2^31-1 points per tree");
  if (n && !points && (!coords || !ids)) return fail(FKD_ERR_ARG, "null coords or ids");
  DeviceScope ds(h->device);
  h->built = false;
  {
    std::lock_guard<std::mutex> g(h->tree_mu);
    h->sdig_valid = false;
    h->inorder_valid = false;
    h->ipts_valid = false;
  }
  h->n = n;
  if (n == 0) {
    h->built = true;
    FKD_CUDA(cudaEventRecord(h->built_ev, h->stream));
    return FKD_OK;
  }
  const int dim = h->dim;
  if (h->plan_n != n) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    PlanHost ph;
    const uint32_t n32 = (uint32_t)n, base0 = 0u;
    plan_build(&n32, &base0, 1, dim, h->hist_ctas ? h->hist_ctas : 4u * (uint32_t)sms, ph, h->subtree_size);
    // a failed upload leaves no plan: the next build must plan again
    h->plan_n = ~0ull;
    FKD_CUDA(h->plan.upload(ph, h->stream));
    h->plan_n = n;
  }
  const size_t rec_bytes = (size_t)(dim + 1) * n * sizeof(uint32_t);
  FKD_CUDA(h->nodes.ensure(n * sizeof(uint4)));
  FKD_CUDA(h->ids.ensure(n * sizeof(uint32_t)));
  FKD_CUDA(h->work1.ensure(rec_bytes));
  if (!h->plan.levels.empty()) {
    FKD_CUDA(h->work0.ensure(rec_bytes));
    FKD_CUDA(h->sel.ensure(sizeof(SegSel) * (size_t)h->plan.maxseg));
    FKD_CUDA(h->bnd.ensure(2 * sizeof(uint2) * (size_t)h->plan.maxseg));
    if (h->small_fix) FKD_CUDA(h->tiebuf.ensure((size_t)h->plan.maxseg * SMALL_CAP * (dim + 1) * sizeof(uint32_t)));
    const size_t gw = (size_t)h->plan.maxseg * HIST_BINS;
    FKD_CUDA(h->ghist.ensure(gw * sizeof(uint32_t)));
    FKD_CUDA(cudaMemsetAsync(h->ghist.p, 0, gw * sizeof(uint32_t), h->stream));
  }
  FKD_CUDA(cudaMemsetAsync(h->err.p, 0, sizeof(uint32_t), h->stream));
  BuildCtx bc;
  if (points) {
    uint32_t* w1 = h->work1.as<uint32_t>();
    const uint32_t* src = (const uint32_t*)points;
    if (mem == FKD_MEM_HOST) {
      FKD_CUDA(h->tmp.ensure(rec_bytes));
      FKD_CUDA(cudaMemcpyAsync(h->tmp.p, points, rec_bytes, cudaMemcpyHostToDevice, h->stream));
      src = h->tmp.as<uint32_t>();
    }
    k_points_to_soa<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(src, n, dim, w1);
    count_launches(1);
    FKD_CUDA(cudaGetLastError());
    bc.input = CSoA{w1, w1 + (size_t)dim * n, n};
  } else if (mem == FKD_MEM_HOST) {
    uint32_t* w1 = h->work1.as<uint32_t>();
    FKD_CUDA(cudaMemcpyAsync(w1, coords, (size_t)dim * n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    FKD_CUDA(cudaMemcpyAsync(w1 + (size_t)dim * n, ids, n * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
    bc.input = CSoA{w1, w1 + (size_t)dim * n, n};
  } else {
    bc.input = CSoA{(const uint32_t*)coords, ids, n};
  }
  uint32_t* w0 = h->work0.as<uint32_t>();
  uint32_t* w1 = h->work1.as<uint32_t>();
  bc.work[0] = SoA{w0, w0 ? w0 + (size_t)dim * n : nullptr, n};
  bc.work[1] = SoA{w1, w1 + (size_t)dim * n, n};
  bc.evs = h->plan.evs;
  bc.nlevels = (uint32_t)h->plan.levels.size();
  bc.levels = h->plan.levels.data();
  bc.subs = h->plan.subs;
  bc.nsub = h->plan.nsub;
  bc.sel = h->sel.as<SegSel>();
  bc.ghist = h->ghist.as<uint32_t>();
  bc.tab = table_of(h);
  bc.err = h->err.as<uint32_t>();
  bc.pending = h->passflags.as<uint32_t>();
  bc.bnd = h->plan.levels.empty() ? nullptr : h->bnd.as<uint2>();
  bc.tiebuf = (h->small_fix && !h->plan.levels.empty()) ? h->tiebuf.as<uint32_t>() : nullptr;
  bc.lin = h->lin_pass;
  bc.bnd_stride = h->plan.maxseg;
  bc.subtree = h->subtree;
  bc.subn = h->subtree_size;
  bc.small_select = h->small_select;
  bc.stream = h->stream;
  memset(&bc.learn, 0, sizeof bc.learn);
  bc.learn.stats = h->lstats.as<unsigned long long>();  // [3] counts the digit passes of every build
  if (h->mlp && !h->plan.levels.empty()) {
    const size_t ms = h->plan.maxseg;
    FKD_CUDA(h->lfeat.ensure(ms * FKD_MLP_FEATURES * sizeof(float)));
    FKD_CUDA(h->lyhat.ensure(ms * sizeof(float)));
    FKD_CUDA(h->lrange.ensure(ms * sizeof(float2)));
    FKD_CUDA(h->lstats.ensure(4 * sizeof(unsigned long long)));
    bc.learn.params = mlp_params(h->mlp);
    bc.learn.delta = h->mlp_delta;
    bc.learn.feat = h->lfeat.as<float>();
    bc.learn.yhat = h->lyhat.as<float>();
    bc.learn.range = h->lrange.as<float2>();
    bc.learn.stats = h->lstats.as<unsigned long long>();
  }
  const bool kt = !h->kev.empty();
  if (kt) {
    FKD_CUDA(cudaEventRecord(h->kev_at(h->kev_builds, 4), h->stream));
    bc.ev_sub = h->kev_at(h->kev_builds, 5);
  }
  FKD_CUDA(launch_build(bc, dim));
  if (kt) {
    FKD_CUDA(cudaEventRecord(h->kev_at(h->kev_builds, 6), h->stream));
    ++h->kev_builds;
  }
  FKD_CUDA(cudaEventRecord(h->built_ev, h->stream));
  h->built = true;
  fkd_status s = finish(h, points ? "fkd_build_points" : "fkd_build", mem);
  if (s != FKD_OK) h->built = false;
  return s;
}

}  // namespace

extern "C" {

fkd_status fkd_build(fkd_tree h, const float* coords, const uint32_t* ids, uint64_t n, int mem) {
  return build_impl(h, coords, ids, nullptr, n, mem);
}

fkd_status fkd_build_points(fkd_tree h, const void* points, uint64_t n, int mem) {
  if (n && !points) return fail(FKD_ERR_ARG, "null points");
  return build_impl(h, nullptr, nullptr, points, n, mem);
}

fkd_status fkd_size(fkd_tree h, uint64_t* n) {
  if (!h || !n) return fail(FKD_ERR_ARG, "null argument");
  *n = h->built ? h->n : 0;
  return FKD_OK;
}

fkd_status fkd_get_tables(fkd_tree h, float* tab, uint32_t* tab_ids, int mem) {
  if (!h) return fail(FKD_ERR_ARG, "null handle");
  if (!h->built) return fail(FKD_ERR_STATE, "tables requested before build");
  if (mem != FKD_MEM_HOST && mem != FKD_MEM_DEVICE) return fail(FKD_ERR_ARG, "mem must be FKD_MEM_HOST or FKD_MEM_DEVICE");
  const uint64_t n = h->n;
  if (n == 0) return FKD_OK;
  DeviceScope ds(h->device);
  std::lock_guard<std::mutex> g(h->tab_mu);
  if (tab) {
    float* dst = tab;
    if (mem == FKD_MEM_HOST) {
      FKD_CUDA(h->work0.ensure((size_t)(h->dim + 1) * n * sizeof(uint32_t)));
      dst = h->work0.as<float>();
    }
    k_tables_out<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>((uint32_t)n, h->dim, h->nodes.as<uint4>(), dst);
    count_launches(1);
    FKD_CUDA(cudaGetLastError());
    if (mem == FKD_MEM_HOST)
      FKD_CUDA(cudaMemcpyAsync(tab, dst, (size_t)h->dim * n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  }
  if (tab_ids)
    FKD_CUDA(cudaMemcpyAsync(tab_ids, h->ids.p, n * sizeof(uint32_t),
                             mem == FKD_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, h->stream));
  if (mem == FKD_MEM_HOST || !(h->flags & FKD_FLAG_ASYNC)) FKD_CUDA(cudaStreamSynchronize(h->stream));
  return FKD_OK;
}

fkd_status fkd_search_count(fkd_tree h, const float* mins, const float* maxs, uint64_t q, uint32_t* counts, int mem) {
  fkd_status s = check_search_args(h, mins, maxs, q, mem);
  if (s != FKD_OK) return s;
  if (q && !counts) return fail(FKD_ERR_ARG, "null counts");
  if (q == 0) return FKD_OK;
  DeviceScope ds(h->device);
  Lease L;
  if ((s = lease_slot(h, mem, &L)) != FKD_OK) return s;
  Boxes b;
  if ((s = stage_boxes(h, L, mins, maxs, q, mem, &b)) != FKD_OK) return s;
  uint32_t* dc = counts;
  if (mem == FKD_MEM_HOST) {
    FKD_CUDA(L.s->counts.ensure(q * sizeof(uint32_t)));
    dc = L.s->counts.as<uint32_t>();
  }
  if ((s = ensure_buckets(h, L.st)) != FKD_OK) return s;
  const uint32_t* order = nullptr;
  if ((s = box_order(h, L, b, &order)) != FKD_OK) return s;
  if ((s = count_pass(h, L, b, dc, order)) != FKD_OK) return s;
  if (mem == FKD_MEM_HOST)
    FKD_CUDA(cudaMemcpyAsync(counts, dc, q * sizeof(uint32_t), cudaMemcpyDeviceToHost, L.st));
  return finish_search(h, L, "fkd_search_count", mem);
}

}  // extern "C"

namespace {

// rec: the run pool the count pass filled (null: traverse every box); with
// it, k_expand writes the recorded runs and the traversal only revisits the
// nflag boxes whose runs did not fit.
fkd_status write_pass(fkd_tree h, const Lease& L, const Boxes& b, const uint64_t* doffsets, uint32_t* dout,
                      uint64_t total, int ordered, const uint32_t* order, const SearchCtx* rec = nullptr,
                      uint32_t nflag = 0) {
  fkd_status s0 = ensure_inorder(h, L.st);
  if (s0 != FKD_OK) return s0;
  SearchCtx sc = search_ctx(h, L, b);
  sc.tab.dids = h->dids.as<uint32_t>();
  sc.tab.dnode = h->dnode.as<uint32_t>();
  sc.order = order;
  sc.offsets = doffsets;
  sc.out = dout;
  sc.capacity = total;
  sc.heap_out = ordered ? 1 : 0;
  if (rec) {
    SearchCtx x = sc;
    x.pool_st = rec->pool_st;
    x.pool_len = rec->pool_len;
    x.pool_s = rec->pool_s;
    x.brec = rec->brec;
    x.brec_ctr = rec->brec_ctr;
    x.brec_cap = rec->brec_cap;
    x.rec_ids = rec->rec_ids;
    x.work_ctr = rec->work_ctr;
    FKD_CUDA(launch_expand(x));
    sc.order = rec->flags;
    sc.boxes.q = nflag;
  }
  if (sc.boxes.q) FKD_CUDA(launch_search(sc, h->dim, SEARCH_WRITE));
  if (ordered) {
    FKD_CUDA(L.s->tmp.ensure(total ? total * sizeof(uint32_t) : 4));
    FKD_CUDA(launch_order_results(sc.g, sc.tab, doffsets, b.q, dout, L.s->tmp.as<uint32_t>(), sc.err, L.st));
  }
  return FKD_OK;
}

}  // namespace

extern "C" {

fkd_status fkd_search_write(fkd_tree h, const float* mins, const float* maxs, uint64_t q, const uint64_t* offsets,
                            uint32_t* ids_out, int ordered, int mem) {
  fkd_status s = check_search_args(h, mins, maxs, q, mem);
  if (s != FKD_OK) return s;
  if (!offsets) return fail(FKD_ERR_ARG, "null offsets");
  if (q == 0) return FKD_OK;
  DeviceScope ds(h->device);
  Lease L;
  if ((s = lease_slot(h, mem, &L)) != FKD_OK) return s;
  SearchSlot* sl = L.s;
  Boxes b;
  if ((s = stage_boxes(h, L, mins, maxs, q, mem, &b)) != FKD_OK) return s;
  const uint64_t* doff = offsets;
  uint32_t* dout = ids_out;
  uint64_t total = 0;
  if (mem == FKD_MEM_HOST) {
    total = offsets[q];
    if (total && !ids_out) return fail(FKD_ERR_ARG, "null ids_out");
    FKD_CUDA(sl->offsets.ensure((q + 1) * sizeof(uint64_t)));
    FKD_CUDA(cudaMemcpyAsync(sl->offsets.p, offsets, (q + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, L.st));
    doff = sl->offsets.as<uint64_t>();
    FKD_CUDA(sl->out.ensure(total ? total * sizeof(uint32_t) : 4));
    dout = sl->out.as<uint32_t>();
  } else {
    FKD_CUDA(cudaMemcpyAsync(sl->herr + 2, offsets + q, sizeof(uint64_t), cudaMemcpyDeviceToHost, L.st));
    FKD_CUDA(cudaStreamSynchronize(L.st));
    memcpy(&total, sl->herr + 2, sizeof(uint64_t));
    if (total && !ids_out) return fail(FKD_ERR_ARG, "null ids_out");
  }
  const uint32_t* order = nullptr;
  if ((s = box_order(h, L, b, &order)) != FKD_OK) return s;
  if ((s = write_pass(h, L, b, doff, dout, total, ordered, order)) != FKD_OK) return s;
  if (mem == FKD_MEM_HOST && total)
    FKD_CUDA(cudaMemcpyAsync(ids_out, dout, total * sizeof(uint32_t), cudaMemcpyDeviceToHost, L.st));
  return finish_search(h, L, "fkd_search_write", mem);
}

}  // extern "C"

namespace {

// fkd_search of one host-memory box (the drop-in's search_in_the_box): one
// launch of k_one, one copy back of its count and first ids, one wait -- in
// place of staging, count pass, scan, write pass and their two waits.  Its
// list is the level-order one (ascending heap index), which serves ordered
// and unordered calls alike.  Sets *general (returning FKD_OK, outputs
// untouched) when the general path must answer instead: a NaN bound (whose
// meaning the general path defines), a frontier too wide for the warp, or
// more results than its buffer holds.
constexpr uint32_t ONE_CAP = 1u << 16;   // ids k_one writes
constexpr uint32_t ONE_FIRST = 1024;     // ids copied back with the count
fkd_status search_one(fkd_tree h, const float* mins, const float* maxs, uint64_t* offsets_out, uint32_t* ids_out,
                      uint64_t capacity, uint64_t* total, bool* general) {
  *general = false;
  OneBox bx;
  for (int c = 0; c < 4; ++c) bx.lo[c] = bx.hi[c] = 0.f;
  for (int c = 0; c < h->dim; ++c) {
    if (mins[c] != mins[c] || maxs[c] != maxs[c]) {
      *general = true;
      return FKD_OK;
    }
    bx.lo[c] = mins[c];
    bx.hi[c] = maxs[c];
  }
  DeviceScope ds(h->device);
  Lease L;
  fkd_status s = lease_slot(h, FKD_MEM_HOST, &L);
  if (s != FKD_OK) return s;
  SearchSlot* sl = L.s;
  FKD_CUDA(sl->one.ensure((4 + ONE_CAP) * sizeof(uint32_t)));
  if (!sl->hone) FKD_CUDA(cudaMallocHost((void**)&sl->hone, (4 + ONE_FIRST) * sizeof(uint32_t)));
  const uint32_t cap = (uint32_t)std::min<uint64_t>(capacity, ONE_CAP);
  const uint32_t first = std::min(cap, ONE_FIRST);
  FKD_CUDA(launch_one(table_of(h), (uint32_t)h->n, h->dim, bx, sl->one.as<uint32_t>(), cap, L.st));
  FKD_CUDA(cudaMemcpyAsync(sl->hone, sl->one.p, (4 + first) * sizeof(uint32_t), cudaMemcpyDeviceToHost, L.st));
  FKD_CUDA(cudaStreamSynchronize(L.st));
  const uint64_t tot = sl->hone[0];
  if (sl->hone[1] || (tot > cap && tot <= capacity)) {
    *general = true;
    return FKD_OK;
  }
  offsets_out[0] = 0;
  offsets_out[1] = tot;
  *total = tot;
  if (tot > capacity) {
    char buf[128];
    snprintf(buf, sizeof buf, "fkd_search: %llu results exceed the capacity of %llu ids", (unsigned long long)tot,
             (unsigned long long)capacity);
    return fail(FKD_ERR_CAPACITY, buf);
  }
  if (tot && !ids_out) return fail(FKD_ERR_ARG, "null ids_out");
  memcpy(ids_out, sl->hone + 4, std::min<uint64_t>(tot, first) * sizeof(uint32_t));
  if (tot > first) {
    FKD_CUDA(cudaMemcpyAsync(ids_out + first, sl->one.as<uint32_t>() + 4 + first, (tot - first) * sizeof(uint32_t),
                             cudaMemcpyDeviceToHost, L.st));
    FKD_CUDA(cudaStreamSynchronize(L.st));
  }
  return FKD_OK;
}

}  // namespace

extern "C" {

fkd_status fkd_search(fkd_tree h, const float* mins, const float* maxs, uint64_t q, uint64_t* offsets_out,
                      uint32_t* ids_out, uint64_t capacity, uint64_t* total, int ordered, int mem) {
  fkd_status s = check_search_args(h, mins, maxs, q, mem);
  if (s != FKD_OK) return s;
  if (!offsets_out || !total) return fail(FKD_ERR_ARG, "null offsets_out or total");
  if (q == 1 && mem == FKD_MEM_HOST && h->search_one && h->n <= 0xffffffffull) {
    bool general = false;
    s = search_one(h, mins, maxs, offsets_out, ids_out, capacity, total, &general);
    if (s != FKD_OK || !general) return s;
  }
  DeviceScope ds(h->device);
  Lease L;
  if ((s = lease_slot(h, mem, &L)) != FKD_OK) return s;
  SearchSlot* sl = L.s;
  const cudaStream_t st = L.st;
  Boxes b;
  if ((s = stage_boxes(h, L, mins, maxs, q, mem, &b)) != FKD_OK) return s;
  FKD_CUDA(sl->counts.ensure(q ? q * sizeof(uint32_t) : 4));
  FKD_CUDA(sl->partials.ensure(scan_partials_words(q) * sizeof(unsigned long long)));
  uint64_t* doff = offsets_out;
  if (mem == FKD_MEM_HOST) {
    FKD_CUDA(sl->offsets.ensure((q + 1) * sizeof(uint64_t)));
    doff = sl->offsets.as<uint64_t>();
  }
  const uint32_t* order = nullptr;
  if (q && (s = box_order(h, L, b, &order)) != FKD_OK) return s;
  if ((s = ensure_inorder(h, st)) != FKD_OK) return s;
  // per-kernel events only for calls on the handle's stream (a benchmark's
  // single-threaded loop); the ring is not shared between threads
  const bool kt = !h->kev.empty() && st == h->stream;
  if (kt) FKD_CUDA(cudaEventRecord(h->kev_at(h->kev_searches, 0), st));
  // The count pass records every box's result as runs of the in-order table
  // (fkd_search.cu: k_search, k_expand) into a pool sized by the previous
  // call's demand; boxes that do not fit are traversed again by the write pass.
  SearchCtx rec;
  memset(&rec, 0, sizeof rec);
  bool rec_on = q > 0 && h->search_record && (h->search_lanes == 0 || h->search_lanes == 32);
  if (rec_on) {
    uint64_t pw = sl->pool_want ? sl->pool_want : 64 * q + (1u << 22);
    uint64_t sw = sl->pool_s_want ? sl->pool_s_want : 256 * q + (1u << 22);
    if (h->search_pool) pw = sw = h->search_pool;
    if (pw > 0xffffffffull) pw = 0xffffffffull;
    if (sw > 0xffffffffull) sw = 0xffffffffull;
    const uint64_t bw = sl->brec_want ? sl->brec_want : q + (1u << 16);
    cudaError_t ae = sl->pool_st.ensure(pw * sizeof(uint32_t));
    if (ae == cudaSuccess) ae = sl->pool_len.ensure(pw * sizeof(uint32_t));
    if (ae == cudaSuccess) ae = sl->pool_s.ensure(sw * sizeof(uint32_t));
    if (ae == cudaSuccess) ae = sl->brec.ensure(2 * bw * sizeof(uint4));
    if (ae == cudaSuccess) ae = sl->rflags.ensure(q * sizeof(uint32_t));
    if (ae == cudaSuccess) ae = sl->jctr.ensure(8 * sizeof(unsigned long long));
    if (ae != cudaSuccess) {
      // no room for the pool: traverse twice
      (void)cudaGetLastError();
      sl->pool_st.release();
      sl->pool_len.release();
      sl->pool_s.release();
      sl->brec.release();
      sl->pool_want = sl->pool_s_want = sl->brec_want = 0;
      rec_on = false;
    } else {
      FKD_CUDA(cudaMemsetAsync(sl->jctr.p, 0, 8 * sizeof(unsigned long long), st));
      // chunk records are reserved in blocks; the unused tail of a block must read as empty
      FKD_CUDA(cudaMemsetAsync(sl->brec.p, 0, sl->brec.bytes, st));
      unsigned long long* ctr = sl->jctr.as<unsigned long long>();
      rec.pool_st = sl->pool_st.as<uint32_t>();
      rec.pool_len = sl->pool_len.as<uint32_t>();
      rec.pool_s = sl->pool_s.as<uint32_t>();
      rec.pool_ctr = ctr;  // [0] runs, [1] singles
      rec.pool_cap = sl->pool_st.bytes / sizeof(uint32_t);
      rec.pool_cap_s = sl->pool_s.bytes / sizeof(uint32_t);
      rec.brec = sl->brec.as<uint4>();
      rec.brec_ctr = ctr + 2;
      rec.brec_cap = sl->brec.bytes / (2 * sizeof(uint4));
      rec.flags = sl->rflags.as<uint32_t>();
      rec.flag_ctr = (uint32_t*)(ctr + 3);
      rec.work_ctr = ctr + 4;  // the write pass's record counter
      rec.rec_ids = ordered ? 0 : 1;  // unordered: singles carry their ids, the write pass copies them
      rec.bucket_runs = h->bucket_runs ? 1 : 0;
    }
  }
  if (q && (s = count_pass(h, L, b, sl->counts.as<uint32_t>(), order, rec_on ? &rec : nullptr)) != FKD_OK) return s;
  if (kt) FKD_CUDA(cudaEventRecord(h->kev_at(h->kev_searches, 1), st));
  FKD_CUDA(launch_scan_counts(sl->counts.as<uint32_t>(), q, doff, sl->partials.as<unsigned long long>(), st));
  FKD_CUDA(cudaMemcpyAsync(sl->herr + 2, doff + q, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  if (rec_on) FKD_CUDA(cudaMemcpyAsync(sl->herr + 4, sl->jctr.p, 4 * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  FKD_CUDA(cudaStreamSynchronize(st));
  uint64_t tot = 0;
  memcpy(&tot, sl->herr + 2, sizeof(uint64_t));
  uint32_t nflag = 0;
  if (rec_on) {
    uint64_t dem[4];
    memcpy(dem, sl->herr + 4, sizeof dem);
    nflag = (uint32_t)dem[3];
    // the next call's pools hold this call's demand with room to spare
    if (!h->search_pool) sl->pool_want = std::max<uint64_t>(sl->pool_want, dem[0] + dem[0] / 4 + (1u << 22));
    if (!h->search_pool) sl->pool_s_want = std::max<uint64_t>(sl->pool_s_want, dem[1] + dem[1] / 4 + (1u << 22));
    sl->brec_want = std::max<uint64_t>(sl->brec_want, dem[2] + dem[2] / 4 + (1u << 16));
  }
  *total = tot;
  if ((s = check_slot_err(L, "fkd_search (count)")) != FKD_OK) return s;
  if (mem == FKD_MEM_HOST)
    FKD_CUDA(cudaMemcpyAsync(offsets_out, doff, (q + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  if (tot > capacity) {
    FKD_CUDA(cudaStreamSynchronize(st));
    char buf[128];
    snprintf(buf, sizeof buf, "fkd_search: %llu results exceed the capacity of %llu ids", (unsigned long long)tot,
             (unsigned long long)capacity);
    return fail(FKD_ERR_CAPACITY, buf);
  }
  if (tot && !ids_out) return fail(FKD_ERR_ARG, "null ids_out");
  if (tot == 0) {
    if (kt) {
      FKD_CUDA(cudaEventRecord(h->kev_at(h->kev_searches, 2), st));
      FKD_CUDA(cudaEventRecord(h->kev_at(h->kev_searches, 3), st));
      ++h->kev_searches;
    }
    FKD_CUDA(cudaStreamSynchronize(st));
    return FKD_OK;
  }
  uint32_t* dout = ids_out;
  if (mem == FKD_MEM_HOST) {
    FKD_CUDA(sl->out.ensure(tot * sizeof(uint32_t)));
    dout = sl->out.as<uint32_t>();
  }
  if (kt) FKD_CUDA(cudaEventRecord(h->kev_at(h->kev_searches, 2), st));
  if ((s = write_pass(h, L, b, doff, dout, tot, ordered, order, rec_on ? &rec : nullptr, nflag)) != FKD_OK) return s;
  if (kt) {
    FKD_CUDA(cudaEventRecord(h->kev_at(h->kev_searches, 3), st));
    ++h->kev_searches;
  }
  if (mem == FKD_MEM_HOST)
    FKD_CUDA(cudaMemcpyAsync(ids_out, dout, tot * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  return finish_search(h, L, "fkd_search", mem);
}

fkd_status fkd_search_digest(fkd_tree h, const float* mins, const float* maxs, uint64_t q, uint32_t* counts,
                             uint64_t* digests, int mem) {
  fkd_status s = check_search_args(h, mins, maxs, q, mem);
  if (s != FKD_OK) return s;
  if (q && (!counts || !digests)) return fail(FKD_ERR_ARG, "null counts or digests");
  if (q == 0) return FKD_OK;
  DeviceScope ds(h->device);
  Lease L;
  if ((s = lease_slot(h, mem, &L)) != FKD_OK) return s;
  Boxes b;
  if ((s = stage_boxes(h, L, mins, maxs, q, mem, &b)) != FKD_OK) return s;
  uint32_t* dc = counts;
  uint64_t* dd = digests;
  if (mem == FKD_MEM_HOST) {
    FKD_CUDA(L.s->counts.ensure(q * sizeof(uint32_t)));
    FKD_CUDA(L.s->digests.ensure(q * sizeof(uint64_t)));
    dc = L.s->counts.as<uint32_t>();
    dd = L.s->digests.as<uint64_t>();
  }
  if ((s = ensure_sdig(h, L.st)) != FKD_OK) return s;
  if ((s = ensure_buckets(h, L.st)) != FKD_OK) return s;
  const uint32_t* order = nullptr;
  if ((s = box_order(h, L, b, &order)) != FKD_OK) return s;
  SearchCtx sc = search_ctx(h, L, b);
  sc.tab.sdig = h->sdig.as<unsigned long long>();
  sc.order = order;
  sc.counts = dc;
  sc.digests = (unsigned long long*)dd;
  FKD_CUDA(launch_search(sc, h->dim, SEARCH_DIGEST));
  if (mem == FKD_MEM_HOST) {
    FKD_CUDA(cudaMemcpyAsync(counts, dc, q * sizeof(uint32_t), cudaMemcpyDeviceToHost, L.st));
    FKD_CUDA(cudaMemcpyAsync(digests, dd, q * sizeof(uint64_t), cudaMemcpyDeviceToHost, L.st));
  }
  return finish_search(h, L, "fkd_search_digest", mem);
}

}  // extern "C"

namespace {

fkd_status check_nn_args(fkd_tree h, const float* centers, uint64_t q, int mem) {
  if (!h) return fail(FKD_ERR_ARG, "null handle");
  if (!h->built) return fail(FKD_ERR_STATE, "search before build");
  if (mem != FKD_MEM_HOST && mem != FKD_MEM_DEVICE) return fail(FKD_ERR_ARG, "mem must be FKD_MEM_HOST or FKD_MEM_DEVICE");
  if (q > 0xffffffffull) return fail(FKD_ERR_ARG, "at most 2^32-1 queries per call");
  if (q && !centers) return fail(FKD_ERR_ARG, "null centers");
  return FKD_OK;
}

// Stages host centres (dim*q SoA) and radii (q, optional) or aliases device ones.
fkd_status stage_centres(fkd_tree h, const Lease& L, const float* centers, const float* radii, uint64_t q, int mem,
                         const float** dctr, const float** drad) {
  if (mem == FKD_MEM_DEVICE) {
    *dctr = centers;
    if (drad) *drad = radii;
    return FKD_OK;
  }
  SearchSlot* s = L.s;
  const size_t cb = (size_t)h->dim * q * sizeof(float);
  FKD_CUDA(s->qlo.ensure(cb ? cb : 4));
  if (cb) FKD_CUDA(cudaMemcpyAsync(s->qlo.p, centers, cb, cudaMemcpyHostToDevice, L.st));
  *dctr = s->qlo.as<float>();
  if (drad) {
    FKD_CUDA(s->qhi.ensure(q ? q * sizeof(float) : 4));
    if (q) FKD_CUDA(cudaMemcpyAsync(s->qhi.p, radii, q * sizeof(float), cudaMemcpyHostToDevice, L.st));
    *drad = s->qhi.as<float>();
  }
  return FKD_OK;
}

// Spatial order of the query centres (the box order of zero-size boxes).
fkd_status centre_order(fkd_tree h, const Lease& L, const float* dctr, uint64_t q, const uint32_t** order) {
  Boxes b;
  b.lo = dctr;
  b.hi = dctr;
  b.stride = q;
  b.q = q;
  return box_order(h, L, b, order);
}

}  // namespace

extern "C" {

fkd_status fkd_search_radius_count(fkd_tree h, const float* centers, const float* radii, uint64_t q,
                                   uint32_t* counts, int mem) {
  fkd_status s = check_nn_args(h, centers, q, mem);
  if (s != FKD_OK) return s;
  if (q && (!radii || !counts)) return fail(FKD_ERR_ARG, "null radii or counts");
  if (q == 0) return FKD_OK;
  DeviceScope ds(h->device);
  Lease L;
  if ((s = lease_slot(h, mem, &L)) != FKD_OK) return s;
  const float *dctr = nullptr, *drad = nullptr;
  if ((s = stage_centres(h, L, centers, radii, q, mem, &dctr, &drad)) != FKD_OK) return s;
  uint32_t* dc = counts;
  if (mem == FKD_MEM_HOST) {
    FKD_CUDA(L.s->counts.ensure(q * sizeof(uint32_t)));
    dc = L.s->counts.as<uint32_t>();
  }
  const uint32_t* order = nullptr;
  if ((s = centre_order(h, L, dctr, q, &order)) != FKD_OK) return s;
  FKD_CUDA(launch_radius(make_geom((uint32_t)h->n), table_of(h), dctr, drad, q, order, dc, nullptr, nullptr, 0,
                         L.s->err.as<uint32_t>(), h->dim, L.st));
  if (mem == FKD_MEM_HOST)
    FKD_CUDA(cudaMemcpyAsync(counts, dc, q * sizeof(uint32_t), cudaMemcpyDeviceToHost, L.st));
  return finish_search(h, L, "fkd_search_radius_count", mem);
}

fkd_status fkd_search_radius(fkd_tree h, const float* centers, const float* radii, uint64_t q, uint64_t* offsets_out,
                             uint32_t* ids_out, uint64_t capacity, uint64_t* total, int ordered, int mem) {
  fkd_status s = check_nn_args(h, centers, q, mem);
  if (s != FKD_OK) return s;
  if (!offsets_out || !total) return fail(FKD_ERR_ARG, "null offsets_out or total");
  if (q && !radii) return fail(FKD_ERR_ARG, "null radii");
  DeviceScope ds(h->device);
  Lease L;
  if ((s = lease_slot(h, mem, &L)) != FKD_OK) return s;
  SearchSlot* sl = L.s;
  const cudaStream_t st = L.st;
  const float *dctr = nullptr, *drad = nullptr;
  if ((s = stage_centres(h, L, centers, radii, q, mem, &dctr, &drad)) != FKD_OK) return s;
  FKD_CUDA(sl->counts.ensure(q ? q * sizeof(uint32_t) : 4));
  FKD_CUDA(sl->partials.ensure(scan_partials_words(q) * sizeof(unsigned long long)));
  uint64_t* doff = offsets_out;
  if (mem == FKD_MEM_HOST) {
    FKD_CUDA(sl->offsets.ensure((q + 1) * sizeof(uint64_t)));
    doff = sl->offsets.as<uint64_t>();
  }
  const uint32_t* order = nullptr;
  if (q && (s = centre_order(h, L, dctr, q, &order)) != FKD_OK) return s;
  const Geom g = make_geom((uint32_t)h->n);
  const Table tab = table_of(h);
  uint32_t* err = sl->err.as<uint32_t>();
  FKD_CUDA(launch_radius(g, tab, dctr, drad, q, order, sl->counts.as<uint32_t>(), nullptr, nullptr, 0, err, h->dim,
                         st));
  FKD_CUDA(launch_scan_counts(sl->counts.as<uint32_t>(), q, doff, sl->partials.as<unsigned long long>(), st));
  FKD_CUDA(cudaMemcpyAsync(sl->herr + 2, doff + q, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  FKD_CUDA(cudaStreamSynchronize(st));
  uint64_t tot = 0;
  memcpy(&tot, sl->herr + 2, sizeof(uint64_t));
  *total = tot;
  if ((s = check_slot_err(L, "fkd_search_radius (count)")) != FKD_OK) return s;
  if (mem == FKD_MEM_HOST)
    FKD_CUDA(cudaMemcpyAsync(offsets_out, doff, (q + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  if (tot > capacity) {
    FKD_CUDA(cudaStreamSynchronize(st));
    char buf[128];
    snprintf(buf, sizeof buf, "fkd_search_radius: %llu results exceed the capacity of %llu ids",
             (unsigned long long)tot, (unsigned long long)capacity);
    return fail(FKD_ERR_CAPACITY, buf);
  }
  if (tot && !ids_out) return fail(FKD_ERR_ARG, "null ids_out");
  if (tot == 0) {
    FKD_CUDA(cudaStreamSynchronize(st));
    return FKD_OK;
  }
  uint32_t* dout = ids_out;
  if (mem == FKD_MEM_HOST) {
    FKD_CUDA(sl->out.ensure(tot * sizeof(uint32_t)));
    dout = sl->out.as<uint32_t>();
  }
  // ordered: the write pass emits heap indices that k_order sorts and maps to ids
  FKD_CUDA(launch_radius(g, tab, dctr, drad, q, order, nullptr, doff, dout, ordered ? 1 : 0, err, h->dim, st));
  if (ordered) {
    FKD_CUDA(sl->tmp.ensure(tot * sizeof(uint32_t)));
    FKD_CUDA(launch_order_results(g, tab, doff, q, dout, sl->tmp.as<uint32_t>(), err, st));
  }
  if (mem == FKD_MEM_HOST)
    FKD_CUDA(cudaMemcpyAsync(ids_out, dout, tot * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  return finish_search(h, L, "fkd_search_radius", mem);
}

uint32_t fkd_knn_max_k(void) { return KNN_MAX; }

fkd_status fkd_search_knn(fkd_tree h, const float* centers, uint64_t q, uint32_t k, uint32_t* ids_out,
                          float* dist2_out, int mem) {
  fkd_status s = check_nn_args(h, centers, q, mem);
  if (s != FKD_OK) return s;
  if (k < 1 || k > KNN_MAX) return fail(FKD_ERR_ARG, "k must be 1..fkd_knn_max_k()");
  if (q && !ids_out) return fail(FKD_ERR_ARG, "null ids_out");
  if (q == 0) return FKD_OK;
  DeviceScope ds(h->device);
  Lease L;
  if ((s = lease_slot(h, mem, &L)) != FKD_OK) return s;
  SearchSlot* sl = L.s;
  const float* dctr = nullptr;
  if ((s = stage_centres(h, L, centers, nullptr, q, mem, &dctr, nullptr)) != FKD_OK) return s;
  const uint64_t cells = q * (uint64_t)k;
  uint32_t* di = ids_out;
  float* dd = dist2_out;
  if (mem == FKD_MEM_HOST) {
    FKD_CUDA(sl->out.ensure(cells * sizeof(uint32_t)));
    di = sl->out.as<uint32_t>();
    if (dist2_out) {
      FKD_CUDA(sl->tmp.ensure(cells * sizeof(float)));
      dd = sl->tmp.as<float>();
    }
  }
  const uint32_t* order = nullptr;
  if ((s = centre_order(h, L, dctr, q, &order)) != FKD_OK) return s;
  FKD_CUDA(launch_knn(make_geom((uint32_t)h->n), table_of(h), dctr, q, order, k, di, dd, sl->err.as<uint32_t>(),
                      h->dim, L.st));
  if (mem == FKD_MEM_HOST) {
    FKD_CUDA(cudaMemcpyAsync(ids_out, di, cells * sizeof(uint32_t), cudaMemcpyDeviceToHost, L.st));
    if (dist2_out) FKD_CUDA(cudaMemcpyAsync(dist2_out, dd, cells * sizeof(float), cudaMemcpyDeviceToHost, L.st));
  }
  return finish_search(h, L, "fkd_search_knn", mem);
}

fkd_status fkd_set_param(fkd_tree h, const char* name, int64_t value) {
  if (!h || !name) return fail(FKD_ERR_ARG, "null argument");
  if (strcmp(name, "hist_ctas") == 0) {
    if (value < 0 || value > (1 << 20)) return fail(FKD_ERR_ARG, "hist_ctas out of range");
    h->hist_ctas = (uint32_t)value;
    h->plan_n = ~0ull;  // re-plan at the next build
    return FKD_OK;
  }
  if (strcmp(name, "search_lanes") == 0) {
    if (value != 0 && value != 1 && value != 2 && value != 4 && value != 8 && value != 16 && value != 32)
      return fail(FKD_ERR_ARG, "search_lanes must be 0, 1, 2, 4, 8, 16 or 32");
    h->search_lanes = (uint32_t)value;
    return FKD_OK;
  }
  if (strcmp(name, "box_order") == 0) {
    if (value != 0 && value != 1) return fail(FKD_ERR_ARG, "box_order must be 0 or 1");
    h->box_order = value != 0;
    return FKD_OK;
  }
  if (strcmp(name, "small_select") == 0) {
    if (value != 0 && value != 1) return fail(FKD_ERR_ARG, "small_select must be 0 or 1");
    h->small_select = value != 0;
    return FKD_OK;
  }
  if (strcmp(name, "subtree") == 0) {
    if (value < 0 || value > 2) return fail(FKD_ERR_ARG, "subtree must be 0, 1 or 2");
    h->subtree = (int)value;
    return FKD_OK;
  }
  if (strcmp(name, "subtree_size") == 0) {
    if (value != 0 && value != 512 && value != 1024) return fail(FKD_ERR_ARG, "subtree_size must be 0, 512 or 1024");
    h->subtree_size = (int)value;
    h->plan_n = ~0ull;  // re-plan at the next build
    return FKD_OK;
  }
  if (strcmp(name, "small_fix") == 0) {
    if (value != 0 && value != 1) return fail(FKD_ERR_ARG, "small_fix must be 0 or 1");
    h->small_fix = value != 0;
    return FKD_OK;
  }
  if (strcmp(name, "lin_pass") == 0) {
    if (value != 0 && value != 1) return fail(FKD_ERR_ARG, "lin_pass must be 0 or 1");
    h->lin_pass = value != 0;
    return FKD_OK;
  }
  if (strcmp(name, "search_bucket") == 0) {
    if (value < 0 || value > (int64_t)BUCKET_MAX) return fail(FKD_ERR_ARG, "search_bucket must be 0..6");
    h->search_bucket = (uint32_t)value;
    return FKD_OK;
  }
  if (strcmp(name, "bucket_runs") == 0) {
    if (value != 0 && value != 1) return fail(FKD_ERR_ARG, "bucket_runs must be 0 or 1");
    h->bucket_runs = value != 0;
    return FKD_OK;
  }
  if (strcmp(name, "search_bucket_lanes") == 0) {
    if (value < 0 || value > 3) return fail(FKD_ERR_ARG, "search_bucket_lanes must be 0..3");
    h->search_bucket_grp = (uint32_t)value;
    return FKD_OK;
  }
  if (strcmp(name, "search_record") == 0) {
    if (value != 0 && value != 1) return fail(FKD_ERR_ARG, "search_record must be 0 or 1");
    h->search_record = value != 0;
    return FKD_OK;
  }
  if (strcmp(name, "search_one") == 0) {
    if (value != 0 && value != 1) return fail(FKD_ERR_ARG, "search_one must be 0 or 1");
    h->search_one = value != 0;
    return FKD_OK;
  }
  if (strcmp(name, "search_pool") == 0) {
    if (value < 0 || value > 0xffffffffll) return fail(FKD_ERR_ARG, "search_pool out of range");
    h->search_pool = (uint64_t)value;
    return FKD_OK;
  }
  if (strcmp(name, "kernel_events") == 0) {
    if (value != 0 && value != 1) return fail(FKD_ERR_ARG, "kernel_events must be 0 or 1");
    FKD_CUDA(cudaStreamSynchronize(h->stream));
    for (cudaEvent_t e : h->kev) cudaEventDestroy(e);
    h->kev.clear();
    h->kev_builds = h->kev_searches = 0;
    if (value) {
      FKD_CUDA(cudaSetDevice(h->device));
      h->kev.resize((size_t)fkd_tree_s::KEV_RING * 7, nullptr);
      for (cudaEvent_t& e : h->kev) {
        cudaError_t ce = cudaEventCreate(&e);
        if (ce != cudaSuccess) {
          e = nullptr;
          for (cudaEvent_t x : h->kev)
            if (x) cudaEventDestroy(x);
          h->kev.clear();
          return fail(FKD_ERR_CUDA, std::string("kernel_events: ") + cudaGetErrorString(ce));
        }
      }
    }
    return FKD_OK;
  }
  return fail(FKD_ERR_ARG, std::string("unknown parameter ") + name);
}

fkd_status fkd_kernel_times(fkd_tree h, uint32_t back, float* ms) {
  if (!h || !ms) return fail(FKD_ERR_ARG, "null argument");
  if (h->kev.empty()) return fail(FKD_ERR_STATE, "kernel_events is off");
  float v[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  if (back < fkd_tree_s::KEV_RING && back < h->kev_searches) {
    const uint64_t c = h->kev_searches - 1 - back;
    FKD_CUDA(cudaEventSynchronize(h->kev_at(c, 3)));
    FKD_CUDA(cudaEventElapsedTime(&v[0], h->kev_at(c, 0), h->kev_at(c, 1)));
    FKD_CUDA(cudaEventElapsedTime(&v[1], h->kev_at(c, 2), h->kev_at(c, 3)));
  }
  if (back < fkd_tree_s::KEV_RING && back < h->kev_builds) {
    const uint64_t c = h->kev_builds - 1 - back;
    FKD_CUDA(cudaEventSynchronize(h->kev_at(c, 6)));
    FKD_CUDA(cudaEventElapsedTime(&v[2], h->kev_at(c, 4), h->kev_at(c, 6)));
    FKD_CUDA(cudaEventElapsedTime(&v[3], h->kev_at(c, 4), h->kev_at(c, 5)));
    FKD_CUDA(cudaEventElapsedTime(&v[4], h->kev_at(c, 5), h->kev_at(c, 6)));
  }
  memcpy(ms, v, sizeof v);
  return FKD_OK;
}

fkd_status fkd_set_mlp(fkd_tree h, fkd_mlp m, float delta) {
  if (!h) return fail(FKD_ERR_ARG, "null handle");
  if (m && !(delta > 0.f)) return fail(FKD_ERR_ARG, "delta must be positive");
  h->mlp = m;
  h->mlp_delta = delta;
  if (m) {
    FKD_CUDA(h->lstats.ensure(4 * sizeof(unsigned long long)));
    FKD_CUDA(cudaMemsetAsync(h->lstats.p, 0, 4 * sizeof(unsigned long long), h->stream));
  }
  return FKD_OK;
}

fkd_status fkd_learn_stats(fkd_tree h, uint64_t* stats, int reset) {
  if (!h || !stats) return fail(FKD_ERR_ARG, "null argument");
  stats[0] = stats[1] = stats[2] = stats[3] = 0;
  if (!h->lstats.p) return FKD_OK;
  FKD_CUDA(cudaMemcpyAsync(stats, h->lstats.p, 4 * sizeof(uint64_t), cudaMemcpyDeviceToHost, h->stream));
  if (reset) FKD_CUDA(cudaMemsetAsync(h->lstats.p, 0, 4 * sizeof(unsigned long long), h->stream));
  FKD_CUDA(cudaStreamSynchronize(h->stream));
  return FKD_OK;
}

fkd_status fkd_sync(fkd_tree h) {
  if (!h) return fail(FKD_ERR_ARG, "null handle");
  DeviceScope ds(h->device);
  fkd_status s = check_err_word(h, "fkd_sync");
  if (s != FKD_OK) return s;
  // asynchronous searches latch into the error word of the slot they leased
  std::vector<SearchSlot*> all;
  {
    std::lock_guard<std::mutex> g(h->slot_mu);
    for (auto& p : h->slots) all.push_back(p.get());
  }
  for (SearchSlot* sl : all) {
    FKD_CUDA(cudaStreamWaitEvent(h->stream, sl->done, 0));
    FKD_CUDA(cudaMemcpyAsync(h->herr + 1, sl->err.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    FKD_CUDA(cudaMemsetAsync(sl->err.p, 0, sizeof(uint32_t), h->stream));
    FKD_CUDA(cudaStreamSynchronize(h->stream));
    if ((s = status_from_err(h->herr[1], "fkd_sync")) != FKD_OK) return s;
  }
  return FKD_OK;
}

}  // extern "C"
