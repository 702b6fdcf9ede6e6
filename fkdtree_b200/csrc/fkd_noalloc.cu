// fkd_noalloc.cu -- a build entry point that allocates no memory.
//
// Who needs it: code that runs inside a host framework which owns every byte
// of device memory through its own pool or caching allocator and forbids
// direct cudaMalloc / cudaFree while events are processed -- those calls
// synchronise the whole device and can fail in the middle of an event -- for
// instance the per-event reconstruction step of an online trigger, where a
// kd-tree is built for every small group of detector hits.  The regular
// fkd_build grows the handle's device buffers on demand; this entry point
// instead works in a fixed scratch area that is part of the library image.
//
// Scratch: the file-scope array g_noalloc_scratch below (one per GPU that
// loads the library, alive until the process exits).  It holds the event
// descriptor, the node table of one subtree and the error word, which limits
// a build to one shared-memory subtree: at most fkd_build_noalloc_max_points(dim)
// points (4096 for dim <= 3, 3072 for dim 4).  Host code may not use the
// array's name as a device address, so the first call on each device looks the
// address up with cudaGetSymbolAddress (with that device current) and keeps
// it; make that first call before any stream capture.  Every call reuses the
// same array and leaves its contents behind: the set-up kernel clears what has
// to start at zero (the error word), and calls whose work overlaps on the GPU
// -- two streams, or two host threads on one device -- race on the array and
// must be serialised by the caller.
#include <mutex>
#include <string>

#include "../../include/fkdtree_b200.h"
#include "fkd_internal.h"

using namespace fkd;

namespace fkd {
fkd_status capi_fail(fkd_status s, const std::string& msg);
fkd_status capi_status_from_err(uint32_t e, const char* what);
}  // namespace fkd

namespace {

constexpr uint32_t NA_MAX = 4096;  // the largest shared-memory subtree (dim <= 3)
constexpr size_t NA_DESC = 256;    // event descriptor, subtree list, error word
constexpr size_t NA_BYTES = NA_DESC + (size_t)NA_MAX * sizeof(uint4) + (size_t)NA_MAX * sizeof(uint32_t);

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

struct NoallocLayout {
  EvDesc* ev;
  uint2* sub;
  uint32_t* err;
  uint4* nodes;
  uint32_t* ids;
};

__host__ __device__ inline NoallocLayout layout_of(unsigned char* base) {
  NoallocLayout l;
  l.ev = (EvDesc*)base;
  l.sub = (uint2*)(base + 128);
  l.err = (uint32_t*)(base + 192);
  l.nodes = (uint4*)(base + NA_DESC);
  l.ids = (uint32_t*)(base + NA_DESC + (size_t)NA_MAX * sizeof(uint4));
  return l;
}

// Writes the one-event, one-subtree plan into the scratch and clears the
// error word (the scratch keeps whatever the previous call left).
__global__ void k_noalloc_setup(uint32_t n) {
  const NoallocLayout l = layout_of(g_noalloc_scratch);
  EvDesc e;
  e.g.n = n;
  e.g.H = floor_log2_u32(n);
  e.g.M = n ? n - ((1u << e.g.H) - 1u) : 0u;
  e.base = 0u;
  e.d0 = 0u;
  e.nq = 0u;
  e.qbase = e.qcbase = e.qout = 0ull;
  *l.ev = e;
  *l.sub = make_uint2(0u, 0u);
  *l.err = 0u;
}

// Node table (scratch) -> the caller's tables in the reference's SoA layout.
__global__ void k_noalloc_tables(uint32_t n, int dim, float* __restrict__ tab, uint32_t* __restrict__ tab_ids) {
  const NoallocLayout l = layout_of(g_noalloc_scratch);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint4 v = l.nodes[i];
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
    for (int c = 0; c < dim; ++c) tab[(uint64_t)c * n + i] = __uint_as_float(w[c]);
    tab_ids[i] = l.ids[i];
  }
}

std::mutex g_mu;
void* g_addr[256];  // scratch address per device ordinal, looked up once

}  // namespace

extern "C" {

uint32_t fkd_build_noalloc_max_points(int dim) { return (uint32_t)(dim >= 1 && dim <= 3 ? sub_capacity(3) : (dim == 4 ? sub_capacity(4) : 0)); }

fkd_status fkd_build_noalloc(int dim, const float* coords, const uint32_t* ids, uint32_t n, float* tab,
                             uint32_t* tab_ids, void* stream) {
  if (dim < 1 || dim > 4) return capi_fail(FKD_ERR_ARG, "fkd_build_noalloc: dim must be 1..4");
  const uint32_t cap = fkd_build_noalloc_max_points(dim);
  if (n > cap)
    return capi_fail(FKD_ERR_ARG, "fkd_build_noalloc: " + std::to_string(n) + " points exceed its fixed scratch (at most " +
                                      std::to_string(cap) + " points for dim " + std::to_string(dim) +
                                      "); use fkd_build");
  if (n == 0) return FKD_OK;
  if (!coords || !ids || !tab || !tab_ids) return capi_fail(FKD_ERR_ARG, "fkd_build_noalloc: null device pointer");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return capi_fail(FKD_ERR_CUDA, std::string("fkd_build_noalloc: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 256) return capi_fail(FKD_ERR_ARG, "fkd_build_noalloc: device ordinal out of range");
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return capi_fail(FKD_ERR_CUDA, std::string("fkd_build_noalloc: scratch address: ") + cudaGetErrorString(e));
      g_addr[dev] = p;
    }
    base = g_addr[dev];
  }
  const NoallocLayout l = layout_of((unsigned char*)base);
  const cudaStream_t s = (cudaStream_t)stream;
  k_noalloc_setup<<<1, 1, 0, s>>>(n);
  count_launches(1);
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = launch_subtree_direct(l.ev, l.sub, 1, CSoA{(const uint32_t*)coords, ids, n}, Table{l.nodes, l.ids}, l.err,
                              dim, s);
  if (e == cudaSuccess) {
    k_noalloc_tables<<<(n + 255) / 256, 256, 0, s>>>(n, dim, tab, tab_ids);
    count_launches(1);
    e = cudaGetLastError();
  }
  uint32_t err = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&err, l.err, sizeof(err), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return capi_fail(FKD_ERR_CUDA, std::string("fkd_build_noalloc: ") + cudaGetErrorString(e));
  return capi_status_from_err(err, "fkd_build_noalloc");
}

}  // extern "C"
