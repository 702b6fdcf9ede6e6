// fkd_features.cu -- node summaries for the learned split, the bracket that
// turns a prediction into the starting state of the exact select, and the
// recorder of training targets.  No reference counterpart.
//
// Features of a segment (tree node) at depth d, split dimension c = d % dim,
// from 256 points at stratified positions start + (2i+1)*len/512 of the
// segment (the working order inside a segment is arbitrary, so these are an
// unbiased sample):
//   [0..5]   sample min / max along dimensions c, c+1, c+2 (mod dim), clamped to [-4, 4]
//   [6]      log2(len) / 32
//   [7]      d / 32
//   [8..39]  histogram of the sample along c: 32 equal bins over [min_c, max_c], fractions
// Target: (split value - min_c) / (max_c - min_c), the position of the exact
// split inside the sample's range.
#include <math.h>

#include "fkd_internal.h"

namespace fkd {

constexpr int NSAMP = 256;
constexpr int NBIN = 32;

__device__ __forceinline__ float warp_min(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// One warp per segment, 8 samples per lane.
template <int DIM>
__global__ void __launch_bounds__(128) k_features(uint32_t d, const EvDesc* __restrict__ evs,
                                                  const uint2* __restrict__ segs, uint32_t nseg, CSoA src,
                                                  float* __restrict__ feat, float2* __restrict__ range) {
  __shared__ uint32_t hist[4][NBIN];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t s = blockIdx.x * 4u + warp;
  if (s >= nseg) return;
  const uint2 sd = segs[s];
  const Geom g = evs[sd.x].g;
  const uint32_t start = evs[sd.x].base + seg_start(g, d, sd.y);
  const uint32_t len = seg_len(g, d, sd.y);
  const uint32_t c = d % DIM;
  float v[8][3];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t i = lane + 32u * k;
    const uint32_t pos = start + (uint32_t)(((2ull * i + 1ull) * len) / (2ull * NSAMP));
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const uint32_t cc = (c + q) % DIM;
      v[k][q] = __uint_as_float(src.base[(uint64_t)cc * src.stride + pos]);
    }
  }
  float mn[3], mx[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    float a = v[0][q], b = v[0][q];
#pragma unroll
    for (int k = 1; k < 8; ++k) {
      a = fminf(a, v[k][q]);
      b = fmaxf(b, v[k][q]);
    }
    mn[q] = warp_min(a);
    mx[q] = warp_max(b);
  }
  if (lane < NBIN) hist[warp][lane] = 0u;
  __syncwarp();
  const float lo = mn[0], width = mx[0] - mn[0];
  const float scale = width > 0.f ? (float)NBIN / width : 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    int b = (int)((v[k][0] - lo) * scale);
    b = b < 0 ? 0 : (b >= NBIN ? NBIN - 1 : b);
    atomicAdd(&hist[warp][b], 1u);
  }
  __syncwarp();
  float* f = feat + (uint64_t)s * FKD_MLP_FEATURES;
  if (lane < 6) {
    const float x = (lane & 1) ? mx[lane >> 1] : mn[lane >> 1];
    f[lane] = fminf(fmaxf(x, -4.f), 4.f);
  }
  if (lane == 6) f[6] = log2f((float)(len > 0 ? len : 1)) / 32.f;
  if (lane == 7) f[7] = (float)d / 32.f;
  f[8 + lane] = (float)hist[warp][lane] / (float)NSAMP;
  if (lane == 0) range[s] = make_float2(mn[0], mx[0]);
}

cudaError_t launch_features(uint32_t d, const EvDesc* evs, const uint2* segs, uint32_t nseg, CSoA src, int dim,
                            float* feat, float2* range, cudaStream_t stream) {
  if (nseg == 0) return cudaSuccess;
  const unsigned blocks = (nseg + 3) / 4;
  switch (dim) {
    case 1: k_features<1><<<blocks, 128, 0, stream>>>(d, evs, segs, nseg, src, feat, range); break;
    case 2: k_features<2><<<blocks, 128, 0, stream>>>(d, evs, segs, nseg, src, feat, range); break;
    case 3: k_features<3><<<blocks, 128, 0, stream>>>(d, evs, segs, nseg, src, feat, range); break;
    default: k_features<4><<<blocks, 128, 0, stream>>>(d, evs, segs, nseg, src, feat, range); break;
  }
  count_launches(1);
  return cudaGetLastError();
}

// Turns the prediction of each segment into a predicted block of the select:
// the value keys of [v - r, v + r], r = delta * range, within the segment's
// own interval, binned linearly by the pass that follows.  That pass counts
// the points below the block; if the pivot's rank falls inside it the select
// continues from the block's bin, otherwise the segment restarts from its own
// interval (fkd_build.cu, k_hist).
__global__ void k_bracket(uint32_t d, const EvDesc* __restrict__ evs, const uint2* __restrict__ segs, uint32_t nseg,
                          const float* __restrict__ yhat, const float2* __restrict__ range, float delta,
                          SegSel* __restrict__ sel, unsigned long long* __restrict__ stats) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  if (sel[s].done) return;
  const float2 rg = range[s];
  const float w = rg.y - rg.x;
  const float y = yhat[s];
  if (!(w > 0.f) || !isfinite(y) || !isfinite(w)) return;
  const float v = rg.x + y * w, r = delta * w;
  const float lo = v - r, hi = v + r;
  if (!isfinite(lo) || !isfinite(hi)) return;
  SegSel* p = &sel[s];
  const uint32_t slo = (uint32_t)(p->klo0 >> 32), shi = (uint32_t)(p->khi0 >> 32);
  uint32_t lk = mono_bits(__float_as_uint(lo)), hk = mono_bits(__float_as_uint(hi));
  lk = lk < slo ? slo : lk;
  hk = hk > shi ? shi : hk;
  if (lk >= hk) return;
  // a block wider than half the segment's value range saves nothing
  const float a = __uint_as_float((lk & 0x80000000u) ? (lk & 0x7fffffffu) : ~lk);
  const float b = __uint_as_float((hk & 0x80000000u) ? (hk & 0x7fffffffu) : ~hk);
  const float bw = __fsub_rn(b, a);
  if (!(bw > 0.f) || !isfinite(bw)) return;
  if (p->lin0 && __fmul_rn(bw, p->scale0) > 1024.f) return;
  const float sc = __fdiv_rn(2048.f, bw);
  if (!(sc > 0.f) || !isfinite(sc)) return;
  p->klo = (unsigned long long)lk << 32;
  p->khi = ((unsigned long long)hk << 32) | 0xffffffffull;
  p->lin = 1u;
  p->vmin = a;
  p->scale = sc;
  p->verify = 1u;
  p->below = 0u;
  if (stats) atomicAdd(&stats[0], 1ull);
}

cudaError_t launch_bracket(uint32_t d, const EvDesc* evs, const uint2* segs, uint32_t nseg, const float* yhat,
                           const float2* range, float delta, SegSel* sel, unsigned long long* stats,
                           cudaStream_t stream) {
  if (nseg == 0) return cudaSuccess;
  k_bracket<<<(nseg + 255) / 256, 256, 0, stream>>>(d, evs, segs, nseg, yhat, range, delta, sel, stats);
  count_launches(1);
  return cudaGetLastError();
}

// After a level's partition: the split value of every segment is in its node;
// append (features, target) of segments with a non-degenerate sample range.
template <int DIM>
__global__ void k_record(uint32_t d, const EvDesc* __restrict__ evs, const uint2* __restrict__ segs, uint32_t nseg,
                         Table tab, const float* __restrict__ feat, const float2* __restrict__ range,
                         float* __restrict__ rec_x, float* __restrict__ rec_t, unsigned long long* __restrict__ rec_n,
                         uint64_t cap) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  const uint2 sd = segs[s];
  const uint32_t node = evs[sd.x].base + (1u << d) - 1u + sd.y;
  const uint4 nd = tab.nodes[node];
  const uint32_t c = d % DIM;
  const uint32_t w4[4] = {nd.x, nd.y, nd.z, nd.w};
  const float v = __uint_as_float(w4[c]);
  const float2 rg = range[s];
  const float w = rg.y - rg.x;
  if (!(w > 0.f)) return;
  const unsigned long long at = atomicAdd(rec_n, 1ull);
  if (at >= cap) return;
  for (int k = 0; k < FKD_MLP_FEATURES; ++k) rec_x[at * FKD_MLP_FEATURES + k] = feat[(uint64_t)s * FKD_MLP_FEATURES + k];
  rec_t[at] = (v - rg.x) / w;
}

cudaError_t launch_record(uint32_t d, const EvDesc* evs, const uint2* segs, uint32_t nseg, int dim, Table tab,
                          const float* feat, const float2* range, float* rec_x, float* rec_t,
                          unsigned long long* rec_n, uint64_t rec_cap, cudaStream_t stream) {
  if (nseg == 0) return cudaSuccess;
  const unsigned blocks = (nseg + 255) / 256;
  switch (dim) {
    case 1: k_record<1><<<blocks, 256, 0, stream>>>(d, evs, segs, nseg, tab, feat, range, rec_x, rec_t, rec_n, rec_cap); break;
    case 2: k_record<2><<<blocks, 256, 0, stream>>>(d, evs, segs, nseg, tab, feat, range, rec_x, rec_t, rec_n, rec_cap); break;
    case 3: k_record<3><<<blocks, 256, 0, stream>>>(d, evs, segs, nseg, tab, feat, range, rec_x, rec_t, rec_n, rec_cap); break;
    default: k_record<4><<<blocks, 256, 0, stream>>>(d, evs, segs, nseg, tab, feat, range, rec_x, rec_t, rec_n, rec_cap); break;
  }
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace fkd
