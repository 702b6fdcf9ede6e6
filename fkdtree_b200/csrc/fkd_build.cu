// fkd_build.cu -- the level-by-level FKDTree build on sm_100a.
//
// What is computed is FKDTree_CPU::build (FKDTree_cpu.h:221-277): for every
// depth d and every node t of that depth, the point of rank
// partition_complete_kdtree(len) (FKDTree_cpu.h:287-296) under the order
// (coordinate d % dim, id) (FKDTree_cpu.h:246-252) becomes node (2^d - 1 + t),
// the smaller points form the left child's interval and the larger ones the
// right child's.  Only the SET of points on each side matters to later levels
// (the order is a strict total order), so the GPU is free to permute points
// inside an interval: partitions are written in any order.
//
// Two phases:
//  * global levels (intervals longer than SUBN points): per level, a
//    segmented MSD radix select over the 64-bit order key
//    (monotone(coordinate) << 32 | id), 11-bit digits, one launch per digit
//    pass with the digit of every segment decided by the last CTA to finish
//    that segment (no grid-wide wait), then one partition launch that streams
//    every record once, classifies it against the segment's pivot prefix and
//    scatters it with one atomic per CTA per side (warp ballots + a CTA scan
//    keep every warp's writes contiguous).  Working records are SoA (dim
//    coordinate words + id word) so a digit pass reads 4 B per point.
//  * subtree phase (first level where every interval fits in shared memory):
//    one CTA per interval loads it once, finishes every remaining level in
//    shared memory -- radix select with per-segment packed 16-bit digit
//    histograms and a min/max common-prefix skip for larger segments, direct
//    rank counting for segments of at most 16 points -- and writes each node
//    to the table as it is decided.  One HBM read + one table write for the
//    bottom ~12 levels.
#include <type_traits>

#include "fkd_internal.h"
#include "fkd_mlp.h"

namespace fkd {

#ifdef FKD_PROF
// Phase cycle counters of the subtree kernel (profiling builds only).
__device__ unsigned long long g_prof[8];
extern "C" __attribute__((visibility("default"))) void fkd_prof_read(unsigned long long* out) {
  cudaMemcpyFromSymbol(out, g_prof, sizeof(g_prof));
}
extern "C" __attribute__((visibility("default"))) void fkd_prof_reset() {
  unsigned long long z[8] = {0};
  cudaMemcpyToSymbol(g_prof, z, sizeof(z));
}
#define PROF_T(v) const unsigned long long v = clock64()
#define PROF_ADD(slot, a, b) \
  if (threadIdx.x == 0) atomicAdd(&g_prof[slot], (b) - (a))
#define PROF_CNT(slot) \
  if (threadIdx.x == 0) atomicAdd(&g_prof[slot], 1ull)
#else
#define PROF_T(v)
#define PROF_ADD(slot, a, b)
#define PROF_CNT(slot)
#endif

// ---------------------------------------------------------------- global

constexpr int GT = 256;            // threads of the global-level kernels
constexpr int PIPT = FKD_PART_PIPT;  // records per thread (partition)
constexpr int PTILE = GT * PIPT;
static_assert(PTILE == (int)PART_TILE, "partition tile");
constexpr int GWARPS = GT / 32;
constexpr int RBITS = 11;          // widest digit of the global select (11, 11, 10 per 32-bit word)
constexpr int RBINS = 1 << RBITS;
// digit passes a level may need: a linear value pass, the value bits the
// bin left open (at most three 11-bit digits), the id bits (three), plus a
// verifying pass of a predicted block that missed
constexpr int RPASSES = 8;

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ void write_node(const Table& tab, uint32_t h, const uint32_t* rec, int dim) {
  uint4 v;
  v.x = rec[0];
  v.y = dim > 1 ? rec[1] : 0u;
  v.z = dim > 2 ? rec[2] : 0u;
  v.w = dim > 3 ? rec[3] : rec[dim];
  tab.nodes[h] = v;
  tab.ids[h] = rec[dim];
}

// The float whose order bits (mono_bits) are m (+0.0 for the folded zero).
__device__ __forceinline__ float from_mono(uint32_t m) {
  return __uint_as_float((m & 0x80000000u) ? (m & 0x7fffffffu) : ~m);
}

// Bin of value v in the linear binning of [vmin, vmin + 2048 / scale]: every
// operation rounded on its own (no contraction), so every kernel that bins v
// gets the same bin; non-decreasing in v, since each step is.
__device__ __forceinline__ uint32_t lin_bin(float v, float vmin, float scale) {
  const float x = __fmul_rn(__fsub_rn(v, vmin), scale);
  return x >= 2047.f ? 2047u : (x > 0.f ? (uint32_t)x : 0u);
}

// Sets up the linear binning of the value keys [vlo, vhi]; false when their
// float range is empty or not finite (the passes then bin key bits).
__device__ __forceinline__ bool lin_setup(uint32_t vlo, uint32_t vhi, float& vmin, float& scale) {
  if (vlo >= vhi) return false;
  const float a = from_mono(vlo), b = from_mono(vhi);
  const float w = __fsub_rn(b, a);
  if (!(w > 0.f) || !isfinite(w) || !isfinite(a)) return false;
  const float sc = __fdiv_rn(2048.f, w);
  if (!(sc > 0.f) || !isfinite(sc)) return false;
  vmin = a;
  scale = sc;
  return true;
}

// Level 0 has no parent partition to report its segments' value range: one
// pass over the split coordinate (the first dimension) reduces each
// segment's min / max order bits into bnd, as (~min, max) from a zeroed
// array.  A CTA takes B0_TILES consecutive partition tiles (in segment
// order) and flushes one pair of atomics per segment it saw.
constexpr uint32_t B0_TILES = 16;
template <int DIM>
__global__ void __launch_bounds__(GT) k_bounds0(const EvDesc* __restrict__ evs, const uint2* __restrict__ segs,
                                                const uint2* __restrict__ tiles, uint32_t ntiles, CSoA src,
                                                uint2* __restrict__ bnd) {
  __shared__ uint32_t red[2][GWARPS];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t q0 = blockIdx.x * B0_TILES;
  uint32_t cur = ~0u;
  uint32_t nmn = 0u, mx = 0u;  // ~min, max
  auto flush = [&]() {  // block-uniform
    const uint32_t a = __reduce_max_sync(0xffffffffu, nmn), b = __reduce_max_sync(0xffffffffu, mx);
    if (lane == 0) {
      red[0][warp] = a;
      red[1][warp] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t x = 0u, y = 0u;
      for (int w = 0; w < GWARPS; ++w) {
        x = max(x, red[0][w]);
        y = max(y, red[1][w]);
      }
      if (x | y) {
        atomicMax(&bnd[cur].x, x);
        atomicMax(&bnd[cur].y, y);
      }
    }
    __syncthreads();
    nmn = mx = 0u;
  };
  for (uint32_t q = q0; q < q0 + B0_TILES && q < ntiles; ++q) {
    const uint2 tl = tiles[q];
    if (tl.x != cur) {
      if (cur != ~0u) flush();
      cur = tl.x;
    }
    const uint2 sd = segs[tl.x];
    const Geom eg = evs[sd.x].g;
    const uint32_t len = seg_len(eg, 0u, sd.y);
    const uint32_t start = evs[sd.x].base + seg_start(eg, 0u, sd.y);
    const uint32_t t0 = start + tl.y * PTILE, t1 = min(start + len, t0 + (uint32_t)PTILE);
    uint32_t v[PIPT];
#pragma unroll
    for (int k = 0; k < PIPT; ++k) {
      const uint32_t e = t0 + k * GT + threadIdx.x;
      v[k] = e < t1 ? __ldcs(src.base + e) : 0u;
    }
#pragma unroll
    for (int k = 0; k < PIPT; ++k) {
      if (t0 + k * GT + threadIdx.x < t1) {
        const uint32_t m = mono_bits(v[k]);
        nmn = max(nmn, ~m);
        mx = max(mx, m);
      }
    }
  }
  if (cur != ~0u) flush();
}

__global__ void k_sel_init(uint32_t d, const EvDesc* __restrict__ evs, const uint2* __restrict__ segs, uint32_t nseg,
                           SegSel* __restrict__ sel, uint32_t* __restrict__ pending, const uint2* __restrict__ bnd_in,
                           bool bnd_inverted_min, uint2* __restrict__ bnd_out, const uint32_t* __restrict__ child,
                           bool lin) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s == 0) {
    // pending[p] != 0: digit pass p has a segment to work on
    pending[0] = 1u;
    for (int p = 1; p <= RPASSES; ++p) pending[p] = 0u;
  }
  if (s >= nseg) return;
  const uint2 sd = segs[s];
  const Geom g = evs[sd.x].g;
  const uint32_t len = seg_len(g, d, sd.y);
  SegSel st;
  st.prefix = 0ull;
  st.bits = 0u;
  uint32_t vlo = 0u, vhi = 0xffffffffu;
  if (bnd_in) {
    // every key of the segment lies between its smallest and largest split
    // coordinate: the select starts from that interval (and, in prefix form,
    // below their common prefix)
    uint2 b = bnd_in[s];
    if (bnd_inverted_min) b.x = ~b.x;
    if (b.x <= b.y) {
      vlo = b.x;
      vhi = b.y;
      const uint32_t cp = b.x == b.y ? 32u : (uint32_t)__clz(b.x ^ b.y);
      st.bits = cp;
      st.prefix = cp == 0u ? 0ull : (unsigned long long)(b.x >> (32u - cp));
    }
  }
  st.bits0 = st.bits;
  st.prefix0 = st.prefix;
  st.krem = (d < g.H) ? seg_rank(g, d, sd.y) : 0u;
  st.cnt = len;
  st.done = len <= 1u ? 1u : 0u;
  st.tiles_done = 0u;
  st.curL = st.curR = st.curE = 0u;
  st.verify = 0u;
  st.below = 0u;
  st.kfull = st.krem;
  st.small = 0u;
  st.klo = st.klo0 = (unsigned long long)vlo << 32;
  st.khi = st.khi0 = ((unsigned long long)vhi << 32) | 0xffffffffull;
  st.vmin = st.vmin0 = 0.f;
  st.scale = st.scale0 = 0.f;
  st.lin = st.lin0 = (lin && lin_setup(vlo, vhi, st.vmin0, st.scale0)) ? 1u : 0u;
  st.vmin = st.vmin0;
  st.scale = st.scale0;
  st.cmin = 0xffffffffu;
  st.cmax = 0u;
  sel[s] = st;
  if (bnd_out && child[s] != ~0u) {
    bnd_out[child[s]] = make_uint2(0xffffffffu, 0u);
    bnd_out[child[s] + 1u] = make_uint2(0xffffffffu, 0u);
  }
}

// One digit pass of the segmented select for every segment of depth d.  CTA
// (s, t) counts the digits of the candidates of tile t of segment s -- tiles
// are `ts` records long, so that a level is covered by about four CTAs per SM
// whatever its segment count -- into HCOPIES interleaved shared histograms
// (lane % HCOPIES picks the copy, so lanes of clustered data do not all hit
// one counter), then adds them to the segment's global histogram once.  The
// last CTA of a segment picks the bin holding the pivot rank and narrows the
// interval to it.  Bins: linear in the float value (the segment's first pass,
// `lin`), else the top 11 bits of (value - vlo) while the value is open, else
// of (id - ilo) among the points holding the value.
constexpr int HCOPIES = 4;
#ifndef FKD_HLOADS
#define FKD_HLOADS 4
#endif
constexpr int HLOADS = FKD_HLOADS;  // 16-byte loads per thread in flight
#ifndef FKD_HIST_MINB
#define FKD_HIST_MINB 4
#endif

__device__ __forceinline__ uint32_t bitlen32(uint32_t x) { return x ? 32u - (uint32_t)__clz(x) : 0u; }

template <int DIM>
__global__ void __launch_bounds__(GT, FKD_HIST_MINB) k_hist(uint32_t d, const EvDesc* __restrict__ evs,
                                                const uint2* __restrict__ segs, const uint2* __restrict__ tiles,
                                                uint32_t ts, CSoA src, SegSel* __restrict__ sel,
                                                uint32_t* __restrict__ ghist, const uint32_t* __restrict__ pending_now,
                                                uint32_t* __restrict__ pending_next, uint32_t* __restrict__ err,
                                                unsigned long long* __restrict__ lstats, uint32_t small_ok) {
  __shared__ uint32_t hist[HCOPIES * RBINS];
  __shared__ uint32_t wsum[GWARPS];
  __shared__ uint32_t s_last;
  // pending_now was raised by the previous pass when some segment still needs
  // a digit; without it the whole launch is a no-op.
  if (*(volatile const uint32_t*)pending_now == 0u) return;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint2 tl = tiles[blockIdx.x];
  const uint32_t s = tl.x, t = tl.y;
  const uint2 sd = segs[s];
  const Geom eg = evs[sd.x].g;
  const uint32_t ebase = evs[sd.x].base;
  const uint32_t len = seg_len(eg, d, sd.y);
  const uint32_t ntiles = (len + ts - 1) / ts;
  if (t >= ntiles) return;
  if (sel[s].done) return;
  const unsigned long long klo = sel[s].klo, khi = sel[s].khi;
  const bool lin = sel[s].lin != 0u;
  const float vmin = sel[s].vmin, scale = sel[s].scale;
  const bool verify = sel[s].verify != 0u;  // [klo, khi] is a predicted block of values
  const uint32_t vlo = (uint32_t)(klo >> 32), vhi = (uint32_t)(khi >> 32);
  const bool vphase = vlo != vhi;  // the value is still open
  const uint32_t ilo = (uint32_t)klo, ihi = (uint32_t)khi;
  const uint32_t span = vphase ? vhi - vlo : ihi - ilo;
  const uint32_t bl = bitlen32(span);
  const uint32_t shift = bl > (uint32_t)RBITS ? bl - (uint32_t)RBITS : 0u;
  const uint32_t nb = lin ? (uint32_t)RBINS : (span >> shift) + 1u;
  const uint32_t c = d % DIM;
  const uint32_t start = ebase + seg_start(eg, d, sd.y);
  const uint32_t tend = min(start + len, start + t * ts + ts);
  uint32_t* myhist = hist + (lane % HCOPIES) * RBINS;
  for (uint32_t i = threadIdx.x; i < HCOPIES * RBINS; i += GT) hist[i] = 0u;
  __syncthreads();
  const uint32_t* X = src.base + (uint64_t)c * src.stride;
  uint32_t nbelow = 0u;  // verify pass: points below the predicted block
  uint32_t cmn = 0xffffffffu, cmx = 0u;  // smallest / largest candidate value key (id in the id phase)
  // one value of the tile: the bin of a candidate.  The binning mode (M: 0
  // linear in the value, 1 key bits of the value, 2 id bits) is a template
  // argument, so that the tile loop below is compiled once per mode
  auto count = [&](auto M, auto V, uint32_t raw, uint32_t e) {
    constexpr int mode = decltype(M)::value;
    const uint32_t mv = mono_bits(raw);
    if constexpr (decltype(V)::value) {
      if (mv < vlo) ++nbelow;
    }
    if (mv < vlo || mv > vhi) return;
    uint32_t dig;
    if constexpr (mode == 0) {
      dig = lin_bin(__uint_as_float(raw), vmin, scale);
      cmn = min(cmn, mv);
      cmx = max(cmx, mv);
    } else if constexpr (mode == 1) {
      dig = (mv - vlo) >> shift;
      cmn = min(cmn, mv);
      cmx = max(cmx, mv);
    } else {
      // the value is fixed: the id of the points holding it
      const uint32_t id = __ldcs(src.ids + e);
      if (id < ilo || id > ihi) return;
      dig = (id - ilo) >> shift;
      cmn = min(cmn, id);
      cmx = max(cmx, id);
    }
    atomicAdd(&myhist[dig], 1u);
  };
  // the tile [tb, tend): a scalar head up to a 16-byte boundary, 16-byte
  // loads (HLOADS per thread in flight), a scalar tail
  const uint32_t tb = start + t * ts;
  const uint32_t tlen = tend > tb ? tend - tb : 0u;
  uint32_t head = (uint32_t)(((16u - ((uint32_t)(uintptr_t)(X + tb) & 15u)) & 15u) >> 2);
  if (head > tlen) head = tlen;
  const uint32_t vb0 = tb + head;
  const uint32_t nv = (tlen - head) >> 2;
  const uint4* X4 = reinterpret_cast<const uint4*>(X + vb0);
  auto load = [&](uint4 (&q)[HLOADS], uint32_t v0) {
#pragma unroll
    for (int u = 0; u < HLOADS; ++u) {
      const uint32_t va = v0 + u * GT + threadIdx.x;
      q[u] = va < nv ? __ldcs(X4 + va) : make_uint4(0u, 0u, 0u, 0u);
    }
  };
  constexpr uint32_t HSTEP = (uint32_t)HLOADS * GT;
  auto tile = [&](auto M, auto V) {
    if (threadIdx.x < head) count(M, V, __ldcs(X + tb + threadIdx.x), tb + threadIdx.x);
    // (two register buffers, the next round's loads in flight while this
    // round is counted, measured slower: 0.714 vs 0.675 ms of digit passes
    // per build; eight loads per round: 0.690 ms)
    for (uint32_t v0 = 0; v0 < nv; v0 += HSTEP) {
      uint4 q[HLOADS];
      load(q, v0);
#pragma unroll
      for (int u = 0; u < HLOADS; ++u) {
        const uint32_t va = v0 + u * GT + threadIdx.x;
        if (va < nv) {
          const uint32_t e = vb0 + 4u * va;
          count(M, V, q[u].x, e);
          count(M, V, q[u].y, e + 1u);
          count(M, V, q[u].z, e + 2u);
          count(M, V, q[u].w, e + 3u);
        }
      }
    }
    const uint32_t tail0 = vb0 + 4u * nv;
    if (tail0 + threadIdx.x < tend) count(M, V, __ldcs(X + tail0 + threadIdx.x), tail0 + threadIdx.x);
  };
  // and once per verify case (a learned bracket's verifying pass also counts
  // the points below the predicted block)
  auto tile_v = [&](auto M) {
    if (verify)
      tile(M, std::true_type{});
    else
      tile(M, std::false_type{});
  };
  if (lin)
    tile_v(std::integral_constant<int, 0>{});
  else if (vphase)
    tile_v(std::integral_constant<int, 1>{});
  else
    tile_v(std::integral_constant<int, 2>{});
  if (verify) {
    for (int o = 16; o > 0; o >>= 1) nbelow += __shfl_xor_sync(0xffffffffu, nbelow, o);
    if (lane == 0 && nbelow) atomicAdd(&sel[s].below, nbelow);
  }
  cmn = __reduce_min_sync(0xffffffffu, cmn);
  cmx = __reduce_max_sync(0xffffffffu, cmx);
  if (lane == 0 && cmn <= cmx) {
    atomicMin(&sel[s].cmin, cmn);
    atomicMax(&sel[s].cmax, cmx);
  }
  __syncthreads();
  uint32_t* gh = ghist + (uint64_t)s * RBINS;
  for (uint32_t i = threadIdx.x; i < nb; i += GT) {
    uint32_t v = 0u;
#pragma unroll
    for (int cpy = 0; cpy < HCOPIES; ++cpy) v += hist[cpy * RBINS + i];
    if (v) atomicAdd(&gh[i], v);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&sel[s].tiles_done, 1u) == ntiles - 1u) ? 1u : 0u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x == 0 && lstats) atomicAdd(&lstats[3], 1ull);  // segment digit passes run
  // Last CTA of segment s: locate the bin holding rank krem.
  uint32_t krem = *(volatile uint32_t*)&sel[s].krem;
  constexpr int BPT = RBINS / GT;  // bins per thread
  uint32_t h[BPT];
  uint32_t mine = 0u;
#pragma unroll
  for (int k = 0; k < BPT; ++k) {
    const uint32_t b = threadIdx.x * BPT + k;
    h[k] = b < nb ? __ldcg(gh + b) : 0u;
    mine += h[k];
  }
  uint32_t incl = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (uint32_t)o) incl += y;
  }
  if (lane == 31u) wsum[warp] = incl;
  __syncthreads();
  uint32_t wbase = 0u, total = 0u;
  for (uint32_t k = 0; k < (uint32_t)GWARPS; ++k) {
    if (k < warp) wbase += wsum[k];
    total += wsum[k];
  }
  if (verify) {
    // the predicted block holds the pivot iff below <= k < below + total
    const uint32_t below = *(volatile uint32_t*)&sel[s].below;
    if (krem >= below && krem - below < total) {
      krem -= below;
      if (threadIdx.x == 0) {
        sel[s].verify = 0u;
        if (lstats) atomicAdd(&lstats[1], 1ull);
      }
    } else {
      // miss: restart this segment from its own interval
      for (uint32_t b = threadIdx.x; b < nb; b += GT) gh[b] = 0u;
      if (threadIdx.x == 0) {
        SegSel* p = &sel[s];
        p->cmin = 0xffffffffu;
        p->cmax = 0u;
        p->klo = p->klo0;
        p->khi = p->khi0;
        p->lin = p->lin0;
        p->vmin = p->vmin0;
        p->scale = p->scale0;
        p->krem = p->kfull;
        p->cnt = len;
        p->verify = 0u;
        p->tiles_done = 0u;
        *pending_next = 1u;
        if (lstats) atomicAdd(&lstats[2], 1ull);
      }
      return;
    }
  }
  // every candidate lies in [cmin, cmax]: the chosen bin is clipped to it
  const uint32_t cmin = *(volatile uint32_t*)&sel[s].cmin, cmax = *(volatile uint32_t*)&sel[s].cmax;
  __syncthreads();
  if (threadIdx.x == 0) {
    sel[s].cmin = 0xffffffffu;
    sel[s].cmax = 0u;
  }
  uint32_t cum = wbase + incl - mine;
#pragma unroll
  for (int k = 0; k < BPT; ++k) {
    const uint32_t b = threadIdx.x * BPT + k;
    if (b < nb && krem >= cum && krem < cum + h[k]) {
      unsigned long long nlo, nhi;
      if (lin) {
        // the values of bin b form an interval (lin_bin is monotone): find
        // its ends among the order bits [vlo, vhi] by bisection
        uint32_t a0 = vlo, a1 = vhi;  // first key with bin >= b
        while (a0 < a1) {
          const uint32_t m = a0 + ((a1 - a0) >> 1);
          if (lin_bin(from_mono(m), vmin, scale) >= b) a1 = m; else a0 = m + 1u;
        }
        uint32_t z0 = a0, z1 = vhi;  // last key with bin <= b
        while (z0 < z1) {
          const uint32_t m = z0 + (uint32_t)(((unsigned long long)(z1 - z0) + 1ull) >> 1);
          if (lin_bin(from_mono(m), vmin, scale) <= b) z0 = m; else z1 = m - 1u;
        }
        nlo = (unsigned long long)a0 << 32;
        nhi = ((unsigned long long)z0 << 32) | 0xffffffffull;
      } else if (vphase) {
        const unsigned long long a = (unsigned long long)vlo + ((unsigned long long)b << shift);
        unsigned long long z = a + ((1ull << shift) - 1ull);
        if (z > vhi) z = vhi;
        nlo = a << 32;
        nhi = (z << 32) | 0xffffffffull;
      } else {
        const unsigned long long a = (unsigned long long)ilo + ((unsigned long long)b << shift);
        unsigned long long z = a + ((1ull << shift) - 1ull);
        if (z > ihi) z = ihi;
        nlo = ((unsigned long long)vlo << 32) | a;
        nhi = ((unsigned long long)vlo << 32) | z;
      }
      if (cmin <= cmax) {
        if (lin || vphase) {
          nlo = max(nlo, (unsigned long long)cmin << 32);
          nhi = min(nhi, ((unsigned long long)cmax << 32) | 0xffffffffull);
        } else {
          nlo = max(nlo, ((unsigned long long)vlo << 32) | cmin);
          nhi = min(nhi, ((unsigned long long)vlo << 32) | cmax);
        }
      }
      SegSel* p = &sel[s];
      p->klo = nlo;
      p->khi = nhi;
      p->lin = 0u;
      p->krem = krem - cum;
      p->cnt = h[k];
      p->done = (h[k] == 1u || nlo == nhi) ? 1u : 0u;
      if (!p->done && small_ok && h[k] <= SMALL_CAP) {
        // few candidates left: the partition parks them and k_small_fix
        // orders them by key (no further digit passes)
        p->done = 1u;
        p->small = 1u;
      }
      if (!p->done) *pending_next = 1u;
    }
    cum += h[k];
  }
  for (uint32_t b = threadIdx.x; b < nb; b += GT) gh[b] = 0u;
  if (threadIdx.x == 0) sel[s].tiles_done = 0u;
  // the last thread's inclusive sum is the number of candidates; it must
  // cover krem, otherwise the select state is inconsistent.
  if (threadIdx.x == GT - 1 && krem >= total) atomicOr(err, ERRB_INTERNAL);
}

template <int DIM>
__device__ __forceinline__ uint32_t pick_coord(const uint32_t* rec, uint32_t c) {
  uint32_t v = rec[0];
#pragma unroll
  for (int w = 1; w < DIM; ++w) v = (c == (uint32_t)w) ? rec[w] : v;
  return v;
}

// resident CTAs per SM the partition is compiled for: 8 (32 registers, a few
// spilled words) keeps 2,048 threads per SM loading; measured on the 16M
// clustered build: 4 / 5 / 6 / 8 CTAs -> 5.92 / 5.72 / 5.69 / 5.61 ms
#ifndef FKD_PART_MINB
#define FKD_PART_MINB (PIPT <= 4 ? 8 : 3)
#endif

// Streams every record of depth-d segments once: records below the pivot go
// to [start, start + rank), the pivot to the table, the rest above it.
template <int DIM>
__global__ void __launch_bounds__(GT, FKD_PART_MINB) k_partition(uint32_t d, const EvDesc* __restrict__ evs,
                                                     const uint2* __restrict__ segs, const uint2* __restrict__ tiles,
                                                     CSoA src, SoA dst, SegSel* __restrict__ sel, Table tab,
                                                     uint32_t* __restrict__ err, uint2* __restrict__ bnd_out,
                                                     const uint32_t* __restrict__ child,
                                                     uint32_t* __restrict__ tiebuf) {
  __shared__ uint32_t sL[PIPT * GWARPS], sR[PIPT * GWARPS];
  __shared__ uint32_t sBL[PIPT * GWARPS], sBR[PIPT * GWARPS];  // the warps' left / right ballots
  __shared__ uint32_t s_base[2];
  __shared__ uint32_t sb[4];  // the children's bounds, reduced over the CTA's warps
  const uint2 tl = tiles[blockIdx.x];
  const uint32_t s = tl.x, t = tl.y;
  const uint2 sd = segs[s];
  const Geom eg = evs[sd.x].g;
  const uint32_t ebase = evs[sd.x].base;
  const uint32_t len = seg_len(eg, d, sd.y);
  const uint32_t ntiles = (len + PTILE - 1) / PTILE;
  if (t >= ntiles) return;
  if (threadIdx.x == 0) {  // ordered before their first use by the barriers below
    sb[0] = 0xffffffffu;
    sb[1] = 0u;
    sb[2] = 0xffffffffu;
    sb[3] = 0u;
  }
  const uint32_t start = ebase + seg_start(eg, d, sd.y);
  const uint32_t rank = seg_rank(eg, d, sd.y);
  const uint32_t node = ebase + (1u << d) - 1u + sd.y;  // this segment's node
  const uint32_t t0 = start + t * PTILE;
  const uint32_t t1 = min(start + len, t0 + (uint32_t)PTILE);
  const unsigned long long klo = sel[s].klo, khi = sel[s].khi;
  const uint32_t vlo = (uint32_t)(klo >> 32), vhi = (uint32_t)(khi >> 32);
  const bool vonly = (uint32_t)klo == 0u && (uint32_t)khi == 0xffffffffu;
  const uint32_t cnt = sel[s].cnt;
  const bool small = sel[s].small != 0u;
  if (threadIdx.x == 0 && !sel[s].done) atomicOr(err, ERRB_INTERNAL);  // the select ran out of passes
  const uint32_t c = d % DIM;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;

  uint32_t rec[PIPT][DIM + 1];
#pragma unroll
  for (int k = 0; k < PIPT; ++k) {
    const uint32_t e = t0 + k * GT + threadIdx.x;
    const bool v = e < t1;
#pragma unroll
    for (int w = 0; w < DIM; ++w) rec[k][w] = v ? __ldcs(src.base + (uint64_t)w * src.stride + e) : 0u;
    rec[k][DIM] = v ? __ldcs(src.ids + e) : 0u;
  }
  uint32_t eqmask = 0u;  // bit k: record k is a candidate of the select (inside [klo, khi])
  bool nan = false;
#pragma unroll
  for (int k = 0; k < PIPT; ++k) {
    const uint32_t e = t0 + k * GT + threadIdx.x;
    uint32_t cls = 3u;  // 0 below, 1 equal, 2 above, 3 none
    if (e < t1) {
      if (d == 0u) {  // deeper levels move the records level 0 checked
#pragma unroll
        for (int w = 0; w < DIM; ++w) nan |= is_nan_bits(rec[k][w]);
      }
      const uint32_t mv = mono_bits(pick_coord<DIM>(rec[k], c));
      if (vonly) {  // the interval spans every id: the order bits decide
        cls = mv < vlo ? 0u : (mv > vhi ? 2u : 1u);
      } else {
        const uint64_t key = ((uint64_t)mv << 32) | rec[k][DIM];
        cls = key < klo ? 0u : (key > khi ? 2u : 1u);
      }
    }
    if (cls == 1u) eqmask |= 1u << k;
    const uint32_t bl = __ballot_sync(0xffffffffu, cls == 0u);
    const uint32_t br = __ballot_sync(0xffffffffu, cls == 2u);
    if (lane == 0) {
      sL[k * GWARPS + warp] = __popc(bl);
      sR[k * GWARPS + warp] = __popc(br);
      sBL[k * GWARPS + warp] = bl;
      sBR[k * GWARPS + warp] = br;
    }
  }
  if (nan) atomicOr(err, ERRB_NAN);
  __syncthreads();
  if (warp == 0) {
    // exclusive scan over the PIPT*GWARPS (slot-major) warp counts
    constexpr int PER = PIPT * GWARPS / 32;
    uint32_t a[PER], b[PER], sa = 0u, sb = 0u;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      a[k] = sL[lane * PER + k];
      b[k] = sR[lane * PER + k];
      sa += a[k];
      sb += b[k];
    }
    uint32_t ia = sa, ib = sb;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t ya = __shfl_up_sync(0xffffffffu, ia, o);
      const uint32_t yb = __shfl_up_sync(0xffffffffu, ib, o);
      if (lane >= (uint32_t)o) {
        ia += ya;
        ib += yb;
      }
    }
    uint32_t ea = ia - sa, eb = ib - sb;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      sL[lane * PER + k] = ea;
      sR[lane * PER + k] = eb;
      ea += a[k];
      eb += b[k];
    }
    if (lane == 31u) {
      s_base[0] = ia ? atomicAdd(&sel[s].curL, ia) : 0u;
      s_base[1] = ib ? atomicAdd(&sel[s].curR, ib) : 0u;
    }
  }
  __syncthreads();
  const uint32_t lt = lanemask_lt();
  const uint32_t endL = start + rank, endR = start + len;
  // bounds of the children's split coordinate (the next level's select starts below their common prefix)
  const uint32_t cnext = (d + 1u) % DIM;
  const uint32_t ch = bnd_out ? child[s] : ~0u;
  uint32_t mnL = 0xffffffffu, mxL = 0u, mnR = 0xffffffffu, mxR = 0u;
  const uint32_t baseL = start + s_base[0], baseR = endL + 1u + s_base[1];
#pragma unroll
  for (int k = 0; k < PIPT; ++k) {
    uint32_t pos = 0xffffffffu, lim = 0u;
    const uint32_t bl = sBL[k * GWARPS + warp], br = sBR[k * GWARPS + warp];
    if ((bl >> lane) & 1u) {
      pos = baseL + sL[k * GWARPS + warp] + __popc(bl & lt);
      lim = endL;
    } else if ((br >> lane) & 1u) {
      pos = baseR + sR[k * GWARPS + warp] + __popc(br & lt);
      lim = endR;
    } else if (((eqmask >> k) & 1u) && small) {
      // the select left a few candidates: parked for k_small_fix, which orders them by key
      const uint32_t slot = atomicAdd(&sel[s].curE, 1u);
      if (slot < SMALL_CAP && tiebuf) {
        uint32_t* tb = tiebuf + ((size_t)s * SMALL_CAP + slot) * (DIM + 1);
#pragma unroll
        for (int w = 0; w <= DIM; ++w) tb[w] = rec[k][w];
      } else {
        atomicOr(err, ERRB_INTERNAL);
      }
    } else if ((eqmask >> k) & 1u) {
      const uint32_t krem = sel[s].krem;
      uint32_t ticket = 0u;
      if (cnt != 1u) ticket = atomicAdd(&sel[s].curE, 1u);  // repeated (coordinate, id) keys only
      if (ticket == krem) {
        write_node(tab, node, rec[k], DIM);
      } else if (ticket < krem) {
        pos = start + atomicAdd(&sel[s].curL, 1u);
        lim = endL;
      } else {
        pos = endL + 1u + atomicAdd(&sel[s].curR, 1u);
        lim = endR;
      }
    }
    if (pos != 0xffffffffu) {
      if (pos < lim) {
#pragma unroll
        for (int w = 0; w < DIM; ++w) __stcs(dst.base + (uint64_t)w * dst.stride + pos, rec[k][w]);
        __stcs(dst.ids + pos, rec[k][DIM]);
        const uint32_t mv = mono_bits(pick_coord<DIM>(rec[k], cnext));
        if (lim == endL) {
          mnL = min(mnL, mv);
          mxL = max(mxL, mv);
        } else {
          mnR = min(mnR, mv);
          mxR = max(mxR, mv);
        }
      } else {
        atomicOr(err, ERRB_INTERNAL);
      }
    }
  }
  if (ch != ~0u) {  // CTA-uniform
    // warp, then CTA reduction; one global atomic per bound per CTA (every
    // CTA of a segment hits the same two words: per-warp atomics would
    // multiply that contention by eight; a last-warp-arrives counter in
    // place of the barrier measured 1-2 us slower per launch)
    mnL = __reduce_min_sync(0xffffffffu, mnL);
    mxL = __reduce_max_sync(0xffffffffu, mxL);
    mnR = __reduce_min_sync(0xffffffffu, mnR);
    mxR = __reduce_max_sync(0xffffffffu, mxR);
    if (lane == 0u) {
      atomicMin(&sb[0], mnL);
      atomicMax(&sb[1], mxL);
      atomicMin(&sb[2], mnR);
      atomicMax(&sb[3], mxR);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      if (sb[0] <= sb[1]) {
        atomicMin(&bnd_out[ch].x, sb[0]);
        atomicMax(&bnd_out[ch].y, sb[1]);
      }
      if (sb[2] <= sb[3]) {
        atomicMin(&bnd_out[ch + 1u].x, sb[2]);
        atomicMax(&bnd_out[ch + 1u].y, sb[3]);
      }
    }
  }
}

// Segments whose select left 2..SMALL_CAP candidates (SegSel::small): the
// partition parked them; one warp per segment orders them by their order key
// (coordinate, then id: the reference comparator, FKDTree_cpu.h:246-252),
// writes the one of rank krem to the table and the others to the ends of the
// children's intervals the partition left free -- the krem smaller ones to
// the last krem slots of the left interval, the larger ones to the last
// slots of the right interval -- and widens the children's coordinate bounds.
template <int DIM>
__global__ void k_small_fix(uint32_t d, const EvDesc* __restrict__ evs, const uint2* __restrict__ segs, uint32_t nseg,
                            const SegSel* __restrict__ sel, const uint32_t* __restrict__ tiebuf, SoA dst, Table tab,
                            uint32_t* __restrict__ err, uint2* __restrict__ bnd_out, const uint32_t* __restrict__ child) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (s >= nseg) return;
  if (!sel[s].small) return;
  const uint32_t m = sel[s].cnt;
  if (m > SMALL_CAP || sel[s].curE != m) {
    if (lane == 0) atomicOr(err, ERRB_INTERNAL);
    return;
  }
  const uint2 sd = segs[s];
  const Geom eg = evs[sd.x].g;
  const uint32_t ebase = evs[sd.x].base;
  const uint32_t len = seg_len(eg, d, sd.y);
  const uint32_t start = ebase + seg_start(eg, d, sd.y);
  const uint32_t rank = seg_rank(eg, d, sd.y);
  const uint32_t node = ebase + (1u << d) - 1u + sd.y;
  const uint32_t endL = start + rank, endR = start + len;
  const uint32_t c = d % DIM;
  uint32_t rec[DIM + 1];
  const bool have = lane < m;
#pragma unroll
  for (int w = 0; w <= DIM; ++w) rec[w] = have ? tiebuf[((size_t)s * SMALL_CAP + lane) * (DIM + 1) + w] : 0u;
  // rank by key (lane order breaks repeated keys, which the reference leaves undefined)
  const unsigned long long mykey = order_key(pick_coord<DIM>(rec, c), rec[DIM]);
  uint32_t r = 0u;
  for (uint32_t o = 0; o < m; ++o) {
    const unsigned long long ok = __shfl_sync(0xffffffffu, mykey, o);
    r += (ok < mykey || (ok == mykey && o < lane)) ? 1u : 0u;
  }
  const uint32_t krem = sel[s].krem;
  const uint32_t cnext = (d + 1u) % DIM;
  const uint32_t ch = bnd_out ? child[s] : ~0u;
  uint32_t pos = 0xffffffffu, lim = 0u;
  bool left = false;
  if (have) {
    if (r == krem) {
      write_node(tab, node, rec, DIM);
    } else if (r < krem) {
      pos = endL - krem + r;
      lim = endL;
      left = true;
    } else {
      pos = endR - (m - 1u - krem) + (r - krem - 1u);
      lim = endR;
    }
  }
  if (pos != 0xffffffffu) {
    if (pos < lim && pos >= start) {
#pragma unroll
      for (int w = 0; w < DIM; ++w) dst.base[(uint64_t)w * dst.stride + pos] = rec[w];
      dst.ids[pos] = rec[DIM];
      if (ch != ~0u) {
        const uint32_t mv = mono_bits(pick_coord<DIM>(rec, cnext));
        uint2* b = &bnd_out[left ? ch : ch + 1u];
        atomicMin(&b->x, mv);
        atomicMax(&b->y, mv);
      }
    } else {
      atomicOr(err, ERRB_INTERNAL);
    }
  }
}

// ------------------------------------------------------- small-segment select
//
// For levels whose segments all hold at most SEL_MAX points, one CTA selects
// a whole segment: its split coordinate is loaded into shared memory once and
// every pass runs there -- one launch per level instead of a digit pass
// launch per 11 bits with a global histogram flush each.  With parking on
// (the partition may leave up to SMALL_CAP candidates to k_small_fix), the
// passes narrow a value interval until it holds at most SMALL_CAP points,
// usually after one pass; otherwise (or for a value held by more points) the
// digit passes of the k_hist select fix the pivot key exactly.
constexpr int SEL_MAX = 32768;
constexpr int SELBINS = 2048;  // bins of a pass
// threads: 128 for segments of at most SEL_FEW points (short CTAs: cheaper
// barriers, more of them resident to hide the loads), 512 up to SEL_MANY,
// 1024 above
constexpr int SEL_FEW = 4096;
// 1024 threads above SEL_MANY points: such a CTA holds up to 128 KB of values,
// one per SM, so its own threads carry the loads in flight
constexpr int SEL_MANY = 16384;

template <int DIM, int SELT>
__global__ void __launch_bounds__(SELT) k_select_small(uint32_t d, const EvDesc* __restrict__ evs,
                                                       const uint2* __restrict__ segs, CSoA src,
                                                       SegSel* __restrict__ sel, uint32_t* __restrict__ err,
                                                       bool park) {
  constexpr int SELB = SELBINS / SELT;  // bins per thread
  extern __shared__ uint32_t vals[];  // mono bits of the segment's split coordinate
  __shared__ uint32_t hist[SELT * SELB];
  __shared__ uint32_t wsum[SELT / 32];
  __shared__ unsigned long long s_prefix;
  __shared__ uint32_t s_bits, s_krem, s_cnt, s_lo, s_hi, s_park;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t s = blockIdx.x;
  if (sel[s].done) return;
  const uint2 sd = segs[s];
  const Geom eg = evs[sd.x].g;
  const uint32_t start = evs[sd.x].base + seg_start(eg, d, sd.y);
  const uint32_t len = seg_len(eg, d, sd.y);
  if (len > (uint32_t)SEL_MAX) {
    if (threadIdx.x == 0) atomicOr(err, ERRB_INTERNAL);
    return;
  }
  const uint32_t c = d % DIM;
  const uint32_t* X = src.base + (uint64_t)c * src.stride + start;
  uint32_t vmn = 0xffffffffu, vmx = 0u;
  uint32_t p = threadIdx.x;
  for (; p + 7u * SELT < len; p += 8u * SELT) {  // eight loads in flight
    uint32_t v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = __ldcs(X + p + u * SELT);
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const uint32_t m = mono_bits(v[u]);
      vals[p + u * SELT] = m;
      vmn = min(vmn, m);
      vmx = max(vmx, m);
    }
  }
  for (; p < len; p += SELT) {
    const uint32_t v = mono_bits(__ldcs(X + p));
    vals[p] = v;
    vmn = min(vmn, v);
    vmx = max(vmx, v);
  }
  if (threadIdx.x == 0) {
    s_prefix = sel[s].prefix;
    s_bits = sel[s].bits;
    s_krem = sel[s].krem;
    s_cnt = sel[s].cnt;
    s_lo = 0xffffffffu;
    s_hi = 0u;
    s_park = 0u;
  }
  __syncthreads();
  vmn = __reduce_min_sync(0xffffffffu, vmn);
  vmx = __reduce_max_sync(0xffffffffu, vmx);
  if (lane == 0u) {
    atomicMin(&s_lo, vmn);
    atomicMax(&s_hi, vmx);
  }
  __syncthreads();
  // interval passes (when the partition may park candidates): bins of
  // 2^sh values of the order bits over [lo, hi], sh the smallest shift that
  // leaves at most 2,048 bins; the bin holding rank krem becomes the interval
  // (clipped to hi).  Usually one pass leaves at most SMALL_CAP candidates:
  // the partition parks them and k_small_fix orders them by the full key.
  // A single value held by more than SMALL_CAP points continues below with
  // the id digits.
  if (park && s_bits < 32u) {
    for (int guard = 0; guard < 4; ++guard) {
      const uint32_t lo = s_lo, hi = s_hi, cnt = s_cnt, krem = s_krem;
      if (cnt <= SMALL_CAP || lo >= hi) break;
      const uint32_t rb = 32u - (uint32_t)__clz(hi - lo);
      const uint32_t sh = rb > 11u ? rb - 11u : 0u;
      const uint32_t nb = ((hi - lo) >> sh) + 1u;
      for (uint32_t i = threadIdx.x; i < nb; i += SELT) hist[i] = 0u;
      __syncthreads();
      for (uint32_t p = threadIdx.x; p < len; p += SELT) {
        const uint32_t v = vals[p];
        if (v >= lo && v <= hi) atomicAdd(&hist[(v - lo) >> sh], 1u);
      }
      __syncthreads();
      uint32_t h[SELB], mine = 0u;
#pragma unroll
      for (int k = 0; k < SELB; ++k) {
        const uint32_t b = threadIdx.x * SELB + k;
        h[k] = b < nb ? hist[b] : 0u;
        mine += h[k];
      }
      uint32_t incl = mine;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
      }
      if (lane == 31u) wsum[warp] = incl;
      __syncthreads();
      uint32_t cum = incl - mine;
      for (uint32_t k = 0; k < warp; ++k) cum += wsum[k];
      if (krem >= cum && krem < cum + mine) {
#pragma unroll
        for (int k = 0; k < SELB; ++k) {
          const uint32_t b = threadIdx.x * SELB + k;
          if (b < nb && krem >= cum && krem < cum + h[k]) {
            const uint32_t nlo = lo + (b << sh);
            s_lo = nlo;
            s_hi = (uint32_t)min((unsigned long long)hi, (unsigned long long)nlo + ((1ull << sh) - 1ull));
            s_krem = krem - cum;
            s_cnt = h[k];
          }
          cum += h[k];
        }
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      if (s_cnt <= SMALL_CAP) {
        s_park = 1u;
      } else if (s_lo == s_hi) {  // one value: its id digits next
        s_bits = 32u;
        s_prefix = s_lo;
      } else {  // not reached: four passes of 11 bits fix a 32-bit value
        atomicOr(err, ERRB_INTERNAL);
        s_park = 1u;
      }
    }
    __syncthreads();
    if (s_park) {
      if (threadIdx.x == 0) {
        SegSel* p = &sel[s];
        p->klo = (unsigned long long)s_lo << 32;
        p->khi = ((unsigned long long)s_hi << 32) | 0xffffffffull;
        p->krem = s_krem;
        p->cnt = s_cnt;
        p->small = s_cnt > 1u ? 1u : 0u;
        p->done = 1u;
        if (s_cnt == 0u) atomicOr(err, ERRB_INTERNAL);
      }
      return;
    }
  }
  for (int guard = 0; guard < 8; ++guard) {
    const uint32_t bits = s_bits, cnt = s_cnt, krem = s_krem;
    const unsigned long long prefix = s_prefix;
    if (bits >= 64u || cnt <= 1u) break;
    const uint32_t w = (32u - (bits & 31u)) < 11u ? (32u - (bits & 31u)) : 11u;
    const uint32_t nb = 1u << w;
    for (uint32_t i = threadIdx.x; i < nb; i += SELT) hist[i] = 0u;
    __syncthreads();
    if (bits < 32u) {
      const uint32_t vpre = (uint32_t)prefix;
      for (uint32_t p = threadIdx.x; p < len; p += SELT) {
        const uint32_t v = vals[p];
        if (bits == 0u || (v >> (32u - bits)) == vpre) atomicAdd(&hist[(v >> (32u - bits - w)) & (nb - 1u)], 1u);
      }
    } else {
      // the value is fixed: the id digits of the points holding it
      const uint32_t vpre = (uint32_t)(prefix >> (bits - 32u));
      const uint32_t ib = bits - 32u;
      const uint32_t ipre = ib ? (uint32_t)(prefix & ((1ull << ib) - 1ull)) : 0u;
      for (uint32_t p = threadIdx.x; p < len; p += SELT) {
        if (vals[p] != vpre) continue;
        const uint32_t id = __ldcs(src.ids + start + p);
        if (ib != 0u && (id >> (32u - ib)) != ipre) continue;
        atomicAdd(&hist[(id >> (32u - ib - w)) & (nb - 1u)], 1u);
      }
    }
    __syncthreads();
    // the digit holding rank krem: block scan of SELB bins per thread
    uint32_t h[SELB], mine = 0u;
#pragma unroll
    for (int k = 0; k < SELB; ++k) {
      const uint32_t b = threadIdx.x * SELB + k;
      h[k] = b < nb ? hist[b] : 0u;
      mine += h[k];
    }
    uint32_t incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
    if (lane == 31u) wsum[warp] = incl;
    __syncthreads();
    uint32_t cum = incl - mine;
    for (uint32_t k = 0; k < warp; ++k) cum += wsum[k];
    if (krem >= cum && krem < cum + mine) {
#pragma unroll
      for (int k = 0; k < SELB; ++k) {
        const uint32_t b = threadIdx.x * SELB + k;
        if (b < nb && krem >= cum && krem < cum + h[k]) {
          s_prefix = (bits == 0u ? 0ull : (prefix << w)) | b;
          s_bits = bits + w;
          s_krem = krem - cum;
          s_cnt = h[k];
        }
        cum += h[k];
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    SegSel* p = &sel[s];
    p->prefix = s_prefix;
    p->bits = s_bits;
    // the prefix as the key interval the partition classifies by
    const uint32_t b = s_bits;
    p->klo = b == 0u ? 0ull : (b >= 64u ? s_prefix : s_prefix << (64u - b));
    p->khi = b == 0u ? ~0ull : (b >= 64u ? s_prefix : (s_prefix << (64u - b)) | (~0ull >> b));
    p->krem = s_krem;
    p->cnt = s_cnt;
    p->done = 1u;
    if (s_cnt == 0u) atomicOr(err, ERRB_INTERNAL);
  }
}

// ---------------------------------------------------------------- subtree

constexpr int ST = 1024;         // threads of the subtree kernel
constexpr int SWARPS = ST / 32;
constexpr int WARPN = 32;        // segments of at most this many points finish in one warp
constexpr int MAXSEG = 256;      // segments of a shared-memory radix level (length > WARPN)
constexpr int HWORDS = 4096;     // packed 16-bit digit counters (16 KB); the scan buffer is bufB's spare row
constexpr uint16_t DONE = 0xffffu;

template <int DIM>
struct SubCfg {
  static constexpr int SUBN = DIM <= 3 ? 4096 : 3072;
  static constexpr int PPT = SUBN / ST;  // positions per thread
  static constexpr int STAGE = DIM + 4;  // words per lane of the warp-phase staging area
  static constexpr size_t smem = 2ull * (DIM + 1) * SUBN * 4 + 2ull * SUBN * 2 + HWORDS * 4ull +
                                 MAXSEG * (4 * 4 + 8 + 4 + 4 + 4 + 4) + (size_t)SWARPS * 32 * STAGE * 4;
};

int sub_capacity(int dim) { return dim <= 3 ? SubCfg<3>::SUBN : SubCfg<4>::SUBN; }

// Finishes one segment of at most 32 points (and every level below it) in the
// registers of one warp.  Lane i starts with point i of the segment; per level
// each lane counts the smaller keys of its segment through shuffles (all
// pairs), the lane whose rank is the split rank writes its node, the others
// move to position (segment start + rank) through a per-warp staging area.
template <int DIM>
__device__ void warp_finish(const Geom& g, uint32_t d1, uint32_t t1, const uint32_t* rec_base, uint32_t m0,
                            uint32_t* stage, const Table& tab, uint32_t* err) {
  constexpr int SUBN = SubCfg<DIM>::SUBN;
  constexpr int W = SubCfg<DIM>::STAGE;
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t rec[DIM + 1];
  bool valid = lane < m0;
#pragma unroll
  for (int w = 0; w <= DIM; ++w) rec[w] = valid ? rec_base[w * SUBN + lane] : 0u;
  uint32_t cur_t = t1, ls = 0u, m = m0;  // my segment: global index-in-level, first lane, length
  for (uint32_t depth = d1;; ++depth) {
    if (depth == g.H) {
      if (valid) {
        if (cur_t < g.M)
          write_node(tab, (1u << g.H) - 1u + cur_t, rec, DIM);
        else
          atomicOr(err, ERRB_INTERNAL);
      }
      break;
    }
    const uint32_t c = depth % DIM;
    const uint64_t key = order_key(pick_coord<DIM>(rec, c), rec[DIM]);
    const uint32_t mmax = __reduce_max_sync(0xffffffffu, valid ? m : 0u);
    if (mmax == 0u) break;
    uint32_t r = 0u;
    for (uint32_t i0 = 0; i0 < mmax; i0 += 4u) {
      uint64_t kq[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) kq[u] = __shfl_sync(0xffffffffu, key, (ls + i0 + u) & 31u);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint32_t i = i0 + u, srcl = (ls + i) & 31u;
        r += (valid && i < m && (kq[u] < key || (kq[u] == key && srcl < lane))) ? 1u : 0u;
      }
    }
    const uint32_t k = seg_rank(g, depth, cur_t);
    stage[lane * W + DIM + 3] = 0u;  // slot empty unless a point moves in
    __syncwarp();
    if (valid) {
      if (r == k) {
        write_node(tab, (1u << depth) - 1u + cur_t, rec, DIM);
      } else if (r < m) {
        const uint32_t dst = ls + r;
        const uint32_t ct = 2u * cur_t + (r > k ? 1u : 0u);
        uint32_t* sl = stage + dst * W;
#pragma unroll
        for (int w = 0; w <= DIM; ++w) sl[w] = rec[w];
        sl[DIM + 1] = ct;
        sl[DIM + 2] = r < k ? ls : ls + k + 1u;
        sl[DIM + 3] = 1u;
      } else {
        atomicOr(err, ERRB_INTERNAL);
      }
    }
    __syncwarp();
    const uint32_t* me = stage + lane * W;
    valid = me[DIM + 3] != 0u;
#pragma unroll
    for (int w = 0; w <= DIM; ++w) rec[w] = me[w];
    cur_t = me[DIM + 1];
    ls = me[DIM + 2];
    m = valid ? seg_len(g, depth + 1, cur_t) : 0u;
    __syncwarp();
  }
}

template <int DIM>
__global__ void __launch_bounds__(ST, 1) k_subtree(const EvDesc* __restrict__ evs, const uint2* __restrict__ subs,
                                                   CSoA src_in, CSoA src_b0, CSoA src_b1, Table tab_all,
                                                   uint32_t* __restrict__ err) {
  constexpr int SUBN = SubCfg<DIM>::SUBN;
  constexpr int PPT = SubCfg<DIM>::PPT;
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* bufA = (uint32_t*)smem;
  uint32_t* bufB = bufA + (DIM + 1) * SUBN;
  uint16_t* segA = (uint16_t*)(bufB + (DIM + 1) * SUBN);
  uint16_t* segB = segA + SUBN;
  uint32_t* work = (uint32_t*)(segB + SUBN);  // histograms / scan
  uint32_t* svmin = work + HWORDS;             // per-segment bounds of the value and id words
  uint32_t* svmax = svmin + MAXSEG;
  uint32_t* simin = svmax + MAXSEG;
  uint32_t* simax = simin + MAXSEG;
  unsigned long long* spre = (unsigned long long*)(simax + MAXSEG);
  uint32_t* sbits = (uint32_t*)(spre + MAXSEG);
  uint32_t* skrem = sbits + MAXSEG;
  uint32_t* scnt = skrem + MAXSEG;
  uint32_t* sdup = scnt + MAXSEG;
  uint32_t* stage_all = sdup + MAXSEG;
  __shared__ uint32_t wtot[SWARPS];

  // this CTA's subtree: event sb.x, root (d0, s0); positions and node indices
  // below are local to the event
  const uint2 sb = subs[blockIdx.x];
  const EvDesc ev = evs[sb.x];
  const Geom g = ev.g;
  const uint32_t d0 = ev.d0;
  const uint32_t s0 = sb.y;
  // an event's records sit where its last global level wrote them: the input
  // (no global level), buffer 0 (odd d0) or buffer 1 (even d0 >= 2)
  const CSoA src_all = d0 == 0u ? src_in : ((d0 & 1u) ? src_b0 : src_b1);
  const CSoA src{src_all.base + ev.base, src_all.ids + ev.base, src_all.stride};
  const Table tab{tab_all.nodes + ev.base, tab_all.ids + ev.base};
  const uint32_t base = seg_start(g, d0, s0);
  const uint32_t nloc = seg_len(g, d0, s0);
  if (nloc > (uint32_t)SUBN) {
    if (threadIdx.x == 0) atomicOr(err, ERRB_INTERNAL);
    return;
  }
  bool nan = false;
  for (uint32_t p = threadIdx.x; p < nloc; p += ST) {
#pragma unroll
    for (int w = 0; w < DIM; ++w) {
      const uint32_t v = __ldcs(src.base + (uint64_t)w * src.stride + base + p);
      nan |= is_nan_bits(v);
      bufA[w * SUBN + p] = v;
    }
    bufA[DIM * SUBN + p] = __ldcs(src.ids + base + p);
    segA[p] = 0;
  }
  if (nan) atomicOr(err, ERRB_NAN);
  __syncthreads();
  PROF_T(tp0);

  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t j = 0;
  for (;; ++j) {
    const uint32_t d = d0 + j;
    const uint32_t t0 = s0 << j;
    if (d >= g.H || seg_len(g, d, t0) <= (uint32_t)WARPN) break;
    const uint32_t c = d % DIM;
    const uint32_t nseg = 1u << j;
    if (nseg > (uint32_t)MAXSEG) {
      if (threadIdx.x == 0) atomicOr(err, ERRB_INTERNAL);
      return;
    }
    PROF_T(tq0);
    PROF_CNT(6);
    // the level's keys, cached in registers (positions p = tid + ST*k)
    uint32_t kv[PPT], ki[PPT], ku[PPT];
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
      const uint32_t p = threadIdx.x + ST * k;
      ku[k] = p < nloc ? segA[p] : DONE;
      kv[k] = ku[k] != DONE ? mono_bits(bufA[c * SUBN + p]) : 0u;
      ki[k] = ku[k] != DONE ? bufA[DIM * SUBN + p] : 0u;
    }
    // digit bits: about two counters per point of the widest segment, and the
    // flattened (segment, digit) counters within 2*HWORDS
    const uint32_t lmax = seg_len(g, d, t0);
    uint32_t hb = floor_log2_u32(2u * lmax - 1u) + 1u;
    if (hb > 12u) hb = 12u;
    while ((nseg << hb) > 2u * HWORDS || (nseg << hb) < (uint32_t)ST) {
      if ((nseg << hb) < (uint32_t)ST) ++hb; else --hb;
    }
    for (uint32_t u = threadIdx.x; u < nseg; u += ST) {
      svmin[u] = simin[u] = 0xffffffffu;
      svmax[u] = simax[u] = 0u;
      skrem[u] = seg_rank(g, d, t0 + u);
      scnt[u] = seg_len(g, d, t0 + u);
      sdup[u] = 0u;
    }
    __syncthreads();
    // bounds of the value and id words per segment (their common prefix is a
    // common prefix of every key of the segment)
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
      const uint32_t u = ku[k];
      const bool valid = u != DONE;
      const uint32_t u0 = __shfl_sync(0xffffffffu, u, 0);
      if (__all_sync(0xffffffffu, valid && u == u0)) {
        const uint32_t a = __reduce_min_sync(0xffffffffu, kv[k]);
        const uint32_t b = __reduce_max_sync(0xffffffffu, kv[k]);
        const uint32_t e = __reduce_min_sync(0xffffffffu, ki[k]);
        const uint32_t f = __reduce_max_sync(0xffffffffu, ki[k]);
        if (lane == 0) {
          atomicMin(&svmin[u], a);
          atomicMax(&svmax[u], b);
          atomicMin(&simin[u], e);
          atomicMax(&simax[u], f);
        }
      } else if (valid) {
        atomicMin(&svmin[u], kv[k]);
        atomicMax(&svmax[u], kv[k]);
        atomicMin(&simin[u], ki[k]);
        atomicMax(&simax[u], ki[k]);
      }
    }
    __syncthreads();
    for (uint32_t u = threadIdx.x; u < nseg; u += ST) {
      const unsigned long long lo = ((unsigned long long)svmin[u] << 32) | simin[u];
      const unsigned long long hi = ((unsigned long long)svmax[u] << 32) | simax[u];
      const uint32_t cp = lo == hi ? 64u : (uint32_t)__clzll((long long)(lo ^ hi));
      spre[u] = cp == 0u ? 0ull : (cp >= 64u ? lo : (lo >> (64u - cp)));
      sbits[u] = cp;
    }
    __syncthreads();
    for (int pass = 0; pass < 64; ++pass) {
      bool active = false;
      for (uint32_t u = threadIdx.x; u < nseg; u += ST) active |= (scnt[u] > 1u && sbits[u] < 64u);
      if (!__syncthreads_or(active)) break;
      PROF_CNT(5);
      for (uint32_t i = threadIdx.x; i < (nseg << hb) / 2u; i += ST) work[i] = 0u;
      __syncthreads();
#pragma unroll
      for (int k = 0; k < PPT; ++k) {
        const uint32_t u = ku[k];
        if (u == DONE) continue;
        const uint32_t bits = sbits[u];
        if (scnt[u] <= 1u || bits >= 64u) continue;
        const uint64_t key = ((uint64_t)kv[k] << 32) | ki[k];
        if (bits != 0u && (key >> (64u - bits)) != spre[u]) continue;
        const uint32_t w = (64u - bits) < hb ? (64u - bits) : hb;
        const uint32_t slot = (u << hb) + ((uint32_t)(key >> (64u - bits - w)) & ((1u << w) - 1u));
        atomicAdd(&work[slot >> 1], 1u << (16u * (slot & 1u)));
      }
      __syncthreads();
      {
        // CTA-wide digit search over the flattened (segment, digit) counters:
        // thread t owns counters [t*cpt, (t+1)*cpt); every segment starts on a
        // thread boundary (2^hb >= cpt).
        const uint32_t T = nseg << hb;
        const uint32_t cpt = T / ST;
        uint32_t* segbase = sdup;  // reused as scratch: exclusive counter prefix at each segment start
        uint32_t loc = 0u;
        for (uint32_t k = 0; k < cpt; ++k) {
          const uint32_t slot = threadIdx.x * cpt + k;
          loc += (work[slot >> 1] >> (16u * (slot & 1u))) & 0xffffu;
        }
        uint32_t incl = loc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= (uint32_t)o) incl += y;
        }
        if (lane == 31u) wtot[warp] = incl;
        __syncthreads();
        uint32_t excl = incl - loc;
        for (uint32_t k = 0; k < warp; ++k) excl += wtot[k];
        const uint32_t first = threadIdx.x * cpt;
        if ((first & ((1u << hb) - 1u)) == 0u) segbase[first >> hb] = excl;
        // read the segment state before anyone updates it
        const uint32_t u = first >> hb;
        const uint32_t bits = sbits[u];
        const uint32_t cntu = scnt[u];
        const uint32_t krem = skrem[u];
        const unsigned long long pre = spre[u];
        __syncthreads();
        uint32_t cum = excl - segbase[u];
        // only the thread whose counters hold rank krem walks them
        if (cntu > 1u && bits < 64u && krem >= cum && krem < cum + loc) {
          const uint32_t w = (64u - bits) < hb ? (64u - bits) : hb;
          for (uint32_t k = 0; k < cpt; ++k) {
            const uint32_t slot = first + k;
            const uint32_t b = slot & ((1u << hb) - 1u);
            const uint32_t h = (work[slot >> 1] >> (16u * (slot & 1u))) & 0xffffu;
            if (b < (1u << w) && h && krem >= cum && krem < cum + h) {
              spre[u] = (bits == 0u ? 0ull : (pre << w)) | b;
              sbits[u] = bits + w;
              skrem[u] = krem - cum;
              scnt[u] = h;
            }
            cum += h;
          }
        }
        __syncthreads();
        for (uint32_t v = threadIdx.x; v < nseg; v += ST) sdup[v] = 0u;
      }
      __syncthreads();
    }

    PROF_T(tq1);
    // Partition: flags (below | above << 16) per position, exclusive scan,
    // then each point moves to its side of its segment.
    uint32_t* scan = work;
    for (uint32_t p = threadIdx.x; p < (uint32_t)SUBN; p += ST) scan[p] = 0u;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
      const uint32_t u = ku[k];
      if (u == DONE) continue;
      const uint32_t bits = sbits[u];
      const uint64_t key = ((uint64_t)kv[k] << 32) | ki[k];
      const uint64_t top = bits >= 64u ? key : (bits == 0u ? 0ull : (key >> (64u - bits)));
      const unsigned long long pre = bits == 0u ? 0ull : spre[u];
      scan[threadIdx.x + ST * k] = top < pre ? 1u : (top > pre ? (1u << 16) : 0u);
    }
    __syncthreads();
    {
      uint32_t fl[PPT];
      uint32_t tsum = 0u;
#pragma unroll
      for (int k = 0; k < PPT; ++k) {
        fl[k] = scan[threadIdx.x * PPT + k];
        tsum += fl[k];
      }
      uint32_t incl = tsum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
      }
      if (lane == 31u) wtot[warp] = incl;
      __syncthreads();
      uint32_t wb = 0u;
      for (uint32_t k = 0; k < warp; ++k) wb += wtot[k];
      uint32_t run = wb + incl - tsum;
#pragma unroll
      for (int k = 0; k < PPT; ++k) {
        scan[threadIdx.x * PPT + k] = run;
        run += fl[k];
      }
    }
    uint32_t total = 0u;
    for (uint32_t k = 0; k < (uint32_t)SWARPS; ++k) total += wtot[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
      const uint32_t p = threadIdx.x + ST * k;
      if (p >= nloc) continue;
      const uint32_t u = ku[k];
      if (u == DONE) {
        segB[p] = DONE;
        continue;
      }
      const uint32_t t = t0 + u;
      const uint32_t ls = seg_start(g, d, t) - base;
      const uint32_t m = seg_len(g, d, t);
      const uint32_t kr = seg_rank(g, d, t);
      const uint32_t bits = sbits[u];
      const uint64_t key = ((uint64_t)kv[k] << 32) | ki[k];
      const uint64_t top = bits >= 64u ? key : (bits == 0u ? 0ull : (key >> (64u - bits)));
      const unsigned long long pre = bits == 0u ? 0ull : spre[u];
      const uint32_t sp = scan[p], s0v = scan[ls];
      uint32_t dstp;
      bool pivot = false;
      if (top < pre) {
        dstp = ls + ((sp & 0xffffu) - (s0v & 0xffffu));
      } else if (top > pre) {
        dstp = ls + kr + 1u + ((sp >> 16) - (s0v >> 16));
      } else {
        const uint32_t krem = skrem[u];
        const uint32_t ticket = scnt[u] == 1u ? krem : atomicAdd(&sdup[u], 1u);  // repeated keys only
        const uint32_t se = (ls + m < nloc) ? scan[ls + m] : total;
        const uint32_t nbelow = (se & 0xffffu) - (s0v & 0xffffu);
        const uint32_t nabove = (se >> 16) - (s0v >> 16);
        if (ticket == krem) {
          pivot = true;
          dstp = ls + kr;
        } else if (ticket < krem) {
          dstp = ls + nbelow + ticket;
        } else {
          dstp = ls + kr + 1u + nabove + (ticket - krem - 1u);
        }
      }
      if (dstp >= ls + m) {
        atomicOr(err, ERRB_INTERNAL);
        continue;
      }
      uint32_t rec[DIM + 1];
#pragma unroll
      for (int w = 0; w <= DIM; ++w) rec[w] = bufA[w * SUBN + p];
      if (pivot) {
        write_node(tab, (1u << d) - 1u + t, rec, DIM);
        segB[dstp] = DONE;
      } else {
#pragma unroll
        for (int w = 0; w <= DIM; ++w) bufB[w * SUBN + dstp] = rec[w];
        segB[dstp] = (uint16_t)(dstp < ls + kr ? 2u * u : 2u * u + 1u);
      }
    }
    __syncthreads();
    PROF_T(tq2);
    PROF_ADD(2, tq0, tq1);
    PROF_ADD(3, tq1, tq2);
    uint32_t* tb = bufA;
    bufA = bufB;
    bufB = tb;
    uint16_t* ts = segA;
    segA = segB;
    segB = ts;
  }

  PROF_T(tp1);
  PROF_ADD(0, tp0, tp1);
  // Warp phase: every segment of level j is at most WARPN points long.
  const uint32_t d1 = d0 + j;
  const uint32_t t0 = s0 << j;
  const uint32_t nseg = 1u << j;
  uint32_t* stage = stage_all + warp * 32 * SubCfg<DIM>::STAGE;
  for (uint32_t u = warp; u < nseg; u += SWARPS) {
    const uint32_t t = t0 + u;
    const uint32_t m = seg_len(g, d1, t);
    if (m > (uint32_t)WARPN) {
      if (lane == 0) atomicOr(err, ERRB_INTERNAL);
      continue;
    }
    const uint32_t ls = seg_start(g, d1, t) - base;
    warp_finish<DIM>(g, d1, t, bufA + ls, m, stage, tab, err);
  }
  PROF_T(tp2);
  PROF_ADD(1, tp1, tp2);
}

// ---------------------------------------------------------------- host

template <int DIM>
static cudaError_t run_build(BuildCtx& bc) {
  CSoA src = bc.input;
  SoA bufs[2] = {bc.work[0], bc.work[1]};
  const CSoA b0{bufs[0].base, bufs[0].ids, bufs[0].stride}, b1{bufs[1].base, bufs[1].ids, bufs[1].stride};
  int nb = 0;
  for (uint32_t d = 0; d < bc.nlevels; ++d) {
    const LevelPlan& lp = bc.levels[d];
    if (lp.nseg == 0) continue;
    // levels of small segments: one CTA selects a whole segment (no learned bracket there)
    const bool small = lp.maxlen <= (uint32_t)SEL_MAX && bc.small_select;
    // per-segment bounds: written by level d - 1's partition into bnd[d & 1],
    // by level d's partition into bnd[(d + 1) & 1]; level 0's by k_bounds0
    const uint2* bnd_in = (bc.bnd && d > 0) ? bc.bnd + (size_t)(d & 1u) * bc.bnd_stride : nullptr;
    uint2* bnd_out = bc.bnd ? bc.bnd + (size_t)((d + 1u) & 1u) * bc.bnd_stride : nullptr;
    bool inv = false;
    if (d == 0 && bc.bnd && bc.lin && !small) {
      cudaError_t e = cudaMemsetAsync(bc.bnd, 0, sizeof(uint2) * lp.nseg, bc.stream);
      if (e != cudaSuccess) return e;
      k_bounds0<DIM><<<(lp.nptile + B0_TILES - 1) / B0_TILES, GT, 0, bc.stream>>>(bc.evs, lp.segs, lp.ptiles,
                                                                                lp.nptile, src, bc.bnd);
      count_launches(1);
      bnd_in = bc.bnd;
      inv = true;
    }
    k_sel_init<<<(lp.nseg + 255) / 256, 256, 0, bc.stream>>>(d, bc.evs, lp.segs, lp.nseg, bc.sel, bc.pending, bnd_in,
                                                            inv, bnd_out, lp.child, bc.lin && !small);
    count_launches(1);
    const LearnCtx& lc = bc.learn;
    if (lc.rec_x || (lc.params && !small)) {
      cudaError_t e = launch_features(d, bc.evs, lp.segs, lp.nseg, src, DIM, lc.feat, lc.range, bc.stream);
      if (e != cudaSuccess) return e;
    }
    if (small) {
      const size_t sm = (size_t)lp.maxlen * sizeof(uint32_t);
      const bool few = lp.maxlen <= (uint32_t)SEL_FEW;
      const bool many = lp.maxlen > (uint32_t)SEL_MANY;
      cudaError_t e =
          few ? cudaFuncSetAttribute(k_select_small<DIM, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)
              : many ? cudaFuncSetAttribute(k_select_small<DIM, 1024>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)sm)
                     : cudaFuncSetAttribute(k_select_small<DIM, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)sm);
      if (e != cudaSuccess) return e;
      if (few)
        k_select_small<DIM, 128><<<lp.nseg, 128, sm, bc.stream>>>(d, bc.evs, lp.segs, src, bc.sel, bc.err,
                                                                  bc.tiebuf != nullptr);
      else if (many)
        k_select_small<DIM, 1024><<<lp.nseg, 1024, sm, bc.stream>>>(d, bc.evs, lp.segs, src, bc.sel, bc.err,
                                                                    bc.tiebuf != nullptr);
      else
        k_select_small<DIM, 512><<<lp.nseg, 512, sm, bc.stream>>>(d, bc.evs, lp.segs, src, bc.sel, bc.err,
                                                                  bc.tiebuf != nullptr);
      count_launches(1);
    } else if (lc.params) {
      cudaError_t e = mlp_infer(lc.params, lc.feat, lp.nseg, lc.yhat, bc.stream);
      if (e == cudaSuccess)
        e = launch_bracket(d, bc.evs, lp.segs, lp.nseg, lc.yhat, lc.range, lc.delta, bc.sel, lc.stats, bc.stream);
      if (e != cudaSuccess) return e;
    }
    // the plain select needs at most 6 passes; a failed prediction costs one more
    const int passes = small ? 0 : (lc.params ? RPASSES : RPASSES - 1);
    for (int pass = 0; pass < passes; ++pass) {
      k_hist<DIM><<<lp.nhtile, GT, 0, bc.stream>>>(d, bc.evs, lp.segs, lp.htiles, lp.hts, src, bc.sel, bc.ghist,
                                                    bc.pending + pass, bc.pending + pass + 1, bc.err, lc.stats,
                                                    bc.tiebuf ? 1u : 0u);
      count_launches(1);
    }
    SoA dst = bufs[nb];
    k_partition<DIM><<<lp.nptile, GT, 0, bc.stream>>>(d, bc.evs, lp.segs, lp.ptiles, src, dst, bc.sel, bc.tab,
                                                        bc.err, bnd_out, lp.child, bc.tiebuf);
    count_launches(1);
    if (bc.tiebuf) {
      k_small_fix<DIM><<<(lp.nseg + 7) / 8, 256, 0, bc.stream>>>(d, bc.evs, lp.segs, lp.nseg, bc.sel, bc.tiebuf, dst,
                                                                bc.tab, bc.err, bnd_out, lp.child);
      count_launches(1);
    }
    if (lc.rec_x) {
      cudaError_t e = launch_record(d, bc.evs, lp.segs, lp.nseg, DIM, bc.tab, lc.feat, lc.range, lc.rec_x, lc.rec_t,
                                    lc.rec_n, lc.rec_cap, bc.stream);
      if (e != cudaSuccess) return e;
    }
    src = CSoA{dst.base, dst.ids, dst.stride};
    nb ^= 1;
  }
  const size_t smem = SubCfg<DIM>::smem;
  cudaError_t e = cudaFuncSetAttribute(k_subtree<DIM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (bc.ev_sub) {
    e = cudaEventRecord(bc.ev_sub, bc.stream);
    if (e != cudaSuccess) return e;
  }
  if (bc.nsub) {
    if (DIM <= 3 && bc.subtree != 1)
      return launch_subtree_sorted(bc.evs, bc.subs, bc.nsub, bc.input, b0, b1, bc.tab, bc.err, DIM, bc.subn,
                                   bc.stream);
    k_subtree<DIM><<<bc.nsub, ST, smem, bc.stream>>>(bc.evs, bc.subs, bc.input, b0, b1, bc.tab, bc.err);
    count_launches(1);
  }
  return cudaGetLastError();
}

uint32_t build_global_levels(uint32_t n, int dim, int subn) {
  if (n == 0) return 0;
  const Geom g = make_geom(n);
  // the global levels stop where every interval fits the subtree kernel
  // (dims 1-3: the presorted-list kernel's size, which the radix kernel also takes)
  const uint32_t cap = (uint32_t)(dim <= 3 ? sorted_sub_capacity(subn) : sub_capacity(dim));
  uint32_t d0 = 0;
  while (seg_len(g, d0, 0) > cap) ++d0;
  return d0;
}

template <int DIM>
static cudaError_t run_subtree_direct(const EvDesc* evs, const uint2* subs, uint32_t nsub, CSoA src, Table tab,
                                     uint32_t* err, cudaStream_t stream) {
  const size_t smem = SubCfg<DIM>::smem;
  cudaError_t e = cudaFuncSetAttribute(k_subtree<DIM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_subtree<DIM><<<nsub, ST, smem, stream>>>(evs, subs, src, src, src, tab, err);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_subtree_direct(const EvDesc* evs, const uint2* subs, uint32_t nsub, CSoA src, Table tab,
                                  uint32_t* err, int dim, cudaStream_t stream) {
  switch (dim) {
    case 1: return run_subtree_direct<1>(evs, subs, nsub, src, tab, err, stream);
    case 2: return run_subtree_direct<2>(evs, subs, nsub, src, tab, err, stream);
    case 3: return run_subtree_direct<3>(evs, subs, nsub, src, tab, err, stream);
    case 4: return run_subtree_direct<4>(evs, subs, nsub, src, tab, err, stream);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_build(BuildCtx& bc, int dim) {
  switch (dim) {
    case 1: return run_build<1>(bc);
    case 2: return run_build<2>(bc);
    case 3: return run_build<3>(bc);
    case 4: return run_build<4>(bc);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fkd
