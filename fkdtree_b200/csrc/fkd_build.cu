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
#include "fkd_internal.h"

namespace fkd {

// ---------------------------------------------------------------- global

constexpr int GT = 256;            // threads of the global-level kernels
constexpr int GIPT = 16;           // records per thread (digit passes)
constexpr int PIPT = 8;            // records per thread (partition)
constexpr int PTILE = GT * PIPT;
constexpr int GTILE = GT * GIPT;   // records per CTA tile
constexpr int GWARPS = GT / 32;
constexpr int RBITS = 11;          // digit width of the global select
constexpr int RBINS = 1 << RBITS;
constexpr int RPASSES = 6;         // 5 * 11 + 9 >= 64

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

__global__ void k_sel_init(Geom g, uint32_t d, SegSel* __restrict__ sel, uint32_t* __restrict__ pending) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s == 0) {
    // pending[p] != 0: digit pass p has a segment to work on
    pending[0] = 1u;
    for (int p = 1; p <= RPASSES; ++p) pending[p] = 0u;
  }
  if (s >= (1u << d)) return;
  const uint32_t len = seg_len(g, d, s);
  SegSel st;
  st.prefix = 0ull;
  st.bits = 0u;
  st.krem = (d < g.H) ? seg_rank(g, d, s) : 0u;
  st.cnt = len;
  st.done = len <= 1u ? 1u : 0u;
  st.tiles_done = 0u;
  st.curL = st.curR = st.curE = 0u;
  st.pad = 0u;
  sel[s] = st;
}

// One digit pass of the segmented select for every segment of depth d.
template <int DIM>
__global__ void __launch_bounds__(GT) k_hist(Geom g, uint32_t d, uint32_t tps, CSoA src, SegSel* __restrict__ sel,
                                             uint32_t* __restrict__ ghist, const uint32_t* __restrict__ pending_now,
                                             uint32_t* __restrict__ pending_next, uint32_t* __restrict__ err) {
  __shared__ uint32_t hist[RBINS];
  __shared__ uint32_t wsum[GWARPS];
  __shared__ uint32_t s_last;
  // pending_now was raised by the previous pass when some segment still needs
  // a digit; without it the whole launch is a no-op.
  if (*(volatile const uint32_t*)pending_now == 0u) return;
  const uint32_t s = blockIdx.x / tps, t = blockIdx.x - s * tps;
  const uint32_t len = seg_len(g, d, s);
  const uint32_t ntiles = (len + GTILE - 1) / GTILE;
  if (t >= ntiles) return;
  if (sel[s].done) return;
  const uint32_t bits = sel[s].bits;
  const unsigned long long prefix = sel[s].prefix;
  const uint32_t w = (64u - bits) < (uint32_t)RBITS ? (64u - bits) : (uint32_t)RBITS;
  const uint32_t nb = 1u << w;
  const uint32_t shift = 64u - bits - w;
  const bool need_id = bits + w > 32u;
  const uint32_t c = d % DIM;
  const uint32_t start = seg_start(g, d, s);
  const uint32_t t0 = start + t * GTILE;
  const uint32_t t1 = min(start + len, t0 + (uint32_t)GTILE);
  for (uint32_t i = threadIdx.x; i < nb; i += GT) hist[i] = 0u;
  __syncthreads();

  const uint32_t* X = src.base + (uint64_t)c * src.stride;
  uint32_t vb[GIPT], idv[GIPT];
#pragma unroll
  for (int k = 0; k < GIPT; ++k) {
    const uint32_t e = t0 + k * GT + threadIdx.x;
    vb[k] = e < t1 ? __ldcs(X + e) : 0u;
  }
  if (need_id) {
#pragma unroll
    for (int k = 0; k < GIPT; ++k) {
      const uint32_t e = t0 + k * GT + threadIdx.x;
      idv[k] = e < t1 ? __ldcs(src.ids + e) : 0u;
    }
  } else {
#pragma unroll
    for (int k = 0; k < GIPT; ++k) idv[k] = 0u;
  }
#pragma unroll
  for (int k = 0; k < GIPT; ++k) {
    const uint32_t e = t0 + k * GT + threadIdx.x;
    uint32_t dig = 0xffffffffu;  // no digit: outside the tile or prefix mismatch
    if (e < t1) {
      const uint64_t key = order_key(vb[k], idv[k]);
      if (bits == 0u || (key >> (64u - bits)) == prefix) dig = (uint32_t)(key >> shift) & (nb - 1u);
    }
    // lanes with the same digit add once (clustered data piles onto few bins);
    // all 32 lanes take part in the match
    const uint32_t peers = __match_any_sync(0xffffffffu, dig);
    if (dig != 0xffffffffu && (threadIdx.x & 31u) == (uint32_t)(__ffs(peers) - 1))
      atomicAdd(&hist[dig], (uint32_t)__popc(peers));
  }
  __syncthreads();
  uint32_t* gh = ghist + (uint64_t)s * RBINS;
  for (uint32_t i = threadIdx.x; i < nb; i += GT) {
    const uint32_t v = hist[i];
    if (v) atomicAdd(&gh[i], v);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&sel[s].tiles_done, 1u) == ntiles - 1u) ? 1u : 0u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();

  // Last CTA of segment s: locate the digit holding rank krem.
  const uint32_t krem = *(volatile uint32_t*)&sel[s].krem;
  constexpr int BPT = RBINS / GT;  // bins per thread
  uint32_t h[BPT];
  uint32_t mine = 0u;
#pragma unroll
  for (int k = 0; k < BPT; ++k) {
    const uint32_t b = threadIdx.x * BPT + k;
    h[k] = b < nb ? __ldcg(gh + b) : 0u;
    mine += h[k];
  }
  // block exclusive scan of `mine`
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t incl = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (uint32_t)o) incl += y;
  }
  if (lane == 31u) wsum[warp] = incl;
  __syncthreads();
  uint32_t wbase = 0u;
  for (uint32_t k = 0; k < warp; ++k) wbase += wsum[k];
  uint32_t cum = wbase + incl - mine;
#pragma unroll
  for (int k = 0; k < BPT; ++k) {
    const uint32_t b = threadIdx.x * BPT + k;
    if (b < nb && krem >= cum && krem < cum + h[k]) {
      SegSel* p = &sel[s];
      const uint32_t nbits = bits + w;
      p->prefix = (w == 64u ? 0ull : (prefix << w)) | (unsigned long long)b;
      p->bits = nbits;
      p->krem = krem - cum;
      p->cnt = h[k];
      p->done = (h[k] == 1u || nbits == 64u) ? 1u : 0u;
      if (!p->done) *pending_next = 1u;
    }
    cum += h[k];
  }
  for (uint32_t b = threadIdx.x; b < nb; b += GT) gh[b] = 0u;
  if (threadIdx.x == 0) sel[s].tiles_done = 0u;
  // wbase + incl of the last thread is the number of matching records; it must
  // cover krem, otherwise the select state is inconsistent.
  if (threadIdx.x == GT - 1 && krem >= wbase + incl) atomicOr(err, ERRB_INTERNAL);
}

template <int DIM>
__device__ __forceinline__ uint32_t pick_coord(const uint32_t* rec, uint32_t c) {
  uint32_t v = rec[0];
#pragma unroll
  for (int w = 1; w < DIM; ++w) v = (c == (uint32_t)w) ? rec[w] : v;
  return v;
}

// Streams every record of depth-d segments once: records below the pivot go
// to [start, start + rank), the pivot to the table, the rest above it.
template <int DIM>
__global__ void __launch_bounds__(GT, 2) k_partition(Geom g, uint32_t d, uint32_t tps, CSoA src, SoA dst,
                                                     SegSel* __restrict__ sel, Table tab, uint32_t* __restrict__ err) {
  __shared__ uint32_t sL[PIPT * GWARPS], sR[PIPT * GWARPS];
  __shared__ uint32_t s_base[2];
  const uint32_t s = blockIdx.x / tps, t = blockIdx.x - s * tps;
  const uint32_t len = seg_len(g, d, s);
  const uint32_t ntiles = (len + PTILE - 1) / PTILE;
  if (t >= ntiles) return;
  const uint32_t start = seg_start(g, d, s);
  const uint32_t rank = seg_rank(g, d, s);
  const uint32_t t0 = start + t * PTILE;
  const uint32_t t1 = min(start + len, t0 + (uint32_t)PTILE);
  const uint32_t bits = sel[s].bits;
  const unsigned long long prefix = sel[s].prefix;
  const uint32_t cnt = sel[s].cnt;
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
  uint32_t bl[PIPT], br[PIPT];
  uint32_t eqmask = 0u;  // bit k: record k matches the pivot prefix
  bool nan = false;
#pragma unroll
  for (int k = 0; k < PIPT; ++k) {
    const uint32_t e = t0 + k * GT + threadIdx.x;
    uint32_t cls = 3u;  // 0 below, 1 equal, 2 above, 3 none
    if (e < t1) {
#pragma unroll
      for (int w = 0; w < DIM; ++w) nan |= is_nan_bits(rec[k][w]);
      const uint64_t key = order_key(pick_coord<DIM>(rec[k], c), rec[k][DIM]);
      if (bits == 0u) {
        cls = 1u;
      } else {
        const uint64_t top = bits >= 64u ? key : (key >> (64u - bits));
        cls = top < prefix ? 0u : (top > prefix ? 2u : 1u);
      }
    }
    if (cls == 1u) eqmask |= 1u << k;
    bl[k] = __ballot_sync(0xffffffffu, cls == 0u);
    br[k] = __ballot_sync(0xffffffffu, cls == 2u);
    if (lane == 0) {
      sL[k * GWARPS + warp] = __popc(bl[k]);
      sR[k * GWARPS + warp] = __popc(br[k]);
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
  const uint32_t baseL = start + s_base[0], baseR = endL + 1u + s_base[1];
#pragma unroll
  for (int k = 0; k < PIPT; ++k) {
    uint32_t pos = 0xffffffffu, lim = 0u;
    if ((bl[k] >> lane) & 1u) {
      pos = baseL + sL[k * GWARPS + warp] + __popc(bl[k] & lt);
      lim = endL;
    } else if ((br[k] >> lane) & 1u) {
      pos = baseR + sR[k * GWARPS + warp] + __popc(br[k] & lt);
      lim = endR;
    } else if ((eqmask >> k) & 1u) {
      const uint32_t krem = sel[s].krem;
      uint32_t ticket = 0u;
      if (cnt != 1u) ticket = atomicAdd(&sel[s].curE, 1u);  // repeated (coordinate, id) keys only
      if (ticket == krem) {
        write_node(tab, (1u << d) - 1u + s, rec[k], DIM);
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
      } else {
        atomicOr(err, ERRB_INTERNAL);
      }
    }
  }
}

// ---------------------------------------------------------------- subtree

constexpr int ST = 512;          // threads of the subtree kernel
constexpr int SWARPS = ST / 32;
constexpr int SMALL = 16;        // rank counting at or below this segment length
constexpr int MAXSEG = 256;      // segments of a radix level (length > SMALL)
constexpr int HWORDS = 8192;     // packed 16-bit digit counters (32 KB), also the scan buffer
constexpr uint16_t DONE = 0xffffu;

template <int DIM>
struct SubCfg {
  static constexpr int SUBN = DIM <= 3 ? 4096 : 3072;
  static constexpr int PPT = SUBN / ST;  // positions per thread in the scan
  static constexpr size_t smem =
      2ull * (DIM + 1) * SUBN * 4 + 2ull * SUBN * 2 + HWORDS * 4ull + MAXSEG * (8 + 8 + 8 + 4 + 4 + 4 + 4);
};

int sub_capacity(int dim) { return dim <= 3 ? SubCfg<3>::SUBN : SubCfg<4>::SUBN; }

template <int DIM>
__device__ __forceinline__ uint64_t skey(const uint32_t* buf, uint32_t p, uint32_t c) {
  constexpr int SUBN = SubCfg<DIM>::SUBN;
  return order_key(buf[c * SUBN + p], buf[DIM * SUBN + p]);
}

template <int DIM>
__global__ void __launch_bounds__(ST, 1) k_subtree(Geom g, uint32_t d0, CSoA src, Table tab,
                                                   uint32_t* __restrict__ err) {
  constexpr int SUBN = SubCfg<DIM>::SUBN;
  constexpr int PPT = SubCfg<DIM>::PPT;
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* bufA = (uint32_t*)smem;
  uint32_t* bufB = bufA + (DIM + 1) * SUBN;
  uint16_t* segA = (uint16_t*)(bufB + (DIM + 1) * SUBN);
  uint16_t* segB = segA + SUBN;
  uint32_t* work = (uint32_t*)(segB + SUBN);  // histograms / scan
  unsigned long long* smin = (unsigned long long*)(work + HWORDS);
  unsigned long long* smax = smin + MAXSEG;
  unsigned long long* spre = smax + MAXSEG;
  uint32_t* sbits = (uint32_t*)(spre + MAXSEG);
  uint32_t* skrem = sbits + MAXSEG;
  uint32_t* scnt = skrem + MAXSEG;
  uint32_t* sdup = scnt + MAXSEG;
  __shared__ uint32_t wtot[SWARPS];

  const uint32_t s0 = blockIdx.x;
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

  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  for (uint32_t j = 0;; ++j) {
    const uint32_t d = d0 + j;
    if (d == g.H) {
      // Last level: every live position is a single-point node.
      for (uint32_t p = threadIdx.x; p < nloc; p += ST) {
        const uint32_t u = segA[p];
        if (u == DONE) continue;
        uint32_t rec[DIM + 1];
#pragma unroll
        for (int w = 0; w <= DIM; ++w) rec[w] = bufA[w * SUBN + p];
        const uint32_t t = (s0 << j) + u;
        if (t < g.M)
          write_node(tab, (1u << g.H) - 1u + t, rec, DIM);
        else
          atomicOr(err, ERRB_INTERNAL);
      }
      break;
    }
    const uint32_t c = d % DIM;
    const uint32_t nseg = 1u << j;
    const uint32_t t0 = s0 << j;
    const uint32_t lmax = seg_len(g, d, t0);

    if (lmax <= (uint32_t)SMALL) {
      // Rank counting: each point counts the smaller keys of its segment; the
      // rank is its position, the rank-k point is the node.
      for (uint32_t p = threadIdx.x; p < nloc; p += ST) {
        const uint32_t u = segA[p];
        if (u == DONE) {
          segB[p] = DONE;
          continue;
        }
        const uint32_t t = t0 + u;
        const uint32_t ls = seg_start(g, d, t) - base;
        const uint32_t m = seg_len(g, d, t);
        const uint32_t k = seg_rank(g, d, t);
        const uint64_t key = skey<DIM>(bufA, p, c);
        uint32_t r = 0;
        for (uint32_t q = ls; q < ls + m; ++q) {
          const uint64_t kq = skey<DIM>(bufA, q, c);
          r += (kq < key || (kq == key && q < p)) ? 1u : 0u;
        }
        const uint32_t dstp = ls + r;
        if (dstp >= nloc) {
          atomicOr(err, ERRB_INTERNAL);
          continue;
        }
        uint32_t rec[DIM + 1];
#pragma unroll
        for (int w = 0; w <= DIM; ++w) rec[w] = bufA[w * SUBN + p];
        if (r == k) {
          write_node(tab, (1u << d) - 1u + t, rec, DIM);
          segB[dstp] = DONE;
        } else {
#pragma unroll
          for (int w = 0; w <= DIM; ++w) bufB[w * SUBN + dstp] = rec[w];
          segB[dstp] = (uint16_t)(r < k ? 2u * u : 2u * u + 1u);
        }
      }
    } else {
      // Radix select per segment with a common-prefix skip.
      if (nseg > (uint32_t)MAXSEG) {
        if (threadIdx.x == 0) atomicOr(err, ERRB_INTERNAL);
        return;
      }
      uint32_t hb = 8u;  // digit bits so that nseg << hb fits 2*HWORDS counters
      while ((nseg << hb) > 2u * HWORDS) --hb;
      for (uint32_t u = threadIdx.x; u < nseg; u += ST) {
        smin[u] = ~0ull;
        smax[u] = 0ull;
        skrem[u] = seg_rank(g, d, t0 + u);
        sdup[u] = 0u;
      }
      __syncthreads();
      for (uint32_t p0 = 0; p0 < nloc; p0 += ST) {
        const uint32_t p = p0 + threadIdx.x;
        const uint32_t u = p < nloc ? segA[p] : DONE;
        const bool valid = u != DONE;
        unsigned long long kmin = valid ? skey<DIM>(bufA, p, c) : ~0ull;
        unsigned long long kmax = valid ? kmin : 0ull;
        // a warp whose lanes all sit in one segment reduces before the atomics
        // (every lane executes the shuffle and the vote)
        const uint32_t u0 = __shfl_sync(0xffffffffu, u, 0);
        const bool same = valid && u == u0;
        if (__all_sync(0xffffffffu, same)) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long a = __shfl_xor_sync(0xffffffffu, kmin, o);
            const unsigned long long b = __shfl_xor_sync(0xffffffffu, kmax, o);
            kmin = a < kmin ? a : kmin;
            kmax = b > kmax ? b : kmax;
          }
          if (lane == 0) {
            atomicMin(&smin[u], kmin);
            atomicMax(&smax[u], kmax);
          }
        } else if (valid) {
          atomicMin(&smin[u], kmin);
          atomicMax(&smax[u], kmax);
        }
      }
      __syncthreads();
      for (uint32_t u = threadIdx.x; u < nseg; u += ST) {
        const unsigned long long lo = smin[u], hi = smax[u];
        const uint32_t cp = lo == hi ? 64u : (uint32_t)__clzll((long long)(lo ^ hi));
        spre[u] = cp == 0u ? 0ull : (cp >= 64u ? lo : (lo >> (64u - cp)));
        sbits[u] = cp;
        scnt[u] = seg_len(g, d, t0 + u);
      }
      __syncthreads();
      for (int pass = 0; pass < 64; ++pass) {
        // a segment is resolved when one point matches its prefix or the full
        // key is known
        bool active = false;
        for (uint32_t u = threadIdx.x; u < nseg; u += ST) active |= (scnt[u] > 1u && sbits[u] < 64u);
        if (!__syncthreads_or(active)) break;
        for (uint32_t i = threadIdx.x; i < (nseg << hb) / 2u; i += ST) work[i] = 0u;
        __syncthreads();
        for (uint32_t p0 = 0; p0 < nloc; p0 += ST) {
          const uint32_t p = p0 + threadIdx.x;
          uint32_t slot = 0xffffffffu;
          const uint32_t u = p < nloc ? segA[p] : DONE;
          if (u != DONE) {
            const uint32_t bits = sbits[u];
            if (scnt[u] > 1u && bits < 64u) {
              const uint64_t key = skey<DIM>(bufA, p, c);
              if (bits == 0u || (key >> (64u - bits)) == spre[u]) {
                const uint32_t w = (64u - bits) < hb ? (64u - bits) : hb;
                const uint32_t dig = (uint32_t)(key >> (64u - bits - w)) & ((1u << w) - 1u);
                slot = (u << hb) + dig;
              }
            }
          }
          // lanes hitting the same counter add once
          const uint32_t peers = __match_any_sync(0xffffffffu, slot);
          if (slot != 0xffffffffu && lane == (uint32_t)(__ffs(peers) - 1))
            atomicAdd(&work[slot >> 1], (uint32_t)__popc(peers) << (16u * (slot & 1u)));
        }
        __syncthreads();
        // warp per segment: find the digit holding krem
        for (uint32_t u = warp; u < nseg; u += SWARPS) {
          const uint32_t bits = sbits[u];
          if (scnt[u] <= 1u || bits >= 64u) continue;
          const uint32_t w = (64u - bits) < hb ? (64u - bits) : hb;
          const uint32_t nb = 1u << w;
          const uint32_t krem = skrem[u];
          uint32_t found = 0xffffffffu, fcum = 0u, fh = 0u;
          uint32_t carry = 0u;
          for (uint32_t b0 = 0; b0 < nb; b0 += 32u) {
            const uint32_t b = b0 + lane;
            uint32_t h = 0u;
            if (b < nb) {
              const uint32_t slot = (u << hb) + b;
              h = (work[slot >> 1] >> (16u * (slot & 1u))) & 0xffffu;
            }
            uint32_t incl = h;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
              const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
              if (lane >= (uint32_t)o) incl += y;
            }
            const uint32_t cum = carry + incl - h;
            const bool hit = b < nb && krem >= cum && krem < cum + h;
            const uint32_t bal = __ballot_sync(0xffffffffu, hit);
            if (bal) {
              const uint32_t src_lane = __ffs(bal) - 1u;
              found = __shfl_sync(0xffffffffu, b, src_lane);
              fcum = __shfl_sync(0xffffffffu, cum, src_lane);
              fh = __shfl_sync(0xffffffffu, h, src_lane);
              break;
            }
            carry += __shfl_sync(0xffffffffu, incl, 31);
          }
          if (lane == 0) {
            if (found == 0xffffffffu) {
              atomicOr(err, ERRB_INTERNAL);
              scnt[u] = 1u;  // stop selecting; the partition check reports it
            } else {
              spre[u] = (bits == 0u ? 0ull : (spre[u] << w)) | found;
              sbits[u] = bits + w;
              skrem[u] = krem - fcum;
              scnt[u] = fh;
            }
          }
        }
        __syncthreads();
      }

      // Partition: exclusive scan of packed (below | above << 16) flags over
      // all positions, then each point moves to its side of its segment.
      uint32_t* scan = work;
      // flags in a strided pass (conflict-free), scan over contiguous chunks
      for (uint32_t p = threadIdx.x; p < (uint32_t)SUBN; p += ST) {
        uint32_t f = 0u;
        if (p < nloc) {
          const uint32_t u = segA[p];
          if (u != DONE) {
            const uint32_t bits = sbits[u];
            const uint64_t key = skey<DIM>(bufA, p, c);
            const uint64_t top = bits >= 64u ? key : (bits == 0u ? 0ull : (key >> (64u - bits)));
            const unsigned long long pre = bits == 0u ? 0ull : spre[u];
            f = top < pre ? 1u : (top > pre ? (1u << 16) : 0u);
          }
        }
        scan[p] = f;
      }
      __syncthreads();
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
      uint32_t total = 0u;
      for (uint32_t k = 0; k < (uint32_t)SWARPS; ++k) total += wtot[k];
      __syncthreads();
      for (uint32_t p = threadIdx.x; p < nloc; p += ST) {
        const uint32_t u = segA[p];
        if (u == DONE) {
          segB[p] = DONE;
          continue;
        }
        const uint32_t t = t0 + u;
        const uint32_t ls = seg_start(g, d, t) - base;
        const uint32_t m = seg_len(g, d, t);
        const uint32_t k = seg_rank(g, d, t);
        const uint32_t bits = sbits[u];
        const uint64_t key = skey<DIM>(bufA, p, c);
        const uint64_t top = bits >= 64u ? key : (bits == 0u ? 0ull : (key >> (64u - bits)));
        const unsigned long long pre = bits == 0u ? 0ull : spre[u];
        const uint32_t sp = scan[p], s0v = scan[ls];
        uint32_t dstp;
        bool pivot = false;
        if (top < pre) {
          dstp = ls + ((sp & 0xffffu) - (s0v & 0xffffu));
        } else if (top > pre) {
          dstp = ls + k + 1u + ((sp >> 16) - (s0v >> 16));
        } else {
          const uint32_t krem = skrem[u];
          const uint32_t ticket = scnt[u] == 1u ? krem : atomicAdd(&sdup[u], 1u);
          const uint32_t se = (ls + m < nloc) ? scan[ls + m] : total;
          const uint32_t nbelow = (se & 0xffffu) - (s0v & 0xffffu);
          const uint32_t nabove = (se >> 16) - (s0v >> 16);
          if (ticket == krem) {
            pivot = true;
            dstp = ls + k;
          } else if (ticket < krem) {
            dstp = ls + nbelow + ticket;
          } else {
            dstp = ls + k + 1u + nabove + (ticket - krem - 1u);
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
          segB[dstp] = (uint16_t)(dstp < ls + k ? 2u * u : 2u * u + 1u);
        }
      }
    }
    __syncthreads();
    uint32_t* tb = bufA;
    bufA = bufB;
    bufB = tb;
    uint16_t* ts = segA;
    segA = segB;
    segB = ts;
  }
}

// ---------------------------------------------------------------- host

template <int DIM>
static cudaError_t run_build(BuildCtx& bc) {
  const Geom g = bc.g;
  const int SUBN = SubCfg<DIM>::SUBN;
  uint32_t d0 = 0;
  while (seg_len(g, d0, 0) > (uint32_t)SUBN) ++d0;
  CSoA src = bc.input;
  SoA bufs[2] = {bc.work[0], bc.work[1]};
  int nb = 0;
  for (uint32_t d = 0; d < d0; ++d) {
    const uint32_t S = 1u << d;
    const uint32_t tps = (seg_len(g, d, 0) + GTILE - 1) / GTILE;
    const uint32_t ptps = (seg_len(g, d, 0) + PTILE - 1) / PTILE;
    k_sel_init<<<(S + 255) / 256, 256, 0, bc.stream>>>(g, d, bc.sel, bc.pending);
    count_launches(1);
    for (int pass = 0; pass < RPASSES; ++pass) {
      k_hist<DIM><<<S * tps, GT, 0, bc.stream>>>(g, d, tps, src, bc.sel, bc.ghist, bc.pending + pass,
                                                  bc.pending + pass + 1, bc.err);
      count_launches(1);
    }
    SoA dst = bufs[nb];
    k_partition<DIM><<<S * ptps, GT, 0, bc.stream>>>(g, d, ptps, src, dst, bc.sel, bc.tab, bc.err);
    count_launches(1);
    src = CSoA{dst.base, dst.ids, dst.stride};
    nb ^= 1;
  }
  const size_t smem = SubCfg<DIM>::smem;
  cudaError_t e = cudaFuncSetAttribute(k_subtree<DIM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_subtree<DIM><<<1u << d0, ST, smem, bc.stream>>>(g, d0, src, bc.tab, bc.err);
  count_launches(1);
  return cudaGetLastError();
}

uint32_t build_global_levels(uint32_t n, int dim) {
  const Geom g = make_geom(n);
  const uint32_t subn = (uint32_t)sub_capacity(dim);
  uint32_t d0 = 0;
  if (n == 0) return 0;
  while (seg_len(g, d0, 0) > subn) ++d0;
  return d0;
}

size_t build_ghist_words(uint32_t n, int dim) {
  const uint32_t d0 = build_global_levels(n, dim);
  return d0 ? (size_t)(1u << (d0 - 1)) * RBINS : 0;
}

cudaError_t launch_build(BuildCtx& bc, int dim) {
  if (bc.g.n == 0) return cudaSuccess;
  switch (dim) {
    case 1: return run_build<1>(bc);
    case 2: return run_build<2>(bc);
    case 3: return run_build<3>(bc);
    case 4: return run_build<4>(bc);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fkd
