// fkd_subtree_sort.cu -- the shared-memory subtree kernel by presorted lists
// (dims 1-3).
//
// Same contract as k_subtree (fkd_build.cu): one CTA finishes every level
// below a subtree root of at most SUBN points and writes its nodes.  Instead
// of a radix select per level, the CTA sorts its points once per dimension
// and then walks the levels with lists:
//
//   1-2. for every dimension c, list_c: the slots of the points in the order
//      of the reference comparator (coordinate c, then id: FKDTree_cpu.h:
//      246-252).  Usually (a subtree is a small cell) the order bits of c span
//      less than 2^22 and a sort of 32-bit keys ((bits - min) << 10 | slot)
//      orders the points by coordinate, then each run of equal coordinates is
//      re-ordered by id; otherwise (or for runs longer than 32) the points are
//      ranked by id first (a sort of (id, slot) keys) and sorted by 64-bit
//      (bits, id rank) keys;
//   3. level d, split dimension c = d % dim: every segment [ls, ls + m) of
//      every list holds the same elements, and list_c holds them in split
//      order, so the pivot is list_c[ls + rank] -- no select at all; the
//      elements before it go left, after it right.  list_c is already
//      partitioned; each other list is partitioned stably (a block scan of
//      left / right flags, segmented at the segments' first slots so that
//      every slot gets its rank inside its own segment), which keeps it
//      sorted inside the children.
//
// The children's intervals [ls, ls + rank) and [ls + rank + 1, ls + m) are
// exactly the heap-tree geometry (fkd_common.cuh), and the pivot slot becomes
// a gap that no later level touches.  Every level costs one flag pass, one
// scan and one scatter per other list: no digit passes, few barriers.
#include "fkd_internal.h"

namespace fkd {

#ifdef FKD_PROF
// Phase cycle counters of the sorted subtree kernel (profiling builds only).
__device__ unsigned long long g_prof_sorted[8];
extern "C" __attribute__((visibility("default"))) void fkd_prof_sorted_read(unsigned long long* out) {
  cudaMemcpyFromSymbol(out, g_prof_sorted, sizeof(g_prof_sorted));
}
extern "C" __attribute__((visibility("default"))) void fkd_prof_sorted_reset() {
  unsigned long long z[8] = {0};
  cudaMemcpyToSymbol(g_prof_sorted, z, sizeof(z));
}
#define XPROF_T(v) const unsigned long long v = clock64()
#define XPROF_ADD(slot, a, b) \
  if (threadIdx.x == 0) atomicAdd(&g_prof_sorted[slot], (b) - (a))
#else
#define XPROF_T(v)
#define XPROF_ADD(slot, a, b)
#endif

namespace {

// XN, a template parameter below: the slots of a CTA, the largest subtree it
// takes (512 or 1,024: a power of two, 512..4096); XN / XPPT threads
constexpr int XPPT = 4;  // slots per thread
constexpr int XN_DEFAULT = 1024;
constexpr uint16_t GAP = 0xffffu;  // a slot outside every segment (a pivot of an earlier level)
constexpr uint8_t SL = 0, SR = 1, SP = 2;
static_assert(XPPT == 4, "a thread's slots move as one vector");

// A thread's XPPT consecutive slots move as one vector access (shared memory
// serves a warp's 8- or 16-byte accesses without bank conflicts; four scalar
// accesses at a stride of XPPT elements conflict).
__device__ __forceinline__ void ld4(const uint16_t* p, uint32_t (&o)[4]) {
  const uint2 v = *reinterpret_cast<const uint2*>(p);
  o[0] = v.x & 0xffffu;
  o[1] = v.x >> 16;
  o[2] = v.y & 0xffffu;
  o[3] = v.y >> 16;
}
__device__ __forceinline__ void st4(uint16_t* p, const uint32_t (&o)[4]) {
  *reinterpret_cast<uint2*>(p) = make_uint2((o[0] & 0xffffu) | (o[1] << 16), (o[2] & 0xffffu) | (o[3] << 16));
}
__device__ __forceinline__ void ld4(const uint32_t* p, uint32_t (&o)[4]) {
  const uint4 v = *reinterpret_cast<const uint4*>(p);
  o[0] = v.x;
  o[1] = v.y;
  o[2] = v.z;
  o[3] = v.w;
}
__device__ __forceinline__ void st4(uint32_t* p, const uint32_t (&o)[4]) {
  *reinterpret_cast<uint4*>(p) = make_uint4(o[0], o[1], o[2], o[3]);
}
__device__ __forceinline__ void ld4(const unsigned long long* p, unsigned long long (&o)[4]) {
  const ulonglong2 a = reinterpret_cast<const ulonglong2*>(p)[0], b = reinterpret_cast<const ulonglong2*>(p)[1];
  o[0] = a.x;
  o[1] = a.y;
  o[2] = b.x;
  o[3] = b.y;
}
__device__ __forceinline__ void st4(unsigned long long* p, const unsigned long long (&o)[4]) {
  reinterpret_cast<ulonglong2*>(p)[0] = make_ulonglong2(o[0], o[1]);
  reinterpret_cast<ulonglong2*>(p)[1] = make_ulonglong2(o[2], o[3]);
}

template <int DIM, int XN>
struct XCfg {
  // recs | eofr | lists (DIM x 2 buffers) | seg (2 buffers) | side | scratch (sort keys, later the
  // list levels' segment tables)
  static constexpr size_t recs = (size_t)(DIM + 1) * XN * 4;
  static constexpr size_t eofr = (size_t)XN * 2;
  static constexpr size_t lists = (size_t)DIM * 2 * XN * 2;
  static constexpr size_t seg = 2ull * XN * 2;
  static constexpr size_t side = XN;
  static constexpr size_t scratch = 2ull * XN * 8;
  static constexpr size_t smem = recs + eofr + lists + seg + side + scratch;
};


// Sorts XN keys (32- or 64-bit, ascending) with the whole CTA: bitonic sort
// of 128 keys per warp in registers, then merge-path rounds through shared
// memory.  Returns the buffer (a or b) that holds the result.  Thread t
// brings the keys of slots 4t .. 4t + 3 in v (cta_sort below loads them
// from a; a caller that computes them passes them straight in, with no
// pass through shared memory and no barrier before the sort).
template <int XN, class K>
__device__ K* cta_sort_regs(K (&v)[4], K* a, K* b) {
  static_assert(XN >= 512 && XN <= 4096 && (XN & (XN - 1)) == 0, "sorted subtree size");
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  K* wbase = a + warp * 128u;
#pragma unroll
  for (uint32_t k = 2; k <= 128; k <<= 1) {
#pragma unroll
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      if (j >= 4) {
        const uint32_t lm = j >> 2;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const uint32_t idx = lane * 4u + i;
          const K o = __shfl_xor_sync(0xffffffffu, v[i], lm);
          const bool lower = (idx & j) == 0u;
          const bool asc = (idx & k) == 0u;
          v[i] = (lower == asc) ? (v[i] < o ? v[i] : o) : (v[i] < o ? o : v[i]);
        }
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          if ((i & (int)j) == 0) {
            const uint32_t idx = lane * 4u + i;
            const bool asc = (idx & k) == 0u;
            const K x = v[i], y = v[i ^ (int)j];
            if ((x > y) == asc) {
              v[i] = y;
              v[i ^ (int)j] = x;
            }
          }
        }
      }
    }
  }
  st4(wbase + lane * 4u, v);
  K* src = a;
  K* dst = b;
  for (uint32_t s = 128; s < (uint32_t)XN; s <<= 1) {
    __syncthreads();
    const uint32_t og = threadIdx.x * XPPT;  // first of this thread's outputs
    const uint32_t pair = og / (2u * s);
    const uint32_t o = og - pair * 2u * s;
    const K* A = src + pair * 2u * s;
    const K* B = A + s;
    uint32_t lo = o > s ? o - s : 0u, hi = o < s ? o : s;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (A[mid] <= B[o - 1u - mid])  // ties: A first, as in the sequential merge below
        lo = mid + 1u;
      else
        hi = mid;
    }
    uint32_t i = lo, jb = o - lo;
    K out[XPPT];
#pragma unroll
    for (int q = 0; q < XPPT; ++q) {
      // an exhausted run reads as the padding key ~0 (never past its end)
      const K va = i < s ? A[i] : (K)~(K)0;
      const K vb = jb < s ? B[jb] : (K)~(K)0;
      const bool takeA = va < vb || (va == vb && i < s);
      out[q] = takeA ? va : vb;
      if (takeA)
        ++i;
      else
        ++jb;
    }
    st4(dst + pair * 2u * s + o, out);
    K* t = src;
    src = dst;
    dst = t;
  }
  __syncthreads();
  return src;
}

template <int XN, class K>
__device__ K* cta_sort(K* a, K* b) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  K v[4];
  ld4(a + warp * 128u + lane * 4u, v);
  return cta_sort_regs<XN, K>(v, a, b);
}

// Segmented exclusive scan of XN uint2 values (slots XPPT*tid ..
// XPPT*tid + XPPT - 1 per thread): head[k] marks a slot that starts a new
// segment; ex[k] is the sum of the values before slot k within its segment.
// Everything stays in registers but the per-warp totals (one barrier).
template <int XN>
__device__ void cta_segscan2(const uint2 (&val)[XPPT], const bool (&head)[XPPT], uint2 (&ex)[XPPT],
                             uint4* wtot) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  // within the thread: prefixes since its last head
  uint32_t rx = 0u, ry = 0u;
  bool th = false;  // the thread holds a head
#pragma unroll
  for (int k = 0; k < XPPT; ++k) {
    if (head[k]) {
      rx = ry = 0u;
      th = true;
    }
    ex[k] = make_uint2(rx, ry);
    rx += val[k].x;
    ry += val[k].y;
  }
  // across the warp: segmented inclusive scan of (tail sums, holds a head)
  uint32_t sx = rx, sy = ry;
  bool f = th;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t yx = __shfl_up_sync(0xffffffffu, sx, o);
    const uint32_t yy = __shfl_up_sync(0xffffffffu, sy, o);
    const bool yf = __shfl_up_sync(0xffffffffu, f, o);
    if (lane >= (uint32_t)o) {
      if (!f) {
        sx += yx;
        sy += yy;
      }
      f = f || yf;
    }
  }
  if (lane == 31u) wtot[warp] = make_uint4(sx, sy, f ? 1u : 0u, 0u);
  // the carry into this thread from the lanes before it (up to their last head)
  uint32_t cx = __shfl_up_sync(0xffffffffu, sx, 1), cy = __shfl_up_sync(0xffffffffu, sy, 1);
  bool cf = __shfl_up_sync(0xffffffffu, f, 1);
  if (lane == 0u) {
    cx = cy = 0u;
    cf = false;
  }
  __syncthreads();
  if (!cf) {
    // no head in the lanes before: add the previous warps' tails back to the last head
    for (int w = (int)warp - 1; w >= 0; --w) {
      const uint4 t = wtot[w];
      cx += t.x;
      cy += t.y;
      if (t.z) break;
    }
  }
#pragma unroll
  for (int k = 0; k < XPPT; ++k) {
    if (head[k]) break;  // from the thread's first head on, the prefixes are its own
    ex[k].x += cx;
    ex[k].y += cy;
  }
}

// Segment (d, t) of the event in subtree-local slots: start, length, rank.
__device__ __forceinline__ void seg_local(const Geom& g, uint32_t d, uint32_t t, uint32_t base, uint32_t& ls,
                                          uint32_t& m, uint32_t& k) {
  const uint32_t sh = g.H - d;
  const uint32_t W = 1u << sh;
  const uint32_t tw = t << sh;
  ls = tw + min(g.M, tw) - base;
  m = W - 1u + (g.M > tw ? min(g.M - tw, W) : 0u);
  if (sh == 0u) {
    k = 0u;
  } else {
    const uint32_t Wh = W >> 1;
    k = Wh - 1u + (g.M > tw ? min(g.M - tw, Wh) : 0u);
  }
}

// A segment's (start, length, rank) in one word: start and length up to
// 2,047, rank up to 1,023 (subtrees of at most 1,024 points).
__device__ __forceinline__ uint32_t seg_pack(uint32_t ls, uint32_t m, uint32_t k) {
  return ls | (m << 11) | (k << 22);
}
__device__ __forceinline__ void seg_unpack(uint32_t w, uint32_t& ls, uint32_t& m, uint32_t& k) {
  ls = w & 0x7ffu;
  m = (w >> 11) & 0x7ffu;
  k = w >> 22;
}

}  // namespace

template <int DIM, int XN>
__global__ void __launch_bounds__(XN / XPPT, 4096 / XN) k_subtree_sorted(const EvDesc* __restrict__ evs,
                                                           const uint2* __restrict__ subs, CSoA src_in, CSoA src_b0,
                                                           CSoA src_b1, Table tab_all, uint32_t* __restrict__ err) {
  constexpr int XST = XN / XPPT;  // threads
  using Cfg = XCfg<DIM, XN>;
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* recs = (uint32_t*)smem;                                 // [DIM + 1][XN], original slot order
  uint16_t* eofr = (uint16_t*)(smem + Cfg::recs);                   // id rank -> slot
  uint16_t* lists = (uint16_t*)(smem + Cfg::recs + Cfg::eofr);      // [DIM][2][XN] slots
  uint16_t* segb = (uint16_t*)(smem + Cfg::recs + Cfg::eofr + Cfg::lists);  // [2][XN]
  uint8_t* side = smem + Cfg::recs + Cfg::eofr + Cfg::lists + Cfg::seg;
  unsigned long long* keys = (unsigned long long*)(smem + Cfg::recs + Cfg::eofr + Cfg::lists + Cfg::seg + Cfg::side);
  __shared__ uint4 wseg[32];  // per-warp totals of the list levels' segmented scan

  const uint2 sb = subs[blockIdx.x];
  const EvDesc ev = evs[sb.x];
  const Geom g = ev.g;
  const uint32_t d0 = ev.d0;
  const uint32_t s0 = sb.y;
  const CSoA src_all = d0 == 0u ? src_in : ((d0 & 1u) ? src_b0 : src_b1);
  const CSoA src{src_all.base + ev.base, src_all.ids + ev.base, src_all.stride};
  const Table tab{tab_all.nodes + ev.base, tab_all.ids + ev.base};
  const uint32_t base = seg_start(g, d0, s0);
  const uint32_t nloc = seg_len(g, d0, s0);
  if (nloc > (uint32_t)XN) {
    if (threadIdx.x == 0) atomicOr(err, ERRB_INTERNAL);
    return;
  }
  // 1. records, and the range of each dimension's order bits
  __shared__ uint32_t s_mn[4], s_mx[4], s_slow;
  if (threadIdx.x < 4u) {
    s_mn[threadIdx.x] = 0xffffffffu;
    s_mx[threadIdx.x] = 0u;
  }
  if (threadIdx.x == 0) s_slow = 0u;
  __syncthreads();
  bool nan = false;
  uint32_t mn[DIM], mx[DIM];
#pragma unroll
  for (int w = 0; w < DIM; ++w) {
    mn[w] = 0xffffffffu;
    mx[w] = 0u;
  }
  for (uint32_t p = threadIdx.x; p < nloc; p += XST) {
#pragma unroll
    for (int w = 0; w < DIM; ++w) {
      const uint32_t v = __ldcs(src.base + (uint64_t)w * src.stride + base + p);
      nan |= is_nan_bits(v);
      recs[w * XN + p] = v;
      const uint32_t m = mono_bits(v);
      mn[w] = min(mn[w], m);
      mx[w] = max(mx[w], m);
    }
    recs[DIM * XN + p] = __ldcs(src.ids + base + p);
  }
  if (nan) atomicOr(err, ERRB_NAN);
#pragma unroll
  for (int w = 0; w < DIM; ++w) {
    const uint32_t a = __reduce_min_sync(0xffffffffu, mn[w]), b = __reduce_max_sync(0xffffffffu, mx[w]);
    if ((threadIdx.x & 31u) == 0u) {
      atomicMin(&s_mn[w], a);
      atomicMax(&s_mx[w], b);
    }
  }
  __syncthreads();
  XPROF_T(tp0);
  // 2. one list of slots per dimension, in the reference's order (coordinate,
  // then id: FKDTree_cpu.h:246-252).  Fast path: 32-bit keys
  // ((bits - min) >> sh) << 10 | slot, sh the smallest shift that brings the
  // dimension's range of order bits below 2^21, sort, then each run of equal
  // shifted keys -- sorted by slot -- is re-ordered by the full (bits, id) key,
  // one thread per run (a subtree is a small cell: sh is 0 and runs are rare
  // unless the cell reaches down to zero).  A run longer than TIE_RUN takes
  // the exact path: a sort by id gives each point its id rank r, then 64-bit
  // keys (bits << 12 | r).
  constexpr uint32_t TIE_RUN = 32;
  static_assert(XN <= 1024, "the 32-bit keys carry a 10-bit slot");
  bool fast = true;
  {
    uint32_t* k32 = (uint32_t*)keys;
    const uint32_t* idv = recs + (size_t)DIM * XN;
#pragma unroll 1
    for (int c = 0; c < DIM; ++c) {
      const uint32_t m0 = s_mn[c];
      const uint32_t rb = nloc ? 32u - (uint32_t)__clz(s_mx[c] - m0) : 0u;  // bit length of the range
      const uint32_t sh = rb > 21u ? rb - 21u : 0u;
      // this thread's four slots (the sort's register layout) straight from the records
      uint32_t kv[4];
      ld4(recs + (size_t)c * XN + threadIdx.x * 4u, kv);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const uint32_t r = threadIdx.x * 4u + (uint32_t)i;
        kv[i] = r < nloc ? ((((mono_bits(kv[i]) - m0) >> sh) << 10) | r) : 0xffffffffu;
      }
      const uint32_t* sk = cta_sort_regs<XN, uint32_t>(kv, k32, k32 + XN);
      uint16_t* lc = lists + (size_t)c * 2 * XN;
      for (uint32_t q = threadIdx.x; q < nloc; q += XST) lc[q] = (uint16_t)(sk[q] & 0x3ffu);
      __syncthreads();
      // runs of equal shifted keys (the sorted keys' upper bits, still in sk):
      // each run's first position re-orders it by the full key (the positions
      // of a run are one block of the order)
      const uint32_t* cx = recs + (size_t)c * XN;
      for (uint32_t q = threadIdx.x; q < nloc; q += XST) {
        const uint32_t mq = sk[q] >> 10;
        if (q > 0u && (sk[q - 1u] >> 10) == mq) continue;  // not the start of a run
        uint32_t e = q + 1u;
        while (e < nloc && e - q <= TIE_RUN && (sk[e] >> 10) == mq) ++e;
        if (e - q > TIE_RUN) {
          s_slow = 1u;
          continue;
        }
        for (uint32_t x = q + 1u; x < e; ++x) {  // insertion sort of [q, e) by (bits, id)
          const uint16_t sv = lc[x];
          const unsigned long long key = ((unsigned long long)mono_bits(cx[sv]) << 32) | idv[sv];
          uint32_t y = x;
          while (y > q) {
            const uint16_t pw = lc[y - 1u];
            if ((((unsigned long long)mono_bits(cx[pw]) << 32) | idv[pw]) <= key) break;
            lc[y] = pw;
            --y;
          }
          lc[y] = sv;
        }
      }
      __syncthreads();
    }
    fast = s_slow == 0u;
  }
  XPROF_T(tp1);
  if (!fast) {
    // exact path: id ranks (eofr[r] = slot of the r-th smallest id)
    for (uint32_t p = threadIdx.x; p < (uint32_t)XN; p += XST)
      keys[p] = p < nloc ? (((unsigned long long)recs[DIM * XN + p] << 12) | p) : ~0ull;
    __syncthreads();
    {
      const unsigned long long* sk = cta_sort<XN, unsigned long long>(keys, keys + XN);
      for (uint32_t r = threadIdx.x; r < nloc; r += XST) eofr[r] = (uint16_t)(sk[r] & 0xfffu);
      __syncthreads();
    }
#pragma unroll 1
    for (int c = 0; c < DIM; ++c) {
      for (uint32_t r = threadIdx.x; r < (uint32_t)XN; r += XST)
        keys[r] = r < nloc ? (((unsigned long long)mono_bits(recs[c * XN + eofr[r]]) << 12) | r) : ~0ull;
      __syncthreads();
      const unsigned long long* sk = cta_sort<XN, unsigned long long>(keys, keys + XN);
      uint16_t* lc = lists + (size_t)c * 2 * XN;
      for (uint32_t q = threadIdx.x; q < nloc; q += XST) lc[q] = eofr[sk[q] & 0xfffu];  // id rank -> slot
      __syncthreads();
    }
  }
  XPROF_T(tp2);
  // 3. levels.  Each level's segments (start, length, pivot rank) sit in a
  // table of packed words, written during the level before (two buffers in
  // the sort keys' space)
  uint32_t* segt = (uint32_t*)keys + 2u * XN;
  int cur[4] = {0, 0, 0, 0};  // which buffer of each list is current
  int sbuf = 0;
  for (uint32_t p = threadIdx.x; p < (uint32_t)XN; p += XST) segb[p] = p < nloc ? 0u : GAP;
  if (threadIdx.x == 0) {
    uint32_t ls, m, k;
    seg_local(g, d0, s0, base, ls, m, k);
    segt[0] = seg_pack(ls, m, k);
  }
  __syncthreads();
  for (uint32_t d = d0; d <= g.H; ++d) {
    const uint32_t j = d - d0;
    const uint32_t t0 = s0 << j;
    const uint32_t c = d % DIM;
    const uint16_t* lc = lists + ((size_t)c * 2 + cur[c]) * XN;
    const uint16_t* sg = segb + (size_t)sbuf * XN;
    uint16_t* sgn = segb + (size_t)(sbuf ^ 1) * XN;
    const uint32_t* T = segt + (j & 1u) * XN;
    if (d < g.H) {  // the next level's table: 2^(j+1) <= XN segments
      uint32_t* Tn = segt + ((j + 1u) & 1u) * XN;
      for (uint32_t u = threadIdx.x; u < (2u << j); u += XST) {
        uint32_t ls, m, k;
        seg_local(g, d + 1u, (t0 << 1) + u, base, ls, m, k);
        Tn[u] = seg_pack(ls, m, k);
      }
    }
    // (a) pivots and sides, from the split dimension's list
    const uint32_t pb = threadIdx.x * XPPT;  // this thread's first slot
    uint32_t uu[XPPT], rr[XPPT], nsg[XPPT];
    ld4(sg + pb, uu);
    ld4(lc + pb, rr);
#pragma unroll
    for (int q = 0; q < XPPT; ++q) {
      const uint32_t p = pb + q;
      const uint32_t u = uu[q];
      nsg[q] = GAP;
      if (u == GAP) continue;
      uint32_t ls, m, k;
      seg_unpack(T[u], ls, m, k);
      if (p < ls || p >= ls + m) {  // a slot outside its segment: broken invariant
        atomicOr(err, ERRB_INTERNAL);
        uu[q] = GAP;
        continue;
      }
      const uint32_t r = rr[q];
      const uint32_t pv = ls + k;
      if (p == pv) {
        side[r] = SP;
        const uint32_t e = r;  // the lists hold slots
        uint32_t rec[DIM + 1];
#pragma unroll
        for (int w = 0; w <= DIM; ++w) rec[w] = recs[w * XN + e];
        uint4 v;
        v.x = rec[0];
        v.y = DIM > 1 ? rec[1] : 0u;
        v.z = DIM > 2 ? rec[2] : 0u;
        v.w = rec[DIM];
        const uint32_t node = (1u << d) - 1u + t0 + u;
        tab.nodes[node] = v;
        tab.ids[node] = rec[DIM];
      } else {
        side[r] = p < pv ? SL : SR;
        nsg[q] = 2u * u + (p < pv ? 0u : 1u);
      }
    }
    st4(sgn + pb, nsg);
    if (d == g.H || DIM == 1) {
      // the last level, or a single list: the split list is the whole partition
      __syncthreads();
      sbuf ^= 1;
      continue;
    }
    __syncthreads();
    // (b) stable partition of the other lists: flags (left | right << 16), scan
    uint2 val[XPPT];
    uint32_t ra[XPPT], rb[XPPT];
    const uint32_t o1 = (c + 1u) % DIM, o2 = (c + 2u) % DIM;
    const uint16_t* l1 = lists + ((size_t)o1 * 2 + cur[o1]) * XN;
    const uint16_t* l2 = lists + ((size_t)o2 * 2 + cur[o2]) * XN;
    ld4(l1 + pb, ra);
    if (DIM > 2) {
      ld4(l2 + pb, rb);
    } else {
#pragma unroll
      for (int q = 0; q < XPPT; ++q) rb[q] = 0u;
    }
#pragma unroll
    for (int q = 0; q < XPPT; ++q) {
      const bool live = uu[q] != GAP;
      if (!live) ra[q] = 0u;
      rb[q] = (live && DIM > 2) ? rb[q] : 0u;
      const uint8_t s1 = live ? side[ra[q]] : SP;
      const uint8_t s2 = (live && DIM > 2) ? side[rb[q]] : SP;
      val[q].x = (s1 == SL ? 1u : 0u) | (s1 == SR ? 0x10000u : 0u);
      val[q].y = (s2 == SL ? 1u : 0u) | (s2 == SR ? 0x10000u : 0u);
    }
    // a slot starts a segment where the segment id changes (slot 0 always);
    // segments are separated by gap slots, which carry no flags
    bool head[XPPT];
    head[0] = pb == 0u || (uint32_t)sg[pb - 1u] != uu[0];
#pragma unroll
    for (int q = 1; q < XPPT; ++q) head[q] = uu[q - 1] != uu[q];
    uint2 at4[XPPT];  // flags before the slot within its segment
    cta_segscan2<XN>(val, head, at4, wseg);
    // (c) scatter into the other buffers (no barrier: the scan left each
    // slot's prefix in its own registers)
    uint16_t* n1 = lists + ((size_t)o1 * 2 + (cur[o1] ^ 1)) * XN;
    uint16_t* n2 = lists + ((size_t)o2 * 2 + (cur[o2] ^ 1)) * XN;
#pragma unroll
    for (int q = 0; q < XPPT; ++q) {
      const uint32_t u = uu[q];
      if (u == GAP) continue;
      uint32_t ls, m, k;
      seg_unpack(T[u], ls, m, k);
      const uint2 at = at4[q];
      // destinations stay inside the segment's child; anything else is a broken invariant
      uint32_t q1 = 0xffffffffu, q2 = 0xffffffffu;
      if (val[q].x & 0xffffu)
        q1 = ls + (at.x & 0xffffu);
      else if (val[q].x)
        q1 = ls + k + 1u + (at.x >> 16);
      if (DIM > 2) {
        if (val[q].y & 0xffffu)
          q2 = ls + (at.y & 0xffffu);
        else if (val[q].y)
          q2 = ls + k + 1u + (at.y >> 16);
      }
      if (q1 != 0xffffffffu) {
        if (q1 < ls + m)
          n1[q1] = (uint16_t)ra[q];
        else
          atomicOr(err, ERRB_INTERNAL);
      }
      if (q2 != 0xffffffffu) {
        if (q2 < ls + m)
          n2[q2] = (uint16_t)rb[q];
        else
          atomicOr(err, ERRB_INTERNAL);
      }
    }
    cur[o1] ^= 1;
    if (DIM > 2) cur[o2] ^= 1;
    sbuf ^= 1;
    __syncthreads();
  }
  XPROF_T(tp3);
  XPROF_ADD(0, tp0, tp1);
  XPROF_ADD(1, tp1, tp2);
  XPROF_ADD(2, tp2, tp3);
}

int sorted_sub_capacity(int subn) { return subn == 512 ? 512 : XN_DEFAULT; }

template <int DIM, int XN>
static cudaError_t run_sorted(const EvDesc* evs, const uint2* subs, uint32_t nsub, CSoA in, CSoA b0, CSoA b1,
                              Table tab, uint32_t* err, cudaStream_t stream) {
  const size_t smem = XCfg<DIM, XN>::smem;
  cudaError_t e =
      cudaFuncSetAttribute(k_subtree_sorted<DIM, XN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_subtree_sorted<DIM, XN><<<nsub, XN / XPPT, smem, stream>>>(evs, subs, in, b0, b1, tab, err);
  count_launches(1);
  return cudaGetLastError();
}

template <int DIM>
static cudaError_t run_sorted_n(int subn, const EvDesc* evs, const uint2* subs, uint32_t nsub, CSoA in, CSoA b0,
                                CSoA b1, Table tab, uint32_t* err, cudaStream_t stream) {
  if (sorted_sub_capacity(subn) == 512) return run_sorted<DIM, 512>(evs, subs, nsub, in, b0, b1, tab, err, stream);
  return run_sorted<DIM, XN_DEFAULT>(evs, subs, nsub, in, b0, b1, tab, err, stream);
}

cudaError_t launch_subtree_sorted(const EvDesc* evs, const uint2* subs, uint32_t nsub, CSoA in, CSoA b0, CSoA b1,
                                  Table tab, uint32_t* err, int dim, int subn, cudaStream_t stream) {
  if (nsub == 0) return cudaSuccess;
  switch (dim) {
    case 1: return run_sorted_n<1>(subn, evs, subs, nsub, in, b0, b1, tab, err, stream);
    case 2: return run_sorted_n<2>(subn, evs, subs, nsub, in, b0, b1, tab, err, stream);
    case 3: return run_sorted_n<3>(subn, evs, subs, nsub, in, b0, b1, tab, err, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fkd
