// fkd_search.cu -- box search on the flat tree (sm_100a).
//
// Semantics: FKDTree_CPU::search_in_the_box (FKDTree_cpu.h:123-169) and its
// BFS / branchless / recursive variants (:72-121, :25-70, :171-207) all return
// the ids of exactly the points inside the closed box (intersects /
// is_in_the_box, FKDTree_cpu.h:302-321): a child is skipped only when the
// node's split value proves the whole subtree lies outside.  The GPU visits
// the same children by the same tests -- left unless v < lo[c], right when
// v < lo[c] or lo[c] <= v <= hi[c] -- so its result set is the reference's.
//
// Shape: one warp per box, boxes handed out by an atomic counter to a
// persistent grid.  The frontier is a per-warp stack in shared memory (the
// FQueue replacement): the warp pops up to 32 nodes, each lane tests one node
// with a single 16-byte load, and the children are pushed back in lane order.
// Popping the top 32 of a depth-sorted stack keeps it depth-sorted and leaves
// at most min(64, 2^d) entries at depth d (stack_cap); the bound is still
// checked and reported (FKD_ERR_CAPACITY) rather than trusted.
//
// Every node also carries a 2*dim-bit mask saying which sides of its cell
// (the closed slab its ancestors' split values bound it by) already lie
// inside the box.  A child whose mask is full is inside entirely: its
// subtree is counted in closed form and, when ids are wanted, copied as one
// contiguous run of the in-order id table (k_inorder): the subtree of node
// (d, t) holds exactly the in-order positions [start(d,t), start(d,t) + len(d,t)),
// the interval the build gave it.
//
// Two passes ("count then write"): SEARCH_COUNT fills counts, a prefix sum
// turns them into offsets, and the ids go to every box's slice.  In
// fkd_search the count pass also records each box's result (single in-order
// positions and in-order runs, k_search<count, REC>) and k_expand writes the
// ids from that record, so the tree is traversed once; SEARCH_WRITE, the
// traversing write pass, serves fkd_search_write called alone and the boxes a
// full record pool missed.  SEARCH_DIGEST replaces the write by a per-box
// order-independent digest (contained subtrees add one precomputed subtree
// digest).  Count and digest also run with 1-16 lanes per box
// (k_search_grp), several boxes per warp.
#include <math.h>

#include "fkd_internal.h"

namespace fkd {

#ifdef FKD_PROF
// Cycle counters of the warp-per-box search (profiling builds only):
// [0] whole boxes, [1] leaf-bucket scans, [2] boxes, [3] walk steps, [4] scan windows.
__device__ unsigned long long g_prof_search[8];
extern "C" __attribute__((visibility("default"))) void fkd_prof_search_read(unsigned long long* out) {
  cudaMemcpyFromSymbol(out, g_prof_search, sizeof(g_prof_search));
}
extern "C" __attribute__((visibility("default"))) void fkd_prof_search_reset() {
  unsigned long long z[8] = {0};
  cudaMemcpyToSymbol(g_prof_search, z, sizeof(z));
}
#define SPROF_T(v) const unsigned long long v = clock64()
#define SPROF_ADD(slot, x) \
  if (lane == 0) atomicAdd(&g_prof_search[slot], (unsigned long long)(x))
#else
#define SPROF_T(v)
#define SPROF_ADD(slot, x)
#endif

constexpr int QT = 128;  // threads per CTA
constexpr int QW = QT / 32;
constexpr int JOBS = 256;      // contained-subtree jobs buffered per warp
constexpr int JFLUSH = JOBS - 64;  // one step adds at most 64
#ifndef FKD_EU
#define FKD_EU 4
#endif
constexpr int EU = FKD_EU;         // emission windows with loads in flight (measured: 4 beats 2 by 5%)
constexpr uint32_t SBLK = 4096;  // recording count pass: singles reserved per warp at a time
constexpr uint32_t RBLK = 2048;  // runs reserved per warp at a time
constexpr uint32_t CBLK = 64;    // chunk records reserved per warp at a time
constexpr uint32_t RCAP = 4096;  // results per chunk record before a new one starts
constexpr int BQ = 128;          // leaf buckets queued per warp (one step adds at most 64)
#ifndef FKD_SU
#define FKD_SU 1
#endif
constexpr int SU = FKD_SU;       // leaf-bucket scan: windows of 32 points with loads in flight

__device__ __forceinline__ uint32_t lanemask_lt_s() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ float sel4(uint32_t c, float a, float b, float d, float e) {
  return c == 0 ? a : (c == 1 ? b : (c == 2 ? d : e));
}

__device__ __forceinline__ unsigned long long warp_sum64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Popping the top 32 of a depth-sorted stack leaves at most 64 entries per
// depth, and depth d has only 2^d nodes: sum over d of min(64, 2^d), plus one.
// With leaf buckets of height b (and the in-order nodes to scan them) no node
// deeper than H - b - 1 is ever pushed.
__host__ __device__ inline uint32_t stack_cap(const Geom& g, uint32_t bucket = 0u) {
  const uint32_t dmax = bucket ? (g.H > bucket ? g.H - bucket - 1u : 0u) : g.H;
  uint32_t c = 1u;
  for (uint32_t d = 0; d <= dmax; ++d) c += d < 6u ? (1u << d) : 64u;
  return c;
}

// Batched search over a subset of the events (sc.evsel, in increasing
// order, with sc.evsel_q the exclusive prefix of their box counts): the
// qi-th box of the subset, and its event.
__device__ __forceinline__ uint32_t select_box(const SearchCtx& sc, uint32_t qi, uint32_t& ev) {
  uint32_t lo = 0u, hi = sc.nsel;  // evsel_q[lo] <= qi < evsel_q[hi]
  while (hi - lo > 1u) {
    const uint32_t mid = (lo + hi) >> 1;
    if (sc.evsel_q[mid] <= (uint64_t)qi)
      lo = mid;
    else
      hi = mid;
  }
  ev = sc.evsel[lo];
  return (uint32_t)(sc.evs[ev].qbase + ((uint64_t)qi - sc.evsel_q[lo]));
}

// Copies the concatenation of nj runs of the in-order table srct -- run k
// starts at srct[st[k]] and lands at out[base + pre[k]], pre being the
// exclusive prefix of the run lengths and total their sum -- with one warp.
// Each lane step writes 32 consecutive output slots; a lane finds its run
// from the bitmask of the runs that start inside the window (EU windows with
// loads in flight).  st / pre live in shared memory; slots at or past
// `limit` are not written and set `failed`.
__device__ __forceinline__ void copy_runs(const uint32_t* st, const uint32_t* pre, uint32_t nj, uint32_t total,
                                          const uint32_t* __restrict__ srct, uint32_t* __restrict__ out,
                                          uint64_t base, uint64_t limit, bool& failed) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t jb = 0u;  // the run holding output slot o0 (warp-uniform)
  for (uint32_t o0 = 0; o0 < total; o0 += 32u * EU) {
    uint32_t src[EU];
    bool ok[EU];
#pragma unroll
    for (int u = 0; u < EU; ++u) {
      const uint32_t w0 = o0 + 32u * u;
      const uint32_t k = jb + lane;
      const bool kv = k < nj;
      const uint32_t pk = kv ? pre[k] : total;
      const uint32_t sk = kv ? st[k] : 0u;
      // runs after jb start after w0 (every run holds at least one id)
      const uint32_t B = __reduce_or_sync(0xffffffffu, (lane > 0u && kv && pk < w0 + 32u) ? (1u << (pk - w0)) : 0u);
      const uint32_t jl = __popc(B & (0xffffffffu >> (31u - lane)));
      const uint32_t mp = __shfl_sync(0xffffffffu, pk, jl);
      const uint32_t ms = __shfl_sync(0xffffffffu, sk, jl);
      ok[u] = w0 + lane < total;
      src[u] = ms + (w0 + lane - mp);
      // the run holding w0 + 32: the one holding w0 + 31, or the next if it starts there
      uint32_t nb = jb + __popc(B);
      if (nb + 1u < nj && pre[nb + 1u] == w0 + 32u) ++nb;
      jb = nb;
    }
    uint32_t v[EU];
#pragma unroll
    for (int u = 0; u < EU; ++u) v[u] = ok[u] ? __ldg(srct + src[u]) : 0u;
#pragma unroll
    for (int u = 0; u < EU; ++u) {
      if (ok[u]) {
        const uint64_t pos = base + o0 + 32u * u + lane;
        if (pos < limit)
          out[pos] = v[u];
        else
          failed = true;
      }
    }
  }
}

// resident CTAs k_search is compiled for: 8 keeps the recording count pass at
// 64 registers (measured on one B200, 16M / 1M-box search: 1 / 5 / 8 / 10 / 12
// -> 21.7 / 21.7 / 21.3 / 24.6 / 24.9 ms count pass)
#ifndef FKD_QMINB
#define FKD_QMINB 8
#endif
template <int DIM, int MODE, bool REC = false>
__global__ void __launch_bounds__(QT, FKD_QMINB) k_search(SearchCtx sc, uint32_t cap) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int JN = REC ? JOBS / 2 : JOBS;  // the recording count pass flushes twice as often (occupancy)
  __shared__ uint32_t jst[QW][JN];   // in-order start of each buffered subtree (write pass, recording count)
  __shared__ uint32_t jlen[QW][JN];  // its size
  __shared__ uint32_t jpre[QW][JN];  // write pass: exclusive prefix of the sizes; recording count: single positions
  __shared__ uint32_t bq_st[QW][BQ];   // leaf buckets: in-order start of each queued subtree
  __shared__ uint32_t bq_len[QW][BQ];  // its size (the scan overwrites it with the exclusive prefix)
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t* stk_node = (uint32_t*)smem_raw + (size_t)warp * cap;
  uint8_t* stk_mask = (uint8_t*)((uint32_t*)smem_raw + (size_t)QW * cap) + (size_t)warp * cap;
  constexpr uint32_t FULL = (1u << (2 * DIM)) - 1u;
  const uint32_t lt = lanemask_lt_s();
  uint32_t cur_ev = 0;  // batched search: the event of the last box (boxes come in increasing order)
  // recording count pass: this warp's current pool blocks and chunk-record block
  uint32_t s_cur = 0u, s_end = 0u, r_cur = 0u, r_end = 0u, c_cur = 0u, c_end = 0u;

  for (;;) {
    uint32_t qi = 0;
    if (lane == 0) qi = atomicAdd(sc.qcounter, 1u);
    qi = __shfl_sync(0xffffffffu, qi, 0);
    if ((uint64_t)qi >= sc.boxes.q) break;
    uint32_t qj = sc.order ? sc.order[qi] : qi;
    if (sc.evsel) qj = select_box(sc, qi, cur_ev);
    uint64_t oj = qj;  // output slot of this box
    Geom g = sc.g;
    Table tab = sc.tab;
    const float* blo = sc.boxes.lo;
    const float* bhi = sc.boxes.hi;
    uint64_t bstride = sc.boxes.stride, bj = qj;
    if (sc.evs) {
      while (cur_ev + 1u < sc.nev && (uint64_t)qj >= sc.evs[cur_ev + 1u].qbase) ++cur_ev;
      const EvDesc& ev = sc.evs[cur_ev];
      g = ev.g;
      tab.nodes = sc.tab.nodes + ev.base;
      tab.ids = sc.tab.ids + ev.base;
      tab.sdig = sc.tab.sdig ? sc.tab.sdig + ev.base : nullptr;
      tab.ipts = sc.tab.ipts ? sc.tab.ipts + ev.base : nullptr;
      tab.dids = sc.tab.dids ? sc.tab.dids + ev.base : nullptr;
      tab.dnode = sc.tab.dnode ? sc.tab.dnode + ev.base : nullptr;
      blo = sc.boxes.lo + ev.qcbase;
      bhi = sc.boxes.hi + ev.qcbase;
      bstride = ev.nq;
      bj = qj - ev.qbase;
      oj = ev.qout + bj;
    }
    SPROF_T(tb0);
    const uint32_t n = g.n;
    // children at depth >= bdep are leaf buckets: subtrees of height <= sc.bucket, scanned in in-order layout
    const uint32_t bdep = (tab.ipts && sc.bucket) ? (g.H > sc.bucket ? g.H - sc.bucket : 0u) : 0xffffffffu;
    float lo[4] = {0.f, 0.f, 0.f, 0.f}, hi[4] = {0.f, 0.f, 0.f, 0.f};
    uint32_t mask0 = 0u;
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      lo[c] = blo[(uint64_t)c * bstride + bj];
      hi[c] = bhi[(uint64_t)c * bstride + bj];
      if (lo[c] == -INFINITY) mask0 |= 1u << (2 * c);
      if (hi[c] == INFINITY) mask0 |= 2u << (2 * c);
    }
    unsigned long long acc = 0ull;   // count (COUNT) / digest (DIGEST)
    unsigned long long acc2 = 0ull;  // count (DIGEST)
    uint64_t cursor = 0, cend = 0;
    if (MODE == SEARCH_WRITE) {
      cursor = sc.offsets[oj];
      cend = sc.offsets[oj + 1];
    }
    bool failed = false;
    uint32_t njobs = 0;  // warp-uniform

    // Emits one id per lane with v set, packed at the cursor.
    auto emit_ballot = [&](bool v, uint32_t node, uint32_t id) {
      const uint32_t bv = __ballot_sync(0xffffffffu, v);
      if (v) {
        if (MODE == SEARCH_WRITE) {
          const uint64_t pos = cursor + __popc(bv & lt);
          if (pos < cend && pos < sc.capacity)
            sc.out[pos] = sc.heap_out ? node : id;
          else
            failed = true;
        } else {
          acc += mix64(id);
        }
      }
      cursor += __popc(bv);
    };

    // Emits the whole subtrees buffered in the job list: job k is the run
    // [jst[k], jst[k] + jlen[k]) of the in-order table (tab.dids, or tab.dnode
    // for heap indices), where every subtree is one contiguous range; the
    // runs are concatenated at the cursor.
    auto run_jobs = [&](uint32_t nj) {
      uint32_t carry = 0u;
      for (uint32_t e0 = 0; e0 < nj; e0 += 32u) {
        const uint32_t e = e0 + lane;
        const uint32_t len = e < nj ? jlen[warp][e] : 0u;
        uint32_t incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= (uint32_t)o) incl += y;
        }
        if (e < nj) jpre[warp][e] = carry + incl - len;
        carry += __shfl_sync(0xffffffffu, incl, 31);
      }
      __syncwarp();
      const uint64_t limit = cend < sc.capacity ? cend : sc.capacity;
      copy_runs(jst[warp], jpre[warp], nj, carry, sc.heap_out ? tab.dnode : tab.dids, sc.out, cursor, limit, failed);
      cursor += carry;
      __syncwarp();
    };

    // Recording count pass (REC): the result of the box is also recorded in
    // the in-order table -- an in-box node whose children are not contained
    // as its position ("single"), a contained subtree (merged with an
    // adjacent in-box node) as a run -- handed to k_expand in chunks
    // (box, offset within the box, singles, runs), so the write pass needs
    // no second traversal.  A box whose record does not fit the pools is
    // listed in sc.flags for the traversing write pass.
    constexpr bool record = REC && MODE == SEARCH_COUNT;
    bool recfail = false;
    uint32_t relcur = 0u;  // results of the box recorded so far
    uint32_t nsing = 0u;   // singles buffered in jpre[warp] (warp-uniform)
    bool ropen = false;    // this box has an open chunk record (rb) that later flushes may extend
    uint32_t rb = 0u, rs0 = 0u, rns = 0u, rr0 = 0u, rnr = 0u, rrel = 0u, rcnt = 0u;
    auto flush_runs = [&](uint32_t nj) {
      uint32_t tot = nsing;
      {
        uint32_t t = 0u;
        for (uint32_t e = lane; e < nj; e += 32u) t += jlen[warp][e];
        tot += __reduce_add_sync(0xffffffffu, t);
      }
      if (!recfail) {
        // pool space comes in per-warp blocks (one atomic per block, not per flush)
        bool ok = true;
        if (s_cur + nsing > s_end) {
          const uint32_t want = nsing > SBLK ? nsing : SBLK;
          unsigned long long b = 0ull;
          if (lane == 0) b = atomicAdd(sc.pool_ctr + 1, (unsigned long long)want);
          b = __shfl_sync(0xffffffffu, b, 0);
          ok = b + want <= sc.pool_cap_s;
          s_cur = ok ? (uint32_t)b : 0u;
          s_end = ok ? (uint32_t)(b + want) : 0u;
          ropen = false;  // the next chunk cannot continue the last one
        }
        if (ok && r_cur + nj > r_end) {
          const uint32_t want = nj > RBLK ? nj : RBLK;
          unsigned long long b = 0ull;
          if (lane == 0) b = atomicAdd(sc.pool_ctr, (unsigned long long)want);
          b = __shfl_sync(0xffffffffu, b, 0);
          ok = b + want <= sc.pool_cap;
          r_cur = ok ? (uint32_t)b : 0u;
          r_end = ok ? (uint32_t)(b + want) : 0u;
          ropen = false;
        }
        if (ropen && rcnt >= RCAP) ropen = false;  // keep records short: k_expand balances by records
        if (ok && !ropen) {
          if (c_cur == c_end) {
            unsigned long long b = 0ull;
            if (lane == 0) b = atomicAdd(sc.brec_ctr, (unsigned long long)CBLK);
            b = __shfl_sync(0xffffffffu, b, 0);
            ok = b + CBLK <= sc.brec_cap;
            c_cur = ok ? (uint32_t)b : 0u;
            c_end = ok ? (uint32_t)(b + CBLK) : 0u;
          }
          if (ok) {
            rb = c_cur++;
            rs0 = s_cur;
            rr0 = r_cur;
            rns = rnr = 0u;
            rcnt = 0u;
            rrel = relcur;
            ropen = true;
          }
        }
        if (ok) {
          for (uint32_t e = lane; e < nj; e += 32u) {
            sc.pool_st[r_cur + e] = jst[warp][e];
            sc.pool_len[r_cur + e] = jlen[warp][e];
          }
          for (uint32_t e = lane; e < nsing; e += 32u) sc.pool_s[s_cur + e] = jpre[warp][e];
          s_cur += nsing;
          r_cur += nj;
          rns += nsing;
          rnr += nj;
          rcnt += tot;
          if (lane == 0) {
            sc.brec[2ull * rb] = make_uint4((uint32_t)oj, rrel, rs0, rns);
            sc.brec[2ull * rb + 1ull] = make_uint4(rr0, rnr, 0u, 0u);
          }
        } else {
          recfail = true;
        }
      } else if (lane == 0) {
        // keep counting what the box would have needed: the next call's pools are sized by it
        atomicAdd(sc.pool_ctr + 1, (unsigned long long)nsing);
        atomicAdd(sc.pool_ctr, (unsigned long long)nj);
        atomicAdd(sc.brec_ctr, 1ull);
      }
      relcur += tot;
      nsing = 0u;
      __syncwarp();
    };

    // Scans the queued leaf buckets: bucket k is the in-order range
    // [bq_st[k], bq_st[k] + bq_len[k]) of a subtree the walk would enter;
    // the ranges are concatenated and every lane tests one point per step
    // (16-byte loads of consecutive in-order nodes) -- the same points the
    // walk would have found, since the walk only skips subtrees that lie
    // outside the box.  Recording: consecutive in-box positions become one
    // run, isolated ones singles.
    uint32_t nb = 0;  // queued buckets (warp-uniform)
    auto scan_buckets = [&](uint32_t nbk) {
      SPROF_T(ts0);
      uint32_t carry = 0u;
      for (uint32_t e0 = 0; e0 < nbk; e0 += 32u) {
        const uint32_t e = e0 + lane;
        const uint32_t len = e < nbk ? bq_len[warp][e] : 0u;
        uint32_t incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= (uint32_t)o) incl += y;
        }
        if (e < nbk) bq_len[warp][e] = carry + incl - len;
        carry += __shfl_sync(0xffffffffu, incl, 31);
      }
      __syncwarp();
      const uint32_t total = carry;
      // one window's points: the in-box test and what the mode does with a hit
      auto take = [&](bool ok, uint32_t pos, const uint4& pt) {
        bool hit = false;
        if (ok) {
          bool in = true;
          if (DIM > 0) in &= (__uint_as_float(pt.x) <= hi[0] && __uint_as_float(pt.x) >= lo[0]);
          if (DIM > 1) in &= (__uint_as_float(pt.y) <= hi[1] && __uint_as_float(pt.y) >= lo[1]);
          if (DIM > 2) in &= (__uint_as_float(pt.z) <= hi[2] && __uint_as_float(pt.z) >= lo[2]);
          if (DIM > 3) in &= (__uint_as_float(pt.w) <= hi[3] && __uint_as_float(pt.w) >= lo[3]);
          hit = in;
        }
        if (MODE == SEARCH_COUNT && !record) {
          acc += hit ? 1u : 0u;
        } else if (MODE == SEARCH_DIGEST) {
          if (hit) {
            acc += mix64(DIM <= 3 ? pt.w : __ldg(tab.dids + pos));
            acc2 += 1u;
          }
        } else if (MODE == SEARCH_WRITE) {
          uint32_t idv = 0u, node = 0u;
          if (hit) {
            if (sc.heap_out)
              node = __ldg(tab.dnode + pos);
            else
              idv = DIM <= 3 ? pt.w : __ldg(tab.dids + pos);
          }
          emit_ballot(hit, node, idv);
        } else {
          acc += hit ? 1u : 0u;
          const uint32_t hb = __ballot_sync(0xffffffffu, hit);
          if (hb == 0u) return;  // nothing to record from this window (warp-uniform)
          if (njobs > (uint32_t)(JN - 16) || nsing > (uint32_t)(JN - 32)) {
            __syncwarp();
            flush_runs(njobs);
            njobs = 0;
          }
          // singles that carry ids cost the write pass one copy each: with
          // them every hit stays a single, unless runs are asked for
          const bool mk_runs = !sc.rec_ids || sc.bucket_runs;
          const uint32_t ppos = __shfl_up_sync(0xffffffffu, pos, 1);
          const bool cont = mk_runs && hit && lane > 0u && ((hb >> (lane - 1u)) & 1u) && ppos + 1u == pos;
          const uint32_t cb = __ballot_sync(0xffffffffu, cont);
          const bool start = hit && !cont;
          const uint32_t after = lane < 31u ? (cb >> (lane + 1u)) : 0u;
          const uint32_t rl = (uint32_t)__ffs(~after);  // 1 + the continuations that follow
          const bool single = start && rl == 1u;
          const bool isrun = start && rl > 1u;
          const uint32_t bs = __ballot_sync(0xffffffffu, single), br = __ballot_sync(0xffffffffu, isrun);
          if (isrun) {
            const uint32_t jp = njobs + __popc(br & lt);
            jst[warp][jp] = pos;
            jlen[warp][jp] = rl;
          }
          if (single) jpre[warp][nsing + __popc(bs & lt)] = sc.rec_ids ? (DIM <= 3 ? pt.w : __ldg(tab.dids + pos)) : pos;
          njobs += __popc(br);
          nsing += __popc(bs);
        }
      };
      uint32_t jb = 0u;  // the bucket holding slot w0 (warp-uniform)
      for (uint32_t w0 = 0; w0 < total; w0 += 32u * SU) {
        // SU windows: their positions first, then all their loads, then the tests
        uint32_t pos[SU];
        bool ok[SU];
#pragma unroll
        for (int u = 0; u < SU; ++u) {
          const uint32_t ww = w0 + 32u * u;
          const uint32_t k = jb + lane;
          const bool kv = k < nbk;
          const uint32_t pk = kv ? bq_len[warp][k] : total;
          const uint32_t sk = kv ? bq_st[warp][k] : 0u;
          // buckets after jb start after ww (every bucket holds at least one point)
          const uint32_t B =
              __reduce_or_sync(0xffffffffu, (lane > 0u && kv && pk < ww + 32u) ? (1u << (pk - ww)) : 0u);
          const uint32_t jl = __popc(B & (0xffffffffu >> (31u - lane)));
          const uint32_t mp = __shfl_sync(0xffffffffu, pk, jl);
          const uint32_t ms = __shfl_sync(0xffffffffu, sk, jl);
          uint32_t nbn = jb + __popc(B);
          if (nbn + 1u < nbk && bq_len[warp][nbn + 1u] == ww + 32u) ++nbn;
          ok[u] = ww + lane < total;
          pos[u] = ms + (ww + lane - mp);
          if (ww < total) jb = nbn;
        }
        uint4 pt[SU];
#pragma unroll
        for (int u = 0; u < SU; ++u) pt[u] = ok[u] ? __ldg(tab.ipts + pos[u]) : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
        for (int u = 0; u < SU; ++u) take(ok[u], pos[u], pt[u]);
      }
      if (record && (njobs > (uint32_t)(JN - 64) || nsing > (uint32_t)(JN - 32))) {
        __syncwarp();
        flush_runs(njobs);
        njobs = 0;
      }
      __syncwarp();
      SPROF_T(ts1);
      SPROF_ADD(1, ts1 - ts0);
      SPROF_ADD(4, (total + 31u) / 32u);
    };

    int top = 0;
    if (n > 0) {
      if (mask0 == FULL) {
        if (MODE == SEARCH_COUNT) {
          if (lane == 0) {
            acc += n;
            if (record) {
              jst[warp][0] = 0u;
              jlen[warp][0] = n;
            }
          }
          if (record) njobs = 1;
          __syncwarp();
        } else if (MODE == SEARCH_DIGEST) {
          if (lane == 0) {
            acc2 += n;
            acc += tab.sdig[0];
          }
        } else {
          if (lane == 0) {
            jst[warp][0] = 0u;
            jlen[warp][0] = n;
          }
          njobs = 1;
          __syncwarp();
        }
      } else {
        // descend, all lanes alike, while the box lies on one side of the
        // node's split: such a node is outside the box and the walk would
        // visit only that one child; the walk starts at the first node the
        // box straddles (its cell's mask is still mask0)
        uint32_t r = 0u, dep = 0u;
        bool empty = false;
        while (dep + 1u < bdep) {
          const uint32_t c = dep % (uint32_t)DIM;
          const uint4 nd = __ldg(tab.nodes + r);
          const float v = sel4(c, __uint_as_float(nd.x), __uint_as_float(nd.y), __uint_as_float(nd.z),
                               __uint_as_float(nd.w));
          const float loc = sel4(c, lo[0], lo[1], lo[2], lo[3]);
          const float hic = sel4(c, hi[0], hi[1], hi[2], hi[3]);
          uint32_t nx;
          if (v < loc)
            nx = 2u * r + 2u;  // the walk visits the right child only
          else if (v > hic)
            nx = 2u * r + 1u;  // the left child only
          else
            break;
          if (nx >= n) {  // that child does not exist: nothing is inside
            empty = true;
            break;
          }
          r = nx;
          ++dep;
        }
        if (!empty) {
          if (lane == 0) {
            stk_node[0] = r;
            stk_mask[0] = (uint8_t)(mask0 | (DIM == 3 ? ((dep % 3u) << 6) : 0u));
          }
          top = 1;
        }
      }
    }
    __syncwarp();

    while (top > 0) {
      SPROF_ADD(3, 1);
      const int gcount = top < 32 ? top : 32;
      const int base = top - gcount;
      const bool have = (int)lane < gcount;
      uint32_t i = 0u, mask = 0u;
      if (have) {
        i = stk_node[base + lane];
        mask = stk_mask[base + lane];
      }
      __syncwarp();
      top = base;
      bool emit = false, pushL = false, pushR = false, contL = false, contR = false;
      bool bucketL = false, bucketR = false;
      uint32_t maskL = 0u, maskR = 0u, idv = 0u, cnext = 0u;
      if (have) {
        // 3D: the node's split dimension rides in the top bits of its mask byte
        uint32_t c;
        if (DIM == 3) {
          c = mask >> 6;
          mask &= 0x3fu;
        } else {
          c = floor_log2_u32(i + 1u) % DIM;
        }
        cnext = c + 1u == (uint32_t)DIM ? 0u : c + 1u;
        const uint4 nd = __ldg(tab.nodes + i);
        const float x0 = __uint_as_float(nd.x), x1 = __uint_as_float(nd.y), x2 = __uint_as_float(nd.z),
                    x3 = __uint_as_float(nd.w);
        const float v = sel4(c, x0, x1, x2, x3);
        const float loc = sel4(c, lo[0], lo[1], lo[2], lo[3]);
        const float hic = sel4(c, hi[0], hi[1], hi[2], hi[3]);
        const bool inter = v <= hic && v >= loc;
        const bool lower = v < loc;
        if (inter) {
          bool in = true;
          if (DIM > 0) in &= (x0 <= hi[0] && x0 >= lo[0]);
          if (DIM > 1) in &= (x1 <= hi[1] && x1 >= lo[1]);
          if (DIM > 2) in &= (x2 <= hi[2] && x2 >= lo[2]);
          if (DIM > 3) in &= (x3 <= hi[3] && x3 >= lo[3]);
          emit = in;
        }
        if (emit && (MODE != SEARCH_COUNT || (record && sc.rec_ids))) idv = DIM <= 3 ? nd.w : __ldg(tab.ids + i);
        const uint32_t l = 2u * i + 1u;
        const bool visitL = !lower && l < n;
        const bool visitR = (lower || inter) && l + 1u < n;
        maskL = mask | (v <= hic ? (2u << (2 * c)) : 0u);
        maskR = mask | (v >= loc ? (1u << (2 * c)) : 0u);
        contL = visitL && maskL == FULL;
        contR = visitR && maskR == FULL;
        pushL = visitL && !contL;
        pushR = visitR && !contR;
        if (pushL || pushR) {
          // children at the bucket depth are scanned, not walked
          const uint32_t dep = 31u - (uint32_t)__clz(i + 1u);
          if (dep + 1u >= bdep) {
            bucketL = pushL;
            bucketR = pushR;
            pushL = pushR = false;
          }
        }
      }
      if (MODE == SEARCH_COUNT) {
        if (!record) {
          acc += (emit ? 1u : 0u) + (contL ? subtree_size(g, 2u * i + 1u) : 0u) +
                 (contR ? subtree_size(g, 2u * i + 2u) : 0u);
        } else {
          // node (dep, t) owns in-order [S, S + len); its left subtree is
          // [S, S + K), itself S + K, its right subtree the rest (32-bit
          // arithmetic: every position is below n < 2^31)
          uint32_t s1 = 0u, l1 = 0u, s2 = 0u, l2 = 0u, sg = 0u;
          const bool single = emit && !contL && !contR;
          if (emit || contL || contR) {
            const uint32_t dep = 31u - (uint32_t)__clz(i + 1u);
            const uint32_t t = i + 1u - (1u << dep);
            const uint32_t sh = g.H - dep;
            const uint32_t tw = t << sh;
            const uint32_t S = tw + min(g.M, tw);
            uint32_t K = 0u, W = 0u;
            if (sh != 0u) {  // len(dep + 1, 2t); (2t) * 2^(H-dep-1) = t * 2^(H-dep)
              W = 1u << (sh - 1u);
              K = W - 1u + (g.M > tw ? min(g.M - tw, W) : 0u);
            }
            const uint32_t P = S + K;
            sg = P;
            if (!single) {
              const uint32_t tw3 = tw + W;  // (2t + 1) * 2^(H-dep-1)
              const uint32_t lenR = contR ? W - 1u + (g.M > tw3 ? min(g.M - tw3, W) : 0u) : 0u;
              if (contL) {
                s1 = S;
                l1 = K;
              }
              if (emit) {
                if (l1 == 0u) s1 = P;
                l1 += 1u;
              }
              if (contR) {
                if (l1 == 0u) {
                  s1 = P + 1u;
                  l1 = lenR;
                } else if (emit) {
                  l1 += lenR;
                } else {
                  s2 = P + 1u;
                  l2 = lenR;
                }
              }
            }
          }
          acc += (single ? 1u : 0u) + l1 + l2;
          const uint32_t b1 = __ballot_sync(0xffffffffu, l1 != 0u), b2 = __ballot_sync(0xffffffffu, l2 != 0u);
          const uint32_t bs = __ballot_sync(0xffffffffu, single);
          uint32_t jp = njobs + __popc(b1 & lt) + __popc(b2 & lt);
          if (l1) {
            jst[warp][jp] = s1;
            jlen[warp][jp] = l1;
            ++jp;
          }
          if (l2) {
            jst[warp][jp] = s2;
            jlen[warp][jp] = l2;
          }
          if (single) jpre[warp][nsing + __popc(bs & lt)] = sc.rec_ids ? idv : sg;
          njobs += __popc(b1) + __popc(b2);
          nsing += __popc(bs);
          if (njobs > (uint32_t)(JN - 64) || nsing > (uint32_t)(JN - 32)) {
            __syncwarp();
            flush_runs(njobs);
            njobs = 0;
          }
        }
      } else {
        if (MODE == SEARCH_DIGEST) {
          // a contained subtree's digest is one table entry (sdig)
          if (emit) acc += mix64(idv);
          if (contL) acc += tab.sdig[2u * i + 1u];
          if (contR) acc += tab.sdig[2u * i + 2u];
          acc2 += (emit ? 1u : 0u) + (contL ? subtree_size(g, 2u * i + 1u) : 0u) +
                  (contR ? subtree_size(g, 2u * i + 2u) : 0u);
        } else {
          emit_ballot(emit, i, idv);
        }
        // buffer the contained subtrees; emit them in bulk when the buffer fills
        if (MODE == SEARCH_WRITE) {
        const uint32_t bl = __ballot_sync(0xffffffffu, contL), br = __ballot_sync(0xffffffffu, contR);
        const uint32_t jp = njobs + __popc(bl & lt) + __popc(br & lt);
        if (contL || contR) {
          // the children of node (dep, t) are (dep + 1, 2t) and (dep + 1, 2t + 1)
          const uint32_t dc = floor_log2_u32(i + 1u) + 1u;
          const uint32_t tl = 2u * (i + 1u - (1u << (dc - 1u)));
          if (contL) {
            jst[warp][jp] = seg_start(g, dc, tl);
            jlen[warp][jp] = seg_len(g, dc, tl);
          }
          if (contR) {
            const uint32_t q2 = jp + (contL ? 1u : 0u);
            jst[warp][q2] = seg_start(g, dc, tl + 1u);
            jlen[warp][q2] = seg_len(g, dc, tl + 1u);
          }
        }
        njobs += __popc(bl) + __popc(br);
        if (njobs > (uint32_t)JFLUSH) {
          __syncwarp();
          run_jobs(njobs);
          njobs = 0;
        }
        }
      }
      // push the children in lane order (keeps the stack depth-sorted)
      const uint32_t bpl = __ballot_sync(0xffffffffu, pushL), bpr = __ballot_sync(0xffffffffu, pushR);
      const uint32_t tot = __popc(bpl) + __popc(bpr);
      if ((uint32_t)top + tot > cap) {
        failed = true;
        break;
      }
      uint32_t p = (uint32_t)top + __popc(bpl & lt) + __popc(bpr & lt);
      const uint32_t ctag = DIM == 3 ? cnext << 6 : 0u;
      if (pushL) {
        stk_node[p] = 2u * i + 1u;
        stk_mask[p] = (uint8_t)(maskL | ctag);
        ++p;
      }
      if (pushR) {
        stk_node[p] = 2u * i + 2u;
        stk_mask[p] = (uint8_t)(maskR | ctag);
      }
      top += (int)tot;
      // queue the leaf buckets
      const uint32_t bbl = __ballot_sync(0xffffffffu, bucketL), bbr = __ballot_sync(0xffffffffu, bucketR);
      if (bbl | bbr) {
        uint32_t q = nb + __popc(bbl & lt) + __popc(bbr & lt);
        if (bucketL || bucketR) {
          const uint32_t dc = floor_log2_u32(i + 1u) + 1u;
          const uint32_t tl = 2u * (i + 1u - (1u << (dc - 1u)));
          if (bucketL) {
            bq_st[warp][q] = seg_start(g, dc, tl);
            bq_len[warp][q] = seg_len(g, dc, tl);
            ++q;
          }
          if (bucketR) {
            bq_st[warp][q] = seg_start(g, dc, tl + 1u);
            bq_len[warp][q] = seg_len(g, dc, tl + 1u);
          }
        }
        nb += __popc(bbl) + __popc(bbr);
        if (nb > (uint32_t)(BQ - 64)) {
          __syncwarp();
          scan_buckets(nb);
          nb = 0;
        }
      }
      __syncwarp();
    }
    if (nb) {
      __syncwarp();
      scan_buckets(nb);
      nb = 0;
    }

    if (MODE == SEARCH_WRITE && njobs) {
      __syncwarp();
      run_jobs(njobs);
    }
    if (record) {
      if (njobs || nsing) {
        __syncwarp();
        flush_runs(njobs);
      }
      if (recfail) {
        // a chunk this box already wrote stays valid: zero its counts, the
        // traversing write pass writes the whole box
        if (ropen && lane == 0) {
          sc.brec[2ull * rb] = make_uint4((uint32_t)oj, 0u, 0u, 0u);
          sc.brec[2ull * rb + 1ull] = make_uint4(0u, 0u, 0u, 0u);
        }
        if (lane == 0) sc.flags[atomicAdd(sc.flag_ctr, 1u)] = qj;
      }
    }
    const bool anyfail = __any_sync(0xffffffffu, failed);
    if (MODE == SEARCH_COUNT) {
      const unsigned long long tot = warp_sum64(acc);
      if (lane == 0) sc.counts[oj] = (uint32_t)tot;
      if (lane == 0 && tot > 0xffffffffull) atomicOr(sc.err, ERRB_CAPACITY);
    } else if (MODE == SEARCH_DIGEST) {
      const unsigned long long dg = warp_sum64(acc);
      const unsigned long long ct = warp_sum64(acc2);
      if (lane == 0) {
        sc.digests[oj] = dg;
        sc.counts[oj] = (uint32_t)ct;
      }
    } else {
      if (lane == 0 && cursor != cend) atomicOr(sc.err, ERRB_INTERNAL);
    }
    if (anyfail && lane == 0) atomicOr(sc.err, ERRB_CAPACITY);
    __syncwarp();
    SPROF_T(tb1);
    SPROF_ADD(0, tb1 - tb0);
    SPROF_ADD(2, 1);
  }
}

// Writes every box's result from what its count pass recorded: a warp per
// chunk record (box, offset within the box, singles, runs) -- the singles'
// ids first, one per lane, then the runs, JOBS at a time -- with no
// traversal state, so the copy runs at full occupancy.  Records never
// written (the tail of a warp's record block) are zero and skipped.
constexpr int XT = 256;  // threads of k_expand
#ifndef FKD_EXU
#define FKD_EXU 8
#endif
// k_expand: single ids with loads in flight per lane (measured on the 16M /
// 1M-box search: 4 / 8 / 16 -> 7.95-9.23 / 8.09 / 11.3 ms write pass)
constexpr int EXU = FKD_EXU;
#ifndef FKD_XMINB
#define FKD_XMINB 1  // resident CTAs k_expand is compiled for (6 / 8 measured no better)
#endif
constexpr uint32_t XREC = 4;  // k_expand: chunk records a warp takes from the counter at a time
__global__ void __launch_bounds__(XT, FKD_XMINB) k_expand(const uint4* __restrict__ brec,
                                               const unsigned long long* __restrict__ brec_ctr, uint64_t brec_cap,
                                               const uint32_t* __restrict__ pool_s,
                                               const uint32_t* __restrict__ pool_st,
                                               const uint32_t* __restrict__ pool_len,
                                               const uint64_t* __restrict__ offsets,
                                               const uint32_t* __restrict__ srct, uint32_t* __restrict__ out,
                                               uint64_t capacity, uint32_t* __restrict__ err, int singles_ids,
                                               unsigned long long* __restrict__ work) {
  __shared__ uint32_t st[XT / 32][JOBS];
  __shared__ uint32_t pre[XT / 32][JOBS];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint64_t nrec = *brec_ctr < brec_cap ? *brec_ctr : brec_cap;
  bool failed = false;
  // records are handed out XREC at a time from a counter (their sizes vary
  // from one id to RCAP), the next block taken before the current one is copied
  auto grab = [&]() {
    unsigned long long v = 0ull;
    if (lane == 0) v = atomicAdd(work, (unsigned long long)XREC);
    return (uint64_t)__shfl_sync(0xffffffffu, v, 0);
  };
  uint64_t r0 = grab();
  while (r0 < nrec) {
    const uint64_t rnext = grab();
  for (uint64_t r = r0; r < r0 + XREC && r < nrec; ++r) {
    const uint4 R = brec[2 * r], R2 = brec[2 * r + 1];
    const uint32_t ns = R.w, nj = R2.y;
    if (ns == 0u && nj == 0u) continue;
    const uint64_t lo = offsets[R.x], hi = offsets[R.x + 1u];
    const uint64_t limit = hi < capacity ? hi : capacity;
    uint64_t base = lo + R.y;
    // singles
    for (uint32_t e0 = 0; e0 < ns; e0 += 32u * EXU) {
      uint32_t v[EXU];
#pragma unroll
      for (int u = 0; u < EXU; ++u) {
        const uint32_t e = e0 + 32u * u + lane;
        v[u] = e < ns ? __ldg(pool_s + R.z + e) : 0u;
      }
      if (!singles_ids) {
#pragma unroll
        for (int u = 0; u < EXU; ++u) {
          const uint32_t e = e0 + 32u * u + lane;
          if (e < ns) v[u] = __ldg(srct + v[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < EXU; ++u) {
        const uint32_t e = e0 + 32u * u + lane;
        if (e < ns) {
          if (base + e < limit)
            out[base + e] = v[u];
          else
            failed = true;
        }
      }
    }
    base += ns;
    // runs, JOBS at a time
    for (uint32_t k0 = 0; k0 < nj; k0 += (uint32_t)JOBS) {
      const uint32_t m = (nj - k0) < (uint32_t)JOBS ? (nj - k0) : (uint32_t)JOBS;
      const uint64_t pb = (uint64_t)R2.x + k0;
      uint32_t carry = 0u;
      for (uint32_t e0 = 0; e0 < m; e0 += 32u) {
        const uint32_t e = e0 + lane;
        const uint32_t len = e < m ? pool_len[pb + e] : 0u;
        uint32_t incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= (uint32_t)o) incl += y;
        }
        if (e < m) {
          st[warp][e] = pool_st[pb + e];
          pre[warp][e] = carry + incl - len;
        }
        carry += __shfl_sync(0xffffffffu, incl, 31);
      }
      __syncwarp();
      copy_runs(st[warp], pre[warp], m, carry, srct, out, base, limit, failed);
      base += carry;
      __syncwarp();
    }
  }
    r0 = rnext;
  }
  if (__any_sync(0xffffffffu, failed) && lane == 0) atomicOr(err, ERRB_CAPACITY);
}

cudaError_t launch_expand(const SearchCtx& sc) {
  if (!sc.pool_st || !sc.work_ctr) return cudaSuccess;
  int dev = 0, sms = 148, per = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_expand, XT, 0);
  if (e != cudaSuccess) return e;
  if (per < 1) per = 1;
  k_expand<<<(unsigned)(sms * per), XT, 0, sc.stream>>>(sc.brec, sc.brec_ctr, sc.brec_cap, sc.pool_s, sc.pool_st,
                                                        sc.pool_len,
                                                        sc.offsets, sc.heap_out ? sc.tab.dnode : sc.tab.dids, sc.out,
                                                        sc.capacity, sc.err, sc.rec_ids, sc.work_ctr);
  count_launches(1);
  return cudaGetLastError();
}

// Count / digest with G < 32 lanes per box (G = 1: a thread per box): a warp
// holds 32/G boxes, each group with its own depth-sorted stack (popping the
// top G keeps at most 2G entries per depth, so 2G*(H+1) + 1 bound it), and a
// group that finishes takes the next box at once.  Small boxes near the root
// keep only a few nodes in flight; packing several per warp fills the lanes
// those steps leave idle.  Same node tests and accumulation as k_search.
__host__ __device__ inline uint32_t stack_cap_lanes(const Geom& g, uint32_t G) { return 2u * G * (g.H + 1u) + 1u; }

template <int DIM, int MODE, int G, bool BKT>
__global__ void __launch_bounds__(QT) k_search_grp(SearchCtx sc, uint32_t cap) {
  static_assert(G == 1 || G == 2 || G == 4 || G == 8 || G == 16, "group width");
  constexpr int NG = QT / G;
  constexpr uint32_t GM = (1u << G) - 1u;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t grp = threadIdx.x / G, gl = threadIdx.x % G;
  const uint32_t gsh = lane & ~(uint32_t)(G - 1);
  const uint32_t gmask = GM << gsh;
  const uint32_t glt = (1u << gl) - 1u;
  uint32_t* stk_node = (uint32_t*)smem_raw + (size_t)grp * cap;
  uint8_t* stk_mask = (uint8_t*)((uint32_t*)smem_raw + (size_t)NG * cap) + (size_t)grp * cap;
  constexpr uint32_t FULL = (1u << (2 * DIM)) - 1u;

  uint32_t cur_ev = 0;
  bool active = false, exhausted = false, failed = false;
  int top = 0;
  uint64_t oj = 0;
  Geom g = sc.g;
  Table tab = sc.tab;
  float lo[4] = {0.f, 0.f, 0.f, 0.f}, hi[4] = {0.f, 0.f, 0.f, 0.f};
  unsigned long long acc = 0ull, acc2 = 0ull;
  // children at depth >= bdep are leaf buckets: pushed with BUCKET_BIT set and,
  // when popped, their points scanned by the lane that popped them
  uint32_t bdep = 0xffffffffu;
  constexpr uint32_t BUCKET_BIT = 0x80000000u;  // node indices stay below 2^31

  // the group's result for its current box (group-uniform call)
  auto finish = [&]() {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
      acc += __shfl_xor_sync(gmask, acc, o);
      if (MODE == SEARCH_DIGEST) acc2 += __shfl_xor_sync(gmask, acc2, o);
    }
    const bool anyfail = __any_sync(gmask, failed);
    if (gl == 0) {
      if (MODE == SEARCH_COUNT) {
        sc.counts[oj] = (uint32_t)acc;
        if (acc > 0xffffffffull) atomicOr(sc.err, ERRB_CAPACITY);
      } else {
        sc.digests[oj] = acc;
        sc.counts[oj] = (uint32_t)acc2;
      }
      if (anyfail) atomicOr(sc.err, ERRB_CAPACITY);
    }
    active = false;
    failed = false;
  };

  for (;;) {
    // groups without a box take boxes until one needs a traversal
    while (!active && !exhausted) {
      uint32_t qi = 0;
      if (gl == 0) qi = atomicAdd(sc.qcounter, 1u);
      qi = __shfl_sync(gmask, qi, 0, G);
      if ((uint64_t)qi >= sc.boxes.q) {
        exhausted = true;
        break;
      }
      uint32_t qj = sc.order ? sc.order[qi] : qi;
      if (sc.evsel) qj = select_box(sc, qi, cur_ev);
      oj = qj;
      g = sc.g;
      tab = sc.tab;
      const float* blo = sc.boxes.lo;
      const float* bhi = sc.boxes.hi;
      uint64_t bstride = sc.boxes.stride, bj = qj;
      if (sc.evs) {
        while (cur_ev + 1u < sc.nev && (uint64_t)qj >= sc.evs[cur_ev + 1u].qbase) ++cur_ev;
        const EvDesc& ev = sc.evs[cur_ev];
        g = ev.g;
        tab.nodes = sc.tab.nodes + ev.base;
        tab.ids = sc.tab.ids + ev.base;
        tab.sdig = sc.tab.sdig ? sc.tab.sdig + ev.base : nullptr;
        tab.ipts = sc.tab.ipts ? sc.tab.ipts + ev.base : nullptr;
        tab.dids = sc.tab.dids ? sc.tab.dids + ev.base : nullptr;
        blo = sc.boxes.lo + ev.qcbase;
        bhi = sc.boxes.hi + ev.qcbase;
        bstride = ev.nq;
        bj = qj - ev.qbase;
        oj = ev.qout + bj;
      }
      uint32_t mask0 = 0u;
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        lo[c] = blo[(uint64_t)c * bstride + bj];
        hi[c] = bhi[(uint64_t)c * bstride + bj];
        if (lo[c] == -INFINITY) mask0 |= 1u << (2 * c);
        if (hi[c] == INFINITY) mask0 |= 2u << (2 * c);
      }
      acc = 0ull;
      acc2 = 0ull;
      if (BKT) bdep = (tab.ipts && sc.bucket_grp) ? (g.H > sc.bucket_grp ? g.H - sc.bucket_grp : 0u) : 0xffffffffu;
      if (g.n == 0) {
        finish();
      } else if (mask0 == FULL) {
        if (gl == 0) {
          if (MODE == SEARCH_COUNT) {
            acc = g.n;
          } else {
            acc = tab.sdig[0];
            acc2 = g.n;
          }
        }
        finish();
      } else {
        // (no descent here: a group taking a box would hold up the other
        // groups of its warp for a chain of dependent loads)
        if (gl == 0) {
          stk_node[0] = 0u;
          stk_mask[0] = (uint8_t)mask0;
        }
        top = 1;
        active = true;
      }
    }
    if (!__any_sync(0xffffffffu, active)) break;
    __syncwarp();

    const int gcount = top < G ? top : G;
    const int base = top - gcount;
    const bool have = (int)gl < gcount;
    uint32_t i = 0u, mask = 0u;
    if (have) {
      i = stk_node[base + gl];
      mask = stk_mask[base + gl];
    }
    __syncwarp();
    top = base;
    bool pushL = false, pushR = false, bucket = false;
    uint32_t maskL = 0u, maskR = 0u;
    if (BKT && have && (i & BUCKET_BIT)) {
      // a leaf bucket: its subtree is the in-order range [S, S + len)
      bucket = true;
      const uint32_t nb = i & ~BUCKET_BIT;
      const uint32_t dep = floor_log2_u32(nb + 1u);
      const uint32_t t = nb + 1u - (1u << dep);
      const uint32_t S = seg_start(g, dep, t), len = seg_len(g, dep, t);
      for (uint32_t k = 0; k < len; ++k) {
        const uint4 pt = __ldg(tab.ipts + S + k);
        bool in = true;
        if (DIM > 0) in &= (__uint_as_float(pt.x) <= hi[0] && __uint_as_float(pt.x) >= lo[0]);
        if (DIM > 1) in &= (__uint_as_float(pt.y) <= hi[1] && __uint_as_float(pt.y) >= lo[1]);
        if (DIM > 2) in &= (__uint_as_float(pt.z) <= hi[2] && __uint_as_float(pt.z) >= lo[2]);
        if (DIM > 3) in &= (__uint_as_float(pt.w) <= hi[3] && __uint_as_float(pt.w) >= lo[3]);
        if (in) {
          if (MODE == SEARCH_COUNT) {
            acc += 1u;
          } else {
            acc2 += 1u;
            acc += mix64(DIM <= 3 ? pt.w : __ldg(tab.dids + S + k));
          }
        }
      }
    }
    if (have && !bucket) {
      const uint32_t dep = floor_log2_u32(i + 1u);
      const uint32_t c = dep % DIM;
      const uint4 nd = __ldg(tab.nodes + i);
      const float x0 = __uint_as_float(nd.x), x1 = __uint_as_float(nd.y), x2 = __uint_as_float(nd.z),
                  x3 = __uint_as_float(nd.w);
      const float v = sel4(c, x0, x1, x2, x3);
      const float loc = sel4(c, lo[0], lo[1], lo[2], lo[3]);
      const float hic = sel4(c, hi[0], hi[1], hi[2], hi[3]);
      const bool inter = v <= hic && v >= loc;
      const bool lower = v < loc;
      bool emit = false;
      if (inter) {
        bool in = true;
        if (DIM > 0) in &= (x0 <= hi[0] && x0 >= lo[0]);
        if (DIM > 1) in &= (x1 <= hi[1] && x1 >= lo[1]);
        if (DIM > 2) in &= (x2 <= hi[2] && x2 >= lo[2]);
        if (DIM > 3) in &= (x3 <= hi[3] && x3 >= lo[3]);
        emit = in;
      }
      const uint32_t l = 2u * i + 1u;
      const bool visitL = !lower && l < g.n;
      const bool visitR = (lower || inter) && l + 1u < g.n;
      maskL = mask | (v <= hic ? (2u << (2 * c)) : 0u);
      maskR = mask | (v >= loc ? (1u << (2 * c)) : 0u);
      const bool contL = visitL && maskL == FULL;
      const bool contR = visitR && maskR == FULL;
      pushL = visitL && !contL;
      pushR = visitR && !contR;
      const uint32_t cnt = (emit ? 1u : 0u) + (contL ? subtree_size(g, l) : 0u) + (contR ? subtree_size(g, l + 1u) : 0u);
      if (MODE == SEARCH_COUNT) {
        acc += cnt;
      } else {
        acc2 += cnt;
        if (emit) acc += mix64(DIM <= 3 ? nd.w : __ldg(tab.ids + i));
        if (contL) acc += tab.sdig[l];
        if (contR) acc += tab.sdig[l + 1u];
      }
    }
    const uint32_t bpl = (__ballot_sync(0xffffffffu, pushL) >> gsh) & GM;
    const uint32_t bpr = (__ballot_sync(0xffffffffu, pushR) >> gsh) & GM;
    const uint32_t tot = __popc(bpl) + __popc(bpr);
    if ((uint32_t)top + tot > cap) {
      failed = true;  // group-uniform: abandon the box, report capacity
      top = 0;
    } else {
      uint32_t p = (uint32_t)top + __popc(bpl & glt) + __popc(bpr & glt);
      // children at the bucket depth go on the stack as buckets
      const uint32_t btag = (BKT && (pushL || pushR) && floor_log2_u32(i + 1u) + 1u >= bdep) ? BUCKET_BIT : 0u;
      if (pushL) {
        stk_node[p] = (2u * i + 1u) | btag;
        stk_mask[p] = (uint8_t)maskL;
        ++p;
      }
      if (pushR) {
        stk_node[p] = (2u * i + 2u) | btag;
        stk_mask[p] = (uint8_t)maskR;
      }
      top += (int)tot;
    }
    __syncwarp();
    if (active && top == 0) finish();
  }
}

template <int DIM, int MODE, int G, bool BKT>
static cudaError_t run_search_grp_b(SearchCtx& sc) {
  const uint32_t cap = stack_cap_lanes(sc.g, G);
  const size_t smem = (size_t)(QT / G) * cap * 5u;
  cudaError_t e =
      cudaFuncSetAttribute(k_search_grp<DIM, MODE, G, BKT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_search_grp<DIM, MODE, G, BKT>, QT, smem);
  if (e != cudaSuccess) return e;
  if (per < 1) per = 1;
  uint64_t blocks = (uint64_t)sms * per;
  const uint64_t need = (sc.boxes.q + (QT / G) - 1) / (QT / G);
  if (blocks > need) blocks = need ? need : 1;
  e = cudaMemsetAsync(sc.qcounter, 0, sizeof(uint32_t), sc.stream);
  if (e != cudaSuccess) return e;
  k_search_grp<DIM, MODE, G, BKT><<<(unsigned)blocks, QT, smem, sc.stream>>>(sc, cap);
  count_launches(1);
  return cudaGetLastError();
}

// The leaf-bucket variant only when buckets are asked for: the plain kernel
// stays free of the bucket branch.
template <int DIM, int MODE, int G>
static cudaError_t run_search_grp(SearchCtx& sc) {
  if (sc.tab.ipts && sc.bucket_grp) return run_search_grp_b<DIM, MODE, G, true>(sc);
  return run_search_grp_b<DIM, MODE, G, false>(sc);
}

template <int DIM, int MODE, bool REC = false>
static cudaError_t run_search(SearchCtx& sc) {
  if constexpr (MODE == SEARCH_COUNT && !REC) {
    if (sc.pool_st) return run_search<DIM, MODE, true>(sc);
  }
  const uint32_t cap = stack_cap(sc.g, sc.tab.ipts ? sc.bucket : 0u);
  const size_t smem = (size_t)QW * cap * 5u;
  cudaError_t e =
      cudaFuncSetAttribute(k_search<DIM, MODE, REC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_search<DIM, MODE, REC>, QT, smem);
  if (e != cudaSuccess) return e;
  if (per < 1) per = 1;
  uint64_t blocks = (uint64_t)sms * per;
  const uint64_t need = (sc.boxes.q + QW - 1) / QW;
  if (blocks > need) blocks = need ? need : 1;
  e = cudaMemsetAsync(sc.qcounter, 0, sizeof(uint32_t), sc.stream);
  if (e != cudaSuccess) return e;
  k_search<DIM, MODE, REC><<<(unsigned)blocks, QT, smem, sc.stream>>>(sc, cap);
  count_launches(1);
  return cudaGetLastError();
}

template <int DIM, int MODE>
static cudaError_t run_search_lanes(SearchCtx& sc) {
  switch (sc.lanes) {
    case 1: return run_search_grp<DIM, MODE, 1>(sc);
    case 2: return run_search_grp<DIM, MODE, 2>(sc);
    case 4: return run_search_grp<DIM, MODE, 4>(sc);
    case 8: return run_search_grp<DIM, MODE, 8>(sc);
    case 16: return run_search_grp<DIM, MODE, 16>(sc);
    default: return run_search<DIM, MODE>(sc);
  }
}

template <int DIM>
static cudaError_t run_search_mode(SearchCtx& sc, int mode) {
  if (sc.lanes != 0 && sc.lanes != 32) {
    if (mode == SEARCH_COUNT) return run_search_lanes<DIM, SEARCH_COUNT>(sc);
    if (mode == SEARCH_DIGEST) return run_search_lanes<DIM, SEARCH_DIGEST>(sc);
  }
  switch (mode) {
    case SEARCH_COUNT: return run_search<DIM, SEARCH_COUNT>(sc);
    case SEARCH_WRITE: return run_search<DIM, SEARCH_WRITE>(sc);
    default: return run_search<DIM, SEARCH_DIGEST>(sc);
  }
}

cudaError_t launch_search(SearchCtx& sc, int dim, int mode) {
  if (sc.boxes.q == 0) return cudaSuccess;
  switch (dim) {
    case 1: return run_search_mode<1>(sc, mode);
    case 2: return run_search_mode<2>(sc, mode);
    case 3: return run_search_mode<3>(sc, mode);
    case 4: return run_search_mode<4>(sc, mode);
    default: return cudaErrorInvalidValue;
  }
}

// ----------------------------------------------------------- in-order table
//
// Node (d, t) owns the interval [start(d,t), start(d,t) + len(d,t)) of the
// build's working order and sits at start + rank(d,t) inside it (its left
// subtree before it, its right subtree after it): the in-order position.
// dids / dnode list the ids / heap indices in that order, so every subtree
// is one contiguous range of them.

__global__ void k_inorder(Geom g, const uint32_t* __restrict__ ids, const uint4* __restrict__ nodes,
                          uint32_t* __restrict__ dids, uint32_t* __restrict__ dnode, uint4* __restrict__ ipts) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
    const uint32_t d = floor_log2_u32(i + 1u);
    const uint32_t t = i + 1u - (1u << d);
    const uint32_t p = seg_start(g, d, t) + (d < g.H ? seg_rank(g, d, t) : 0u);
    dids[p] = ids[i];
    dnode[p] = i;
    if (ipts) ipts[p] = nodes[i];
  }
}

cudaError_t launch_inorder(const Geom& g, Table tab, cudaStream_t stream) {
  if (g.n == 0) return cudaSuccess;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  uint32_t blocks = (g.n + 255u) / 256u;
  const uint32_t cap = (uint32_t)sms * 8u;
  if (blocks > cap) blocks = cap;
  k_inorder<<<blocks, 256, 0, stream>>>(g, tab.ids, tab.nodes, tab.dids, tab.dnode, tab.ipts);
  count_launches(1);
  return cudaGetLastError();
}

// In-order tables of every event of a batch (event x in block x, grid.y
// blocks striding over its points): ipts always, dids where given (dim 4,
// whose ids do not ride in the node).  Node i of event e sits at
// ev.base + i; its in-order position at ev.base + p.
__global__ void k_inorder_events(const EvDesc* __restrict__ evs, const uint32_t* __restrict__ ids,
                                 const uint4* __restrict__ nodes, uint32_t* __restrict__ dids,
                                 uint4* __restrict__ ipts) {
  const EvDesc ev = evs[blockIdx.x];
  const Geom g = ev.g;
  for (uint32_t i = blockIdx.y * blockDim.x + threadIdx.x; i < g.n; i += gridDim.y * blockDim.x) {
    const uint32_t d = floor_log2_u32(i + 1u);
    const uint32_t t = i + 1u - (1u << d);
    const uint32_t p = seg_start(g, d, t) + (d < g.H ? seg_rank(g, d, t) : 0u);
    ipts[ev.base + p] = nodes[ev.base + i];
    if (dids) dids[ev.base + p] = ids[ev.base + i];
  }
}

cudaError_t launch_inorder_events(const EvDesc* evs, uint32_t nev, uint32_t max_n, Table tab, cudaStream_t stream) {
  if (nev == 0 || max_n == 0) return cudaSuccess;
  const uint32_t gy = (max_n + 255u) / 256u < 16u ? (max_n + 255u) / 256u : 16u;
  k_inorder_events<<<dim3(nev, gy), 256, 0, stream>>>(evs, tab.ids, tab.nodes, tab.dids, tab.ipts);
  count_launches(1);
  return cudaGetLastError();
}

// ---------------------------------------------------------- subtree digests
//
// sdig[i] = mix64(id_i) + sdig[2i+1] + sdig[2i+2] (mod 2^64), level by level
// from the deepest level up.  Block x handles event x (grid.y blocks share an
// event's level).  With it a digest search adds one entry per contained
// subtree instead of hashing every id in it.

__global__ void k_sdig_level(uint32_t d, const EvDesc* __restrict__ evs, Table tab) {
  const EvDesc ev = evs[blockIdx.x];
  const uint32_t n = ev.g.n;
  if (d > ev.g.H || n == 0) return;
  const uint32_t a = (1u << d) - 1u;
  const uint32_t b = min(n, (2u << d) - 1u);
  const uint32_t* ids = tab.ids + ev.base;
  unsigned long long* sd = tab.sdig + ev.base;
  for (uint32_t i = a + blockIdx.y * blockDim.x + threadIdx.x; i < b; i += gridDim.y * blockDim.x) {
    unsigned long long v = mix64(ids[i]);
    const uint32_t l = 2u * i + 1u;
    if (l < n) v += sd[l];
    if (l + 1u < n) v += sd[l + 1u];
    sd[i] = v;
  }
}

cudaError_t launch_subtree_digests(const EvDesc* evs, uint32_t nev, uint32_t max_n, Table tab, cudaStream_t stream) {
  if (nev == 0 || max_n == 0) return cudaSuccess;
  const uint32_t H = floor_log2_u32(max_n);
  for (int d = (int)H; d >= 0; --d) {
    const uint32_t width = 1u << d;
    uint32_t gy = (width + 255u) / 256u;
    const uint32_t cap = nev >= 1024u ? 1u : 4096u / nev;
    if (gy > cap) gy = cap;
    if (gy < 1u) gy = 1u;
    k_sdig_level<<<dim3(nev, gy), 256, 0, stream>>>((uint32_t)d, evs, tab);
    count_launches(1);
  }
  return cudaGetLastError();
}

// ------------------------------------------------------------ box order
//
// Boxes are processed in the order of the tree cell their centre falls in
// (the root-to-depth-D path of the centre, D = min(H, 16)), so the warps
// running at the same time walk neighbouring parts of the tree and share
// its nodes in L2.  The order only changes which warp does which box, never
// a box's result.

constexpr int QO_BITS = 16;

template <int DIM>
__global__ void k_box_keys(Geom g, Table tab, Boxes b, uint32_t* __restrict__ keys, uint32_t* __restrict__ hist) {
  const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= b.q) return;
  float ctr[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int c = 0; c < DIM; ++c) ctr[c] = 0.5f * (b.lo[(uint64_t)c * b.stride + j] + b.hi[(uint64_t)c * b.stride + j]);
  const uint32_t D = g.H < (uint32_t)QO_BITS ? g.H : (uint32_t)QO_BITS;
  uint32_t i = 0u, path = 0u, dep = 0u;
  while (dep < D) {
    const uint32_t c = dep % DIM;
    const uint4 nd = __ldg(tab.nodes + i);
    const float v = sel4(c, __uint_as_float(nd.x), __uint_as_float(nd.y), __uint_as_float(nd.z), __uint_as_float(nd.w));
    const uint32_t right = (sel4(c, ctr[0], ctr[1], ctr[2], ctr[3]) < v) ? 0u : 1u;
    path = (path << 1) | right;
    i = 2u * i + 1u + right;
    ++dep;
    if (i >= g.n) break;
  }
  const uint32_t key = path << (QO_BITS - dep);
  keys[j] = key;
  atomicAdd(&hist[key], 1u);
}

__global__ void k_box_scatter(uint64_t q, const uint32_t* __restrict__ keys, unsigned long long* __restrict__ offs,
                              uint32_t* __restrict__ order) {
  const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= q) return;
  const unsigned long long pos = atomicAdd(&offs[keys[j]], 1ull);
  if (pos < q) order[pos] = (uint32_t)j;
}

size_t box_order_words(uint64_t q) {
  // keys (q) + hist (2^16) + offsets (2^16 + 1, 64-bit) + partials + order (q)
  return q + (1u << QO_BITS) + 2ull * ((1u << QO_BITS) + 1) + 2ull * scan_partials_words(1u << QO_BITS) + q + 16;
}

cudaError_t launch_box_order(const Geom& g, const Table& tab, const Boxes& b, int dim, uint32_t* scratch,
                             uint32_t** order_out, cudaStream_t stream) {
  *order_out = nullptr;
  if (b.q == 0 || g.n == 0) return cudaSuccess;
  uint32_t* keys = scratch;
  uint32_t* hist = keys + b.q;
  unsigned long long* offs = (unsigned long long*)(((uintptr_t)(hist + (1u << QO_BITS)) + 15) & ~(uintptr_t)15);
  unsigned long long* partials = offs + (1u << QO_BITS) + 1;
  uint32_t* order = (uint32_t*)(partials + scan_partials_words(1u << QO_BITS));
  cudaError_t e = cudaMemsetAsync(hist, 0, sizeof(uint32_t) << QO_BITS, stream);
  if (e != cudaSuccess) return e;
  const unsigned blocks = (unsigned)((b.q + 255) / 256);
  switch (dim) {
    case 1: k_box_keys<1><<<blocks, 256, 0, stream>>>(g, tab, b, keys, hist); break;
    case 2: k_box_keys<2><<<blocks, 256, 0, stream>>>(g, tab, b, keys, hist); break;
    case 3: k_box_keys<3><<<blocks, 256, 0, stream>>>(g, tab, b, keys, hist); break;
    default: k_box_keys<4><<<blocks, 256, 0, stream>>>(g, tab, b, keys, hist); break;
  }
  count_launches(1);
  e = launch_scan_counts(hist, 1u << QO_BITS, (uint64_t*)offs, partials, stream);
  if (e != cudaSuccess) return e;
  k_box_scatter<<<blocks, 256, 0, stream>>>(b.q, keys, offs, order);
  count_launches(1);
  *order_out = order;
  return cudaGetLastError();
}

// ------------------------------------------------------------------- scan

constexpr int SCT = 256;
constexpr int SCIPT = 16;
constexpr int SCB = SCT * SCIPT;

size_t scan_partials_words(uint64_t q) { return (q + SCB - 1) / SCB + 1; }

__device__ __forceinline__ unsigned long long block_excl_scan64(unsigned long long v, unsigned long long* wsum,
                                                                unsigned long long* total) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  unsigned long long incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (uint32_t)o) incl += y;
  }
  if (lane == 31u) wsum[warp] = incl;
  __syncthreads();
  unsigned long long base = 0ull, tot = 0ull;
  for (uint32_t k = 0; k < blockDim.x / 32u; ++k) {
    if (k < warp) base += wsum[k];
    tot += wsum[k];
  }
  __syncthreads();
  *total = tot;
  return base + incl - v;
}

__global__ void __launch_bounds__(SCT) k_scan_partials(const uint32_t* __restrict__ counts, uint64_t q,
                                                       unsigned long long* __restrict__ partials) {
  __shared__ unsigned long long wsum[SCT / 32];
  const uint64_t b0 = (uint64_t)blockIdx.x * SCB;
  unsigned long long s = 0ull;
#pragma unroll
  for (int k = 0; k < SCIPT; ++k) {
    const uint64_t i = b0 + (uint64_t)k * SCT + threadIdx.x;
    if (i < q) s += counts[i];
  }
  unsigned long long tot;
  block_excl_scan64(s, wsum, &tot);
  if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) k_scan_top(unsigned long long* __restrict__ partials, uint64_t nb) {
  __shared__ unsigned long long wsum[32];
  unsigned long long carry = 0ull;
  for (uint64_t c0 = 0; c0 < nb; c0 += blockDim.x) {
    const uint64_t i = c0 + threadIdx.x;
    const unsigned long long v = i < nb ? partials[i] : 0ull;
    unsigned long long tot;
    const unsigned long long ex = block_excl_scan64(v, wsum, &tot);
    if (i < nb) partials[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) partials[nb] = carry;
}

__global__ void __launch_bounds__(SCT) k_scan_down(const uint32_t* __restrict__ counts, uint64_t q,
                                                   const unsigned long long* __restrict__ partials,
                                                   uint64_t* __restrict__ offsets, uint64_t nb) {
  __shared__ unsigned long long wsum[SCT / 32];
  const uint64_t b0 = (uint64_t)blockIdx.x * SCB;
  // each thread owns SCIPT consecutive counts
  const uint64_t t0 = b0 + (uint64_t)threadIdx.x * SCIPT;
  uint32_t v[SCIPT];
  unsigned long long s = 0ull;
#pragma unroll
  for (int k = 0; k < SCIPT; ++k) {
    v[k] = (t0 + k < q) ? counts[t0 + k] : 0u;
    s += v[k];
  }
  unsigned long long tot;
  unsigned long long run = partials[blockIdx.x] + block_excl_scan64(s, wsum, &tot);
#pragma unroll
  for (int k = 0; k < SCIPT; ++k) {
    if (t0 + k < q) offsets[t0 + k] = run;
    run += v[k];
  }
  if (blockIdx.x == nb - 1 && threadIdx.x == 0) offsets[q] = partials[nb];
}

cudaError_t launch_scan_counts(const uint32_t* counts, uint64_t q, uint64_t* offsets, unsigned long long* partials,
                               cudaStream_t stream) {
  if (q == 0) return cudaMemsetAsync(offsets, 0, sizeof(uint64_t), stream);
  const uint64_t nb = (q + SCB - 1) / SCB;
  k_scan_partials<<<(unsigned)nb, SCT, 0, stream>>>(counts, q, partials);
  count_launches(1);
  k_scan_top<<<1, 1024, 0, stream>>>(partials, nb);
  count_launches(1);
  k_scan_down<<<(unsigned)nb, SCT, 0, stream>>>(counts, q, partials, offsets, nb);
  count_launches(1);
  return cudaGetLastError();
}

// ------------------------------------------------------ ordered results
//
// search_in_the_box and its BFS / branchless variants emit the in-box nodes
// level by level in frontier order, and the frontier of every level is sorted
// by heap index (children are appended in order), so their output is the
// in-box set sorted by heap index.  For that order the write pass stores heap
// indices, this kernel sorts each box's slice and replaces the indices by ids.

constexpr int OT = 256;
constexpr int ORUN = 8192;  // slice length sorted in shared memory

__device__ void bitonic_smem(uint32_t* a, uint32_t m) {  // m a power of two
  for (uint32_t k = 2; k <= m; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
        const uint32_t p = i ^ j;
        if (p > i) {
          const uint32_t x = a[i], y = a[p];
          const bool up = (i & k) == 0;
          if ((x > y) == up) {
            a[i] = y;
            a[p] = x;
          }
        }
      }
      __syncthreads();
    }
  }
}

// Merges sorted runs a[0,la) and b[0,lb) into o (distinct keys), CTA-wide by
// merge-path partitioning.
__device__ void merge_cta(const uint32_t* a, uint32_t la, const uint32_t* b, uint32_t lb, uint32_t* o) {
  const uint32_t total = la + lb;
  const uint32_t per = (total + blockDim.x - 1) / blockDim.x;
  const uint32_t k0 = min(total, threadIdx.x * per), k1 = min(total, k0 + per);
  if (k0 >= k1) return;
  // find i in [max(0,k0-lb), min(k0,la)] with a[i-1] < b[k0-i] and b[k0-i-1] < a[i]
  uint32_t lo = k0 > lb ? k0 - lb : 0u, hi = k0 < la ? k0 : la;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a[mid] < b[k0 - mid - 1u])
      lo = mid + 1u;
    else
      hi = mid;
  }
  uint32_t i = lo, j = k0 - lo;
  for (uint32_t k = k0; k < k1; ++k) {
    if (j >= lb || (i < la && a[i] < b[j]))
      o[k] = a[i++];
    else
      o[k] = b[j++];
  }
}

__global__ void __launch_bounds__(OT) k_order(Geom g, Table tab, const uint64_t* __restrict__ offsets, uint64_t q,
                                              uint32_t* __restrict__ out, uint32_t* __restrict__ tmp,
                                              uint32_t* __restrict__ err) {
  __shared__ uint32_t buf[ORUN];
  for (uint64_t qj = blockIdx.x; qj < q; qj += gridDim.x) {
    const uint64_t s0 = offsets[qj];
    const uint32_t len = (uint32_t)(offsets[qj + 1] - s0);
    uint32_t* seg = out + s0;
    uint32_t* alt = tmp + s0;
    if (len > 1u) {
      // sort runs of ORUN in shared memory
      for (uint32_t r0 = 0; r0 < len; r0 += ORUN) {
        const uint32_t rl = min((uint32_t)ORUN, len - r0);
        uint32_t m = 1u;
        while (m < rl) m <<= 1;
        for (uint32_t i = threadIdx.x; i < m; i += OT) buf[i] = i < rl ? seg[r0 + i] : 0xffffffffu;
        __syncthreads();
        bitonic_smem(buf, m);
        for (uint32_t i = threadIdx.x; i < rl; i += OT) seg[r0 + i] = buf[i];
        __syncthreads();
      }
      // merge runs pairwise, ping-ponging between out and tmp
      uint32_t* src = seg;
      uint32_t* dst = alt;
      for (uint32_t w = ORUN; w < len; w <<= 1) {
        for (uint32_t a0 = 0; a0 < len; a0 += 2u * w) {
          const uint32_t la = min(w, len - a0);
          const uint32_t lb = (a0 + w < len) ? min(w, len - a0 - w) : 0u;
          merge_cta(src + a0, la, src + a0 + la, lb, dst + a0);
        }
        __syncthreads();
        uint32_t* t = src;
        src = dst;
        dst = t;
      }
      if (src != seg) {
        for (uint32_t i = threadIdx.x; i < len; i += OT) seg[i] = src[i];
        __syncthreads();
      }
    }
    for (uint32_t i = threadIdx.x; i < len; i += OT) {
      const uint32_t hidx = seg[i];
      if (hidx < g.n) {
        seg[i] = __ldg(tab.ids + hidx);
      } else {
        seg[i] = 0xffffffffu;
        atomicOr(err, ERRB_INTERNAL);
      }
    }
    __syncthreads();
  }
}

cudaError_t launch_order_results(const Geom& g, const Table& tab, const uint64_t* offsets, uint64_t q, uint32_t* out,
                                 uint32_t* tmp, uint32_t* err, cudaStream_t stream) {
  if (q == 0) return cudaSuccess;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t blocks = q < (uint64_t)sms * 8 ? q : (uint64_t)sms * 8;
  k_order<<<(unsigned)blocks, OT, 0, stream>>>(g, tab, offsets, q, out, tmp, err);
  count_launches(1);
  return cudaGetLastError();
}

// One box with a host round trip (a caller that searches box by box, as the
// reference's driver does from its TBB loop, main.cpp:351-359): a single warp
// walks the tree level by level like search_in_the_box (FKDTree_cpu.h:
// 123-169) -- the frontier of each depth in ascending heap order, the left
// child visited when min <= split value, the right when split value <= max --
// so the in-box nodes come out in ascending heap order, the reference's list,
// with no count pass, scan or sort.  out[0] = results (all of them, also past
// cap), out[1] = 1 when a depth's frontier outgrew ONE_FRONTIER (the caller
// then takes the general path), out[4 ..] = the first cap ids.
constexpr uint32_t ONE_FRONTIER = 2048;
template <int DIM>
__global__ void __launch_bounds__(32) k_one(Table tab, uint32_t n, OneBox bx, uint32_t* __restrict__ out,
                                            uint32_t cap) {
  __shared__ uint32_t fr[2][ONE_FRONTIER];
  const uint32_t lane = threadIdx.x;
  const uint32_t lt = (1u << lane) - 1u;
  uint32_t nf = n ? 1u : 0u, total = 0u, cur = 0u;
  bool ovf = false;
  if (lane == 0) fr[0][0] = 0u;
  __syncwarp();
  for (uint32_t d = 0; nf > 0u && !ovf; ++d) {
    const uint32_t c = d % DIM;
    uint32_t nn = 0u;
    for (uint32_t b0 = 0; b0 < nf; b0 += 32u) {
      const uint32_t i = b0 + lane;
      const bool v = i < nf;
      const uint32_t node = v ? fr[cur][i] : 0u;
      uint4 p = make_uint4(0u, 0u, 0u, 0u);
      if (v) p = __ldg(tab.nodes + node);
      const float x[4] = {__uint_as_float(p.x), __uint_as_float(p.y), __uint_as_float(p.z), __uint_as_float(p.w)};
      bool in = v;
#pragma unroll
      for (int w = 0; w < DIM; ++w) in &= bx.lo[w] <= x[w] && x[w] <= bx.hi[w];
      const float sv = sel4(c, x[0], x[1], x[2], x[3]);
      const float lo = sel4(c, bx.lo[0], bx.lo[1], bx.lo[2], bx.lo[3]);
      const float hi = sel4(c, bx.hi[0], bx.hi[1], bx.hi[2], bx.hi[3]);
      const bool l = v && 2ull * node + 1ull < n && lo <= sv;
      const bool r = v && 2ull * node + 2ull < n && sv <= hi;
      const uint32_t bin = __ballot_sync(0xffffffffu, in);
      const uint32_t at = total + __popc(bin & lt);
      if (in && at < cap) out[4 + at] = __ldg(tab.ids + node);
      total += __popc(bin);
      // children in lane order, left before right: ascending heap order
      const uint32_t k = (l ? 1u : 0u) + (r ? 1u : 0u);
      uint32_t incl = k;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
      }
      const uint32_t q0 = nn + incl - k;
      const uint32_t add = __shfl_sync(0xffffffffu, incl, 31);
      if (nn + add > ONE_FRONTIER) {
        ovf = true;  // warp-uniform
        break;
      }
      uint32_t q = q0;
      if (l) fr[cur ^ 1u][q++] = 2u * node + 1u;
      if (r) fr[cur ^ 1u][q] = 2u * node + 2u;
      nn += add;
    }
    __syncwarp();
    cur ^= 1u;
    nf = nn;
  }
  if (lane == 0) {
    out[0] = total;
    out[1] = ovf ? 1u : 0u;
  }
}

cudaError_t launch_one(const Table& tab, uint32_t n, int dim, const OneBox& bx, uint32_t* out, uint32_t cap,
                       cudaStream_t stream) {
  switch (dim) {
    case 1: k_one<1><<<1, 32, 0, stream>>>(tab, n, bx, out, cap); break;
    case 2: k_one<2><<<1, 32, 0, stream>>>(tab, n, bx, out, cap); break;
    case 3: k_one<3><<<1, 32, 0, stream>>>(tab, n, bx, out, cap); break;
    case 4: k_one<4><<<1, 32, 0, stream>>>(tab, n, bx, out, cap); break;
    default: return cudaErrorInvalidValue;
  }
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace fkd
