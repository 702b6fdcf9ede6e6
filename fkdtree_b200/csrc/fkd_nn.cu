// fkd_nn.cu -- radius (ball) search and k-nearest-neighbour search on the
// flat tree.
//
// No reference counterpart: the reference answers axis-aligned boxes only
// (FKDTree_cpu.h:25-207).  Both searches walk the tree the reference builds
// with its own split rule -- node i splits coordinate depth(i) % dim at its
// own point; its left subtree holds points whose coordinate is <= the split
// value and its right subtree points whose coordinate is >= it
// (FKDTree_cpu.h:240-269) -- and skip a subtree only when the distance from
// the query to the split plane proves that none of its points can qualify.
//
// Distances are squared Euclidean distances in float32, every operation
// rounded on its own (no fused multiply-add):
//
//     d2 = (((0 + (p0-q0)^2) + (p1-q1)^2) + (p2-q2)^2) + (p3-q3)^2
//
// so a restatement that evaluates the same expression in the same order gets
// the same bits.  The plane bound fl((q_a - s)^2) is a lower bound of d2 for
// every point beyond the plane: rounding is monotone, so |fl(p_a - q_a)| >=
// |fl(s - q_a)|, and adding non-negative rounded terms never lowers a sum.
// The pruning therefore never drops a qualifying point.  (When q_a - s is
// NaN -- an infinite query coordinate meeting the same infinite split value --
// both sides are visited.)
//
// Radius: point p qualifies for query (c, r) when d2 <= fl(r*r) and r >= 0.
//   A negative or NaN radius, or a centre with a NaN coordinate, qualifies
//   nothing.  A count pass, then a write pass: of ids in the walk's
//   depth-first order, or (ordered) of heap indices that
//   launch_order_results sorts and maps to ids -- ascending heap-index order,
//   the order of the ordered box search.
// kNN: the k points smallest in (d2, id) order, ascending.  Ties of d2 go to
//   the smaller id, so the answer depends on the point set only, not on the
//   tree.  Points whose d2 is NaN never qualify; a centre with a NaN
//   coordinate has no neighbours.  Rows with fewer than k neighbours end in
//   id 0xffffffff with d2 = +inf.
//
// Queries run in the spatial order of launch_box_order (neighbouring warps
// walk neighbouring parts of the tree and share its nodes in L1/L2).  The
// radius search runs a warp per query (below); kNN a thread per query, a
// depth-first walk with an explicit stack of pending far children whose
// depths strictly increase from the bottom of the stack to its top, so it
// never holds more than H + 1 <= 32 entries.  (Stopping the radius walk at
// subtrees whose whole cell lies inside the ball, as the box search does for
// boxes, was measured slower: kd cells are rarely inside a ball -- 11% fewer
// visits on clustered points -- and carrying the cell doubled the cost of a
// visit.)
#include <math.h>

#include "fkd_internal.h"

namespace fkd {
namespace {

constexpr int NNT = 128;      // threads per block
constexpr int NN_STACK = 32;  // H + 1 for trees below 2^31 points

template <int DIM>
__device__ __forceinline__ float node_coord(const uint4& nd, uint32_t c) {
  const uint32_t w = c == 0u ? nd.x : c == 1u ? nd.y : c == 2u ? nd.z : nd.w;
  return __uint_as_float(w);
}

template <int DIM>
__device__ __forceinline__ float node_dist2(const uint4& nd, const float (&qc)[4]) {
  float acc = 0.f;
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    const float t = __fsub_rn(node_coord<DIM>(nd, (uint32_t)c), qc[c]);
    acc = __fadd_rn(acc, __fmul_rn(t, t));
  }
  return acc;
}

template <int DIM>
__device__ __forceinline__ bool load_centre(const float* __restrict__ ctr, uint64_t q, uint64_t j, float (&qc)[4]) {
  bool ok = true;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    qc[c] = c < DIM ? ctr[(uint64_t)c * q + j] : 0.f;
    ok = ok && !(qc[c] != qc[c]);
  }
  return ok;
}

// ---------------------------------------------------------------- radius
//
// A warp per query.  The warp keeps the query's pending nodes in a
// shared-memory stack and takes up to 32 of them per round from its top, one
// per lane: each lane tests its node's point and its two children, the hits
// leave as one coalesced store at consecutive positions (ballot prefix), and
// the children are pushed back in lane order.  Lane k takes the k-th of the
// popped entries from below, so the stack stays sorted by depth (children of
// shallower nodes go lower); then a depth's entries can only come from the
// one round that popped its parents, so no depth holds more than
// min(64, 2^d) entries and the stack never exceeds 1 + sum_{d=1..H} min(64,
// 2^d) words (a check latches an error instead of overflowing).  The result
// order within a query is this walk's order (deterministic).

// Stack words per warp for a tree of depth H.
inline uint32_t radius_stack_words(uint32_t H) {
  uint32_t w = 1u;
  for (uint32_t d = 1; d <= H; ++d) w += d < 6u ? (1u << d) : 64u;
  return w;
}

template <int DIM, int MODE>  // MODE 0: counts, 1: ids, 2: heap indices
__global__ void __launch_bounds__(NNT) k_radius(Geom g, const uint4* __restrict__ nodes,
                                                const uint32_t* __restrict__ ids, const float* __restrict__ ctr,
                                                const float* __restrict__ rad, uint64_t q,
                                                const uint32_t* __restrict__ order, uint32_t* __restrict__ counts,
                                                const uint64_t* __restrict__ offsets, uint32_t* __restrict__ out,
                                                uint32_t cap, uint32_t* __restrict__ err) {
  extern __shared__ uint32_t nn_stack[];
  const uint32_t lane = threadIdx.x & 31u, wp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  uint32_t* stk = nn_stack + (size_t)wp * cap;
  const uint64_t t = (uint64_t)blockIdx.x * (NNT / 32) + wp;  // warp-uniform
  if (t >= q) return;
  const uint64_t j = order ? (uint64_t)order[t] : t;
  if (j >= q) {
    if (lane == 0u) atomicOr(err, ERRB_INTERNAL);
    return;
  }
  float qc[4];
  const bool centre_ok = load_centre<DIM>(ctr, q, j, qc);
  const float r = rad[j];
  uint64_t base = 0ull, room = 0ull;
  if (MODE != 0) {
    base = offsets[j];
    room = offsets[j + 1] - base;
  }
  uint64_t found = 0ull;
  if (centre_ok && r >= 0.f && g.n > 0u) {
    const float r2 = __fmul_rn(r, r);
    if (lane == 0u) stk[0] = 0u;
    uint32_t sp = 1u;
    __syncwarp();
    while (sp > 0u) {
      const uint32_t cnt = sp < 32u ? sp : 32u;
      const uint32_t b0 = sp - cnt;
      const bool act = lane < cnt;
      const uint32_t i = act ? stk[b0 + lane] : 0u;
      __syncwarp();  // every entry read before the pushes overwrite them
      bool hit = false, go_l = false, go_r = false;
      uint32_t v = 0u;
      const uint32_t l = 2u * i + 1u;
      if (act) {
        const uint4 nd = __ldg(nodes + i);
        hit = node_dist2<DIM>(nd, qc) <= r2;
        if (MODE == 1) v = DIM <= 3 ? nd.w : (hit ? __ldg(ids + i) : 0u);
        if (MODE == 2) v = i;
        const uint32_t a = floor_log2_u32(i + 1u) % (uint32_t)DIM;
        const float diff = __fsub_rn(qc[a], node_coord<DIM>(nd, a));
        const float pd = __fmul_rn(diff, diff);
        // the left side holds coordinates <= s: beyond reach when q_a > s and
        // the plane is farther than r; the right side mirrors it
        go_l = l < g.n && !(diff > 0.f && pd > r2);
        go_r = l + 1u < g.n && !(diff < 0.f && pd > r2);
      }
      const uint32_t hm = __ballot_sync(0xffffffffu, hit);
      if (MODE != 0 && hit) {
        const uint64_t pos = found + __popc(hm & lt);
        if (pos < room)
          out[base + pos] = v;
        else
          atomicOr(err, ERRB_INTERNAL);
      }
      found += __popc(hm);
      const uint32_t ml = __ballot_sync(0xffffffffu, go_l), mr = __ballot_sync(0xffffffffu, go_r);
      const uint32_t np = b0 + __popc(ml) + __popc(mr);
      if (np > cap) {  // not reachable by the bound above
        if (lane == 0u) atomicOr(err, ERRB_INTERNAL);
        break;
      }
      uint32_t p = b0 + __popc(ml & lt) + __popc(mr & lt);
      if (go_l) stk[p++] = l;
      if (go_r) stk[p] = l + 1u;
      sp = np;
      __syncwarp();
    }
  }
  if (lane == 0u) {
    if (MODE == 0)
      counts[j] = (uint32_t)found;
    else if (found != room)
      atomicOr(err, ERRB_INTERNAL);
  }
}

// (d2, id) < (bd, bi)
__device__ __forceinline__ bool nn_less(float d2, uint32_t id, float bd, uint32_t bi) {
  return d2 < bd || (d2 == bd && id < bi);
}

template <int DIM>
__global__ void __launch_bounds__(NNT) k_knn(Geom g, const uint4* __restrict__ nodes, const uint32_t* __restrict__ ids,
                                             const float* __restrict__ ctr, uint64_t q,
                                             const uint32_t* __restrict__ order, uint32_t k,
                                             uint32_t* __restrict__ out_ids, float* __restrict__ out_d2,
                                             uint32_t* __restrict__ err) {
  const uint64_t t = (uint64_t)blockIdx.x * NNT + threadIdx.x;
  if (t >= q) return;
  const uint64_t j = order ? (uint64_t)order[t] : t;
  if (j >= q || k == 0u || k > KNN_MAX) {
    atomicOr(err, ERRB_INTERNAL);
    return;
  }
  float qc[4];
  const bool centre_ok = load_centre<DIM>(ctr, q, j, qc);
  float bd[KNN_MAX];
  uint32_t bi[KNN_MAX];
  uint32_t cnt = 0u;
  if (centre_ok && g.n > 0u) {
    uint32_t st_i[NN_STACK];
    float st_d[NN_STACK];
    int sp = 0;
    uint32_t i = 0u;
    for (;;) {
      for (;;) {
        const uint4 nd = __ldg(nodes + i);
        const float d2 = node_dist2<DIM>(nd, qc);
        const float worst = cnt < k ? INFINITY : bd[k - 1u];
        if (d2 <= worst) {
          const uint32_t id = DIM <= 3 ? nd.w : __ldg(ids + i);
          if (cnt < k || nn_less(d2, id, bd[k - 1u], bi[k - 1u])) {
            uint32_t p = cnt < k ? cnt : k - 1u;
            while (p > 0u && nn_less(d2, id, bd[p - 1u], bi[p - 1u])) {
              bd[p] = bd[p - 1u];
              bi[p] = bi[p - 1u];
              --p;
            }
            bd[p] = d2;
            bi[p] = id;
            if (cnt < k) ++cnt;
          }
        }
        const uint32_t a = floor_log2_u32(i + 1u) % (uint32_t)DIM;
        const float diff = __fsub_rn(qc[a], node_coord<DIM>(nd, a));
        // lower bound of d2 beyond the plane (0 when it is not a number)
        const float bound = diff == diff ? __fmul_rn(diff, diff) : 0.f;
        const uint32_t l = 2u * i + 1u;
        const bool near_left = !(diff > 0.f);
        const uint32_t nearc = near_left ? l : l + 1u;
        const uint32_t farc = near_left ? l + 1u : l;
        const bool has_near = nearc < g.n, has_far = farc < g.n;
        const float w2 = cnt < k ? INFINITY : bd[k - 1u];
        const bool want_far = has_far && bound <= w2;
        if (has_near) {
          if (want_far) {
            if (sp < NN_STACK) {
              st_i[sp] = farc;
              st_d[sp] = bound;
              ++sp;
            } else {
              atomicOr(err, ERRB_INTERNAL);
            }
          }
          i = nearc;
        } else if (want_far) {
          i = farc;
        } else {
          break;
        }
      }
      // next pending subtree still within reach
      bool found = false;
      while (sp > 0) {
        --sp;
        const float w2 = cnt < k ? INFINITY : bd[k - 1u];
        if (st_d[sp] <= w2) {
          i = st_i[sp];
          found = true;
          break;
        }
      }
      if (!found) break;
    }
  }
  const uint64_t row = j * (uint64_t)k;
  for (uint32_t m = 0; m < k; ++m) {
    const bool have = m < cnt;
    out_ids[row + m] = have ? bi[m] : 0xffffffffu;
    if (out_d2) out_d2[row + m] = have ? bd[m] : INFINITY;
  }
}

template <int DIM, int MODE>
cudaError_t radius_mode(const Geom& g, const Table& tab, const float* ctr, const float* rad, uint64_t q,
                        const uint32_t* order, uint32_t* counts, const uint64_t* offsets, uint32_t* out, uint32_t* err,
                        cudaStream_t stream) {
  const uint32_t cap = radius_stack_words(g.H);
  const size_t smem = (size_t)(NNT / 32) * cap * sizeof(uint32_t);
  const uint64_t blocks = (q + NNT / 32 - 1) / (NNT / 32);
  k_radius<DIM, MODE><<<(unsigned)blocks, NNT, smem, stream>>>(g, tab.nodes, tab.ids, ctr, rad, q, order, counts,
                                                               offsets, out, cap, err);
  count_launches(1);
  return cudaGetLastError();
}

template <int DIM>
cudaError_t radius_dim(const Geom& g, const Table& tab, const float* ctr, const float* rad, uint64_t q,
                       const uint32_t* order, uint32_t* counts, const uint64_t* offsets, uint32_t* out, int heap_out,
                       uint32_t* err, cudaStream_t stream) {
  if (!out) return radius_mode<DIM, 0>(g, tab, ctr, rad, q, order, counts, offsets, out, err, stream);
  if (heap_out) return radius_mode<DIM, 2>(g, tab, ctr, rad, q, order, counts, offsets, out, err, stream);
  return radius_mode<DIM, 1>(g, tab, ctr, rad, q, order, counts, offsets, out, err, stream);
}

template <int DIM>
cudaError_t knn_dim(const Geom& g, const Table& tab, const float* ctr, uint64_t q, const uint32_t* order, uint32_t k,
                    uint32_t* ids, float* d2, uint32_t* err, cudaStream_t stream) {
  const uint64_t blocks = (q + NNT - 1) / NNT;
  k_knn<DIM><<<(unsigned)blocks, NNT, 0, stream>>>(g, tab.nodes, tab.ids, ctr, q, order, k, ids, d2, err);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_radius(const Geom& g, const Table& tab, const float* ctr, const float* rad, uint64_t q,
                          const uint32_t* order, uint32_t* counts, const uint64_t* offsets, uint32_t* out,
                          int heap_out, uint32_t* err, int dim, cudaStream_t stream) {
  if (q == 0) return cudaSuccess;
  switch (dim) {
    case 1: return radius_dim<1>(g, tab, ctr, rad, q, order, counts, offsets, out, heap_out, err, stream);
    case 2: return radius_dim<2>(g, tab, ctr, rad, q, order, counts, offsets, out, heap_out, err, stream);
    case 3: return radius_dim<3>(g, tab, ctr, rad, q, order, counts, offsets, out, heap_out, err, stream);
    default: return radius_dim<4>(g, tab, ctr, rad, q, order, counts, offsets, out, heap_out, err, stream);
  }
}

cudaError_t launch_knn(const Geom& g, const Table& tab, const float* ctr, uint64_t q, const uint32_t* order,
                       uint32_t k, uint32_t* ids, float* d2, uint32_t* err, int dim, cudaStream_t stream) {
  if (q == 0) return cudaSuccess;
  switch (dim) {
    case 1: return knn_dim<1>(g, tab, ctr, q, order, k, ids, d2, err, stream);
    case 2: return knn_dim<2>(g, tab, ctr, q, order, k, ids, d2, err, stream);
    case 3: return knn_dim<3>(g, tab, ctr, q, order, k, ids, d2, err, stream);
    default: return knn_dim<4>(g, tab, ctr, q, order, k, ids, d2, err, stream);
  }
}

}  // namespace fkd
