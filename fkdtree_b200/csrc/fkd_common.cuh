// fkd_common.cuh -- shared device/host helpers of the B200 FKDTree library.
//
// Tree geometry.  The reference builds a complete binary tree in heap order
// (FKDTree_cpu.h:221-277): node i at depth d = floor(log2(i+1)) owns the
// interval theIntervalMin/Length of the working array, splits it at rank
// partition_complete_kdtree(len) (FKDTree_cpu.h:287-296) and hands the left
// part to 2i+1 and the right part to 2i+2.  Because the tree is complete, every
// interval is a closed-form function of (n, depth, index-in-level) -- the
// helpers below -- so no kernel ever stores or reads an interval table:
//
//   H = floor(log2 n)              depth of the last level (theDepth)
//   M = n - (2^H - 1)              nodes on the last level, 1 <= M <= 2^H
//   W = 2^(H-d)                    last-level span of a depth-d node
//   len(d,t)   = W - 1 + clamp(M - t*W, 0, W)
//   start(d,t) = t*W + min(M, t*W)
//   rank(d,t)  = len(d+1, 2t)      the split rank partition_complete_kdtree
//                                  returns for len(d,t)
//
// (tests/test_geometry.py checks these against the reference's own interval
// recurrence for every node of many tree sizes.)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define FKD_HD __host__ __device__ __forceinline__

namespace fkd {

struct Geom {
  uint32_t n;  // points
  uint32_t H;  // depth of the last level
  uint32_t M;  // nodes on the last level
};

FKD_HD uint32_t floor_log2_u32(uint32_t x) {
#ifdef __CUDA_ARCH__
  return 31u - (uint32_t)__clz(x | 1u);
#else
  return 31u - (uint32_t)__builtin_clz(x | 1u);
#endif
}

inline Geom make_geom(uint32_t n) {
  Geom g;
  g.n = n;
  g.H = floor_log2_u32(n);
  g.M = n ? n - ((1u << g.H) - 1u) : 0u;
  return g;
}

// (Device code uses 32-bit arithmetic: a tree holds fewer than 2^31 points,
// so t * W <= 2^H < 2^31 and no term overflows; host code keeps 64 bits.)
FKD_HD uint32_t seg_len(const Geom& g, uint32_t d, uint32_t t) {
#ifdef __CUDA_ARCH__
  const uint32_t W = 1u << (g.H - d);
  const uint32_t tw = t * W;
  return W - 1u + (g.M > tw ? min(g.M - tw, W) : 0u);
#else
  const uint64_t W = 1ull << (g.H - d);
  const uint64_t tw = (uint64_t)t * W;
  const uint64_t last = (uint64_t)g.M > tw ? (((uint64_t)g.M - tw) < W ? ((uint64_t)g.M - tw) : W) : 0ull;
  return (uint32_t)(W - 1ull + last);
#endif
}

FKD_HD uint32_t seg_start(const Geom& g, uint32_t d, uint32_t t) {
#ifdef __CUDA_ARCH__
  const uint32_t tw = t << (g.H - d);
  return tw + min(g.M, tw);
#else
  const uint64_t tw = (uint64_t)t << (g.H - d);
  return (uint32_t)(tw + ((uint64_t)g.M < tw ? (uint64_t)g.M : tw));
#endif
}

// Split rank of node (d, t), d < H: the size of its left subtree.
FKD_HD uint32_t seg_rank(const Geom& g, uint32_t d, uint32_t t) { return seg_len(g, d + 1, 2u * t); }

// Subtree size of heap node i.
FKD_HD uint32_t subtree_size(const Geom& g, uint32_t i) {
  const uint32_t d = floor_log2_u32(i + 1u);
  return seg_len(g, d, i + 1u - (1u << d));
}

// Order key of the reference comparator (FKDTree_cpu.h:246-252): the float
// mapped to an unsigned integer with the same order, -0.0 folded onto +0.0
// (they compare equal, so the tie falls to the id), then the id below it.
FKD_HD uint32_t mono_bits(uint32_t b) {
  b = (b == 0x80000000u) ? 0u : b;
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
FKD_HD uint64_t order_key(uint32_t value_bits, uint32_t id) { return ((uint64_t)mono_bits(value_bits) << 32) | id; }

FKD_HD bool is_nan_bits(uint32_t b) { return (b & 0x7fffffffu) > 0x7f800000u; }

// Digest finaliser shared with the oracle (fkd_oracle.c: fkd_mix64).
FKD_HD uint64_t mix64(uint32_t id) {
  uint64_t z = (uint64_t)id + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Device-side error latch bits (OR-ed into a word the host reads back).
enum : uint32_t {
  ERRB_NAN = 1u << 0,
  ERRB_CAPACITY = 1u << 1,
  ERRB_INTERNAL = 1u << 2,
  ERRB_TIMEOUT = 1u << 3,
};

// Records of the working arrays: DIM coordinate words then the id word, each
// an array of n uint32 (SoA), so a pass that needs one coordinate reads 4 B
// per point.
struct SoA {
  uint32_t* base;  // coordinate c of element i at base[c*stride + i]
  uint32_t* ids;   // id of element i
  uint64_t stride;
};
struct CSoA {
  const uint32_t* base;
  const uint32_t* ids;
  uint64_t stride;
};

// The built tree in device memory: nodes[i] = (c0, c1, c2, c3) with unused
// coordinates zero and, for dim <= 3, the id in the last word; ids[i] =
// theIds[i].  One 16-byte load serves a node visit of the search.
struct Table {
  uint4* nodes;
  uint32_t* ids;
  // optional: sdig[i] = sum of mix64(id) over the subtree of node i (mod 2^64),
  // filled by launch_subtree_digests before a digest search
  unsigned long long* sdig = nullptr;
  // optional: ids / heap indices in in-order position (launch_inorder), for
  // the write pass
  uint32_t* dids = nullptr;
  uint32_t* dnode = nullptr;
  // optional: the nodes in in-order position (ipts[p] = nodes[dnode[p]]), so
  // a subtree's points are one contiguous range -- the searches scan the
  // bottom subtrees ("leaf buckets") with coalesced loads instead of walking them
  uint4* ipts = nullptr;
};

}  // namespace fkd
