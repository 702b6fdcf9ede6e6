// fkd_mlp.cu -- the learned split predictor: a 40 -> 64 -> 64 -> 1 MLP with
// GELU, BF16 operands and FP32 accumulation on the tensor cores
// (mma.sync.m16n8k16 bf16; the layers are 16-row tiles of a 48x64 and a 64x64
// product, far too small for tcgen05 to pay), trained on the GPU by the
// forward / backward / Adam kernels below.  No reference counterpart.
//
// Inputs of one tree node (fkd_features.cu): the bounding box of a 256-point
// sample (6), log2 of the node's point count (1), its depth (1) and a 32-bin
// histogram of the sample along the split dimension (32).  Output: the
// position of the split value inside the sample's range along the split
// dimension, in [0, 1].
//
// Parameters (fp32 master copy, layout fixed for the C ABI):
//   W1[48][64] (rows 40..47 zero), b1[64], W2[64][64], b2[64], w3[64], b3[1]
// Forward:  Z1 = X W1 + b1, H1 = gelu(Z1), Z2 = H1 W2 + b2, H2 = gelu(Z2),
//           y = H2 . w3 + b3.  X, W1, H1, W2 are rounded to bf16 for the
//           products; everything else is fp32.  Loss = mean((y - t)^2) / 2.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <new>
#include <random>
#include <string>
#include <vector>

#include <cuda_bf16.h>

#include "../../include/fkdtree_b200.h"
#include "fkd_internal.h"
#include "fkd_mlp.h"

using namespace fkd;

namespace fkd {
fkd_status capi_fail(fkd_status s, const std::string& msg);

static_assert(FKD_MLP_IN == FKD_MLP_FEATURES, "feature width");
constexpr int MK1 = 48;  // padded input width
constexpr int MH = 64;   // hidden width
constexpr int OFF_W1 = 0, OFF_B1 = MK1 * MH, OFF_W2 = OFF_B1 + MH, OFF_B2 = OFF_W2 + MH * MH, OFF_W3 = OFF_B2 + MH,
              OFF_B3 = OFF_W3 + MH, NPARAM = OFF_B3 + 1;

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.f + erff(x * 0.70710678118654752f)) + x * 0.3989422804014327f * expf(-0.5f * x * x);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x = lo (low half), .y = hi
  return *reinterpret_cast<const uint32_t*>(&v);
}

// D += A(16x16, row) * B(16x8, col), bf16 in, fp32 accumulate
__device__ __forceinline__ void mma16816(float* d, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Fragment helpers.  For a 16-row tile with row/col accessor M(r, c):
//   A fragment of k-step kk: a[0] = M(g, 16kk + 2t .. +1), a[1] = M(g+8, ..),
//                            a[2] = M(g, 16kk + 8 + 2t ..), a[3] = M(g+8, ..)
//   B fragment (K x N, element (k, n)) of k-step kk, n-tile j:
//     b[0] = (k = 16kk + 2t .. +1, n = 8j + g), b[1] = (k + 8 ..)
//   C fragment of n-tile j: c[0..1] = (g, 8j + 2t .. +1), c[2..3] = (g+8, ..)
// with g = lane / 4, t = lane % 4.

// Weights in shared memory as bf16, B-operand friendly: Wt[n][k] (k fastest).
struct MlpSmem {
  __nv_bfloat16 w1t[MH][MK1 + 8];  // +8: bank spread
  __nv_bfloat16 w2t[MH][MH + 8];
  float b1[MH], b2[MH], w3[MH], b3;
};

__device__ void load_weights(MlpSmem& s, const float* __restrict__ p) {
  for (int i = threadIdx.x; i < MK1 * MH; i += blockDim.x) {
    const int k = i / MH, n = i % MH;
    s.w1t[n][k] = __float2bfloat16_rn(p[OFF_W1 + i]);
  }
  for (int i = threadIdx.x; i < MH * MH; i += blockDim.x) {
    const int k = i / MH, n = i % MH;
    s.w2t[n][k] = __float2bfloat16_rn(p[OFF_W2 + i]);
  }
  for (int i = threadIdx.x; i < MH; i += blockDim.x) {
    s.b1[i] = p[OFF_B1 + i];
    s.b2[i] = p[OFF_B2 + i];
    s.w3[i] = p[OFF_W3 + i];
  }
  if (threadIdx.x == 0) s.b3 = p[OFF_B3];
}

__device__ __forceinline__ void load_b(const __nv_bfloat16 (*wt)[MK1 + 8], int kk, int j, int g, int t, uint32_t* b) {
  const __nv_bfloat16* r = &wt[8 * j + g][16 * kk + 2 * t];
  b[0] = *reinterpret_cast<const uint32_t*>(r);
  b[1] = *reinterpret_cast<const uint32_t*>(r + 8);
}
__device__ __forceinline__ void load_b2(const __nv_bfloat16 (*wt)[MH + 8], int kk, int j, int g, int t, uint32_t* b) {
  const __nv_bfloat16* r = &wt[8 * j + g][16 * kk + 2 * t];
  b[0] = *reinterpret_cast<const uint32_t*>(r);
  b[1] = *reinterpret_cast<const uint32_t*>(r + 8);
}

// Forward of one 16-row tile held by a warp: X rows [r0, r0+16) of x (n x 40,
// fp32).  Leaves Z1, Z2 (pre-activations, fp32 C layout) and y for the rows
// of lanes t == 0 (y0 = row g, y1 = row g + 8).
struct Fwd {
  float z1[8][4], z2[8][4];
  float y0, y1;
};

__device__ void forward_tile(const MlpSmem& s, const float* __restrict__ x, uint64_t n, uint64_t r0, Fwd& f) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  auto X = [&](int r, int c) -> float {
    const uint64_t row = r0 + r;
    return (row < n && c < FKD_MLP_IN) ? x[row * FKD_MLP_IN + c] : 0.f;
  };
  // layer 1: 3 k-steps x 8 n-tiles
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int q = 0; q < 4; ++q) f.z1[j][q] = 0.f;
#pragma unroll
  for (int kk = 0; kk < 3; ++kk) {
    uint32_t a[4];
    const int c0 = 16 * kk + 2 * t;
    a[0] = pack_bf16(X(g, c0), X(g, c0 + 1));
    a[1] = pack_bf16(X(g + 8, c0), X(g + 8, c0 + 1));
    a[2] = pack_bf16(X(g, c0 + 8), X(g, c0 + 9));
    a[3] = pack_bf16(X(g + 8, c0 + 8), X(g + 8, c0 + 9));
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      uint32_t b[2];
      load_b(s.w1t, kk, j, g, t, b);
      mma16816(f.z1[j], a, b);
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int c = 8 * j + 2 * t;
    f.z1[j][0] += s.b1[c];
    f.z1[j][1] += s.b1[c + 1];
    f.z1[j][2] += s.b1[c];
    f.z1[j][3] += s.b1[c + 1];
  }
  // layer 2: A = gelu(Z1) in bf16 straight from the C fragments
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int q = 0; q < 4; ++q) f.z2[j][q] = 0.f;
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    uint32_t a[4];
    a[0] = pack_bf16(gelu(f.z1[2 * kk][0]), gelu(f.z1[2 * kk][1]));
    a[1] = pack_bf16(gelu(f.z1[2 * kk][2]), gelu(f.z1[2 * kk][3]));
    a[2] = pack_bf16(gelu(f.z1[2 * kk + 1][0]), gelu(f.z1[2 * kk + 1][1]));
    a[3] = pack_bf16(gelu(f.z1[2 * kk + 1][2]), gelu(f.z1[2 * kk + 1][3]));
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      uint32_t b[2];
      load_b2(s.w2t, kk, j, g, t, b);
      mma16816(f.z2[j], a, b);
    }
  }
  float p0 = 0.f, p1 = 0.f;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int c = 8 * j + 2 * t;
    f.z2[j][0] += s.b2[c];
    f.z2[j][1] += s.b2[c + 1];
    f.z2[j][2] += s.b2[c];
    f.z2[j][3] += s.b2[c + 1];
    p0 += gelu(f.z2[j][0]) * s.w3[c] + gelu(f.z2[j][1]) * s.w3[c + 1];
    p1 += gelu(f.z2[j][2]) * s.w3[c] + gelu(f.z2[j][3]) * s.w3[c + 1];
  }
  // the four lanes of a row group hold its 64 columns: reduce across t
  p0 += __shfl_xor_sync(0xffffffffu, p0, 1);
  p0 += __shfl_xor_sync(0xffffffffu, p0, 2);
  p1 += __shfl_xor_sync(0xffffffffu, p1, 1);
  p1 += __shfl_xor_sync(0xffffffffu, p1, 2);
  f.y0 = p0 + s.b3;
  f.y1 = p1 + s.b3;
}

__global__ void __launch_bounds__(128) k_mlp_infer(const float* __restrict__ params, const float* __restrict__ x,
                                                   uint64_t n, float* __restrict__ y) {
  __shared__ MlpSmem s;
  load_weights(s, params);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  for (uint64_t r0 = ((uint64_t)blockIdx.x * 4 + warp) * 16; r0 < n; r0 += (uint64_t)gridDim.x * 64) {
    Fwd f;
    forward_tile(s, x, n, r0, f);
    if (t == 0) {
      if (r0 + g < n) y[r0 + g] = f.y0;
      if (r0 + g + 8 < n) y[r0 + g + 8] = f.y1;
    }
  }
}

// One training step's gradient over rows [0, n): every warp runs the forward
// of a 16-row tile, then the backward:
//   dy = (y - t) / n,  dw3 = H2^T dy,  dZ2 = (dy w3^T) * gelu'(Z2),
//   dW2 = H1^T dZ2,    dH1 = dZ2 W2^T,  dZ1 = dH1 * gelu'(Z1),  dW1 = X^T dZ1
// The products with the batch as the contraction dimension (dW1, dW2) use
// the tensor cores on bf16 copies staged in shared memory; the partial
// gradients of each warp are added to `grad` (fp32 atomics).
struct TileSmem {
  __nv_bfloat16 xt[MK1][16 + 8];   // X^T of the tile   (k = feature, row = batch)
  __nv_bfloat16 h1t[MH][16 + 8];   // H1^T
  __nv_bfloat16 dz2[16][MH + 8];   // dZ2 (row = batch)
  __nv_bfloat16 dz1[16][MH + 8];   // dZ1
};

constexpr int GWARPS_MLP = 2;  // warps of the gradient kernel

__global__ void __launch_bounds__(32 * GWARPS_MLP) k_mlp_grad(const float* __restrict__ params,
                                                             const float* __restrict__ x, const float* __restrict__ tgt,
                                                             uint64_t n, float* __restrict__ grad,
                                                             float* __restrict__ loss) {
  __shared__ MlpSmem s;
  __shared__ TileSmem ts[GWARPS_MLP];
  load_weights(s, params);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  TileSmem& T = ts[warp];
  const float inv_n = 1.f / (float)n;
  for (uint64_t r0 = ((uint64_t)blockIdx.x * GWARPS_MLP + warp) * 16; r0 < n;
       r0 += (uint64_t)gridDim.x * 16 * GWARPS_MLP) {
    Fwd f;
    forward_tile(s, x, n, r0, f);
    const bool v0 = r0 + g < n, v1 = r0 + g + 8 < n;
    float dy0 = 0.f, dy1 = 0.f;
    if (t == 0) {
      if (v0) dy0 = (f.y0 - tgt[r0 + g]) * inv_n;
      if (v1) dy1 = (f.y1 - tgt[r0 + g + 8]) * inv_n;
      float l = 0.f;
      if (v0) l += 0.5f * (f.y0 - tgt[r0 + g]) * (f.y0 - tgt[r0 + g]);
      if (v1) l += 0.5f * (f.y1 - tgt[r0 + g + 8]) * (f.y1 - tgt[r0 + g + 8]);
      atomicAdd(loss, l * inv_n);
    }
    dy0 = __shfl_sync(0xffffffffu, dy0, lane & ~3);
    dy1 = __shfl_sync(0xffffffffu, dy1, lane & ~3);
    // b3, w3, dZ2 (rows g, g+8; columns 8j + 2t, +1)
    float db3 = dy0 + dy1;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = 8 * j + 2 * t;
      float dw3a = gelu(f.z2[j][0]) * dy0 + gelu(f.z2[j][2]) * dy1;
      float dw3b = gelu(f.z2[j][1]) * dy0 + gelu(f.z2[j][3]) * dy1;
      // sum over the 8 row groups (lanes with the same t)
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) {
        dw3a += __shfl_xor_sync(0xffffffffu, dw3a, o);
        dw3b += __shfl_xor_sync(0xffffffffu, dw3b, o);
      }
      if (g == 0) {
        atomicAdd(&grad[OFF_W3 + c], dw3a);
        atomicAdd(&grad[OFF_W3 + c + 1], dw3b);
      }
      const float d00 = dy0 * s.w3[c] * gelu_grad(f.z2[j][0]);
      const float d01 = dy0 * s.w3[c + 1] * gelu_grad(f.z2[j][1]);
      const float d10 = dy1 * s.w3[c] * gelu_grad(f.z2[j][2]);
      const float d11 = dy1 * s.w3[c + 1] * gelu_grad(f.z2[j][3]);
      f.z2[j][0] = d00;  // reuse: now dZ2
      f.z2[j][1] = d01;
      f.z2[j][2] = d10;
      f.z2[j][3] = d11;
      float bb0 = d00 + d10, bb1 = d01 + d11;
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) {
        bb0 += __shfl_xor_sync(0xffffffffu, bb0, o);
        bb1 += __shfl_xor_sync(0xffffffffu, bb1, o);
      }
      if (g == 0) {
        atomicAdd(&grad[OFF_B2 + c], bb0);
        atomicAdd(&grad[OFF_B2 + c + 1], bb1);
      }
      const __nv_bfloat162 p0 = __floats2bfloat162_rn(d00, d01), p1 = __floats2bfloat162_rn(d10, d11);
      *reinterpret_cast<__nv_bfloat162*>(&T.dz2[g][c]) = p0;
      *reinterpret_cast<__nv_bfloat162*>(&T.dz2[g + 8][c]) = p1;
      // H1^T for dW2
      T.h1t[c][g] = __float2bfloat16_rn(gelu(f.z1[j][0]));
      T.h1t[c + 1][g] = __float2bfloat16_rn(gelu(f.z1[j][1]));
      T.h1t[c][g + 8] = __float2bfloat16_rn(gelu(f.z1[j][2]));
      T.h1t[c + 1][g + 8] = __float2bfloat16_rn(gelu(f.z1[j][3]));
    }
    db3 += __shfl_xor_sync(0xffffffffu, db3, 4);
    db3 += __shfl_xor_sync(0xffffffffu, db3, 8);
    db3 += __shfl_xor_sync(0xffffffffu, db3, 16);
    if (lane == 0) atomicAdd(&grad[OFF_B3], db3);
    // X^T for dW1
    for (int i = lane; i < 16 * MK1; i += 32) {
      const int r = i / MK1, c = i % MK1;
      const uint64_t row = r0 + r;
      T.xt[c][r] = __float2bfloat16_rn((row < n && c < FKD_MLP_IN) ? x[row * FKD_MLP_IN + c] : 0.f);
    }
    __syncwarp();
    // dH1 = dZ2 W2^T (bf16 operands, fp32 accumulate over 64), then dZ1 = dH1 * gelu'(Z1)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = 8 * j + 2 * t;
      float h00 = 0.f, h01 = 0.f, h10 = 0.f, h11 = 0.f;
      for (int m = 0; m < MH; ++m) {
        const float a0 = __bfloat162float(T.dz2[g][m]), a1 = __bfloat162float(T.dz2[g + 8][m]);
        const float wa = __bfloat162float(s.w2t[m][c]), wb = __bfloat162float(s.w2t[m][c + 1]);
        h00 += a0 * wa;
        h01 += a0 * wb;
        h10 += a1 * wa;
        h11 += a1 * wb;
      }
      const float d00 = h00 * gelu_grad(f.z1[j][0]), d01 = h01 * gelu_grad(f.z1[j][1]);
      const float d10 = h10 * gelu_grad(f.z1[j][2]), d11 = h11 * gelu_grad(f.z1[j][3]);
      float bb0 = d00 + d10, bb1 = d01 + d11;
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) {
        bb0 += __shfl_xor_sync(0xffffffffu, bb0, o);
        bb1 += __shfl_xor_sync(0xffffffffu, bb1, o);
      }
      if (g == 0) {
        atomicAdd(&grad[OFF_B1 + c], bb0);
        atomicAdd(&grad[OFF_B1 + c + 1], bb1);
      }
      *reinterpret_cast<__nv_bfloat162*>(&T.dz1[g][c]) = __floats2bfloat162_rn(d00, d01);
      *reinterpret_cast<__nv_bfloat162*>(&T.dz1[g + 8][c]) = __floats2bfloat162_rn(d10, d11);
    }
    __syncwarp();
    // dW2 (64 x 64) = H1^T (64 x 16) dZ2 (16 x 16.. 64): 4 m-tiles x 8 n-tiles, one k-step
    // dW1 (48 x 64) = X^T  (48 x 16) dZ1 (16 x 64):     3 m-tiles x 8 n-tiles
#pragma unroll 1
    for (int which = 0; which < 2; ++which) {
      const int mt = which == 0 ? 4 : 3;
      for (int mi = 0; mi < mt; ++mi) {
        uint32_t a[4];
        const __nv_bfloat16* A0 = which == 0 ? &T.h1t[16 * mi + g][2 * t] : &T.xt[16 * mi + g][2 * t];
        const __nv_bfloat16* A1 = which == 0 ? &T.h1t[16 * mi + g + 8][2 * t] : &T.xt[16 * mi + g + 8][2 * t];
        a[0] = *reinterpret_cast<const uint32_t*>(A0);
        a[1] = *reinterpret_cast<const uint32_t*>(A1);
        a[2] = *reinterpret_cast<const uint32_t*>(A0 + 8);
        a[3] = *reinterpret_cast<const uint32_t*>(A1 + 8);
        for (int j = 0; j < 8; ++j) {
          // B(k = batch row, n = 8j + g): from dZ (row-major [row][col])
          const __nv_bfloat16(*D)[MH + 8] = which == 0 ? T.dz2 : T.dz1;
          const __nv_bfloat162 q0 = __halves2bfloat162(D[2 * t][8 * j + g], D[2 * t + 1][8 * j + g]);
          const __nv_bfloat162 q1 = __halves2bfloat162(D[2 * t + 8][8 * j + g], D[2 * t + 9][8 * j + g]);
          uint32_t b[2] = {*reinterpret_cast<const uint32_t*>(&q0), *reinterpret_cast<const uint32_t*>(&q1)};
          float d[4] = {0.f, 0.f, 0.f, 0.f};
          mma16816(d, a, b);
          const int row = 16 * mi + g, col = 8 * j + 2 * t;
          const int off = which == 0 ? OFF_W2 : OFF_W1;
          atomicAdd(&grad[off + row * MH + col], d[0]);
          atomicAdd(&grad[off + row * MH + col + 1], d[1]);
          atomicAdd(&grad[off + (row + 8) * MH + col], d[2]);
          atomicAdd(&grad[off + (row + 8) * MH + col + 1], d[3]);
        }
      }
    }
    __syncwarp();
  }
}

// Adam on the fp32 master weights; rows 40..47 of W1 stay zero.
__global__ void k_mlp_adam(float* __restrict__ p, const float* __restrict__ gr, float* __restrict__ m1,
                           float* __restrict__ m2, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NPARAM) return;
  if (i < OFF_B1 && i / MH >= FKD_MLP_IN) return;
  const float gi = gr[i];
  m1[i] = b1 * m1[i] + (1.f - b1) * gi;
  m2[i] = b2 * m2[i] + (1.f - b2) * gi * gi;
  p[i] -= lr * (m1[i] / c1) / (sqrtf(m2[i] / c2) + eps);
}

}  // namespace fkd

struct fkd_mlp_s {
  float* params = nullptr;  // device fp32 master
  float* grad = nullptr;
  float* m1 = nullptr;
  float* m2 = nullptr;
  float* dloss = nullptr;
  float* stage_x = nullptr;
  float* stage_t = nullptr;
  size_t stage_rows = 0;
  uint64_t steps = 0;
  ~fkd_mlp_s() {
    cudaFree(params);
    cudaFree(grad);
    cudaFree(m1);
    cudaFree(m2);
    cudaFree(dloss);
    cudaFree(stage_x);
    cudaFree(stage_t);
  }
};

namespace fkd {
const float* mlp_params(fkd_mlp m) { return m ? m->params : nullptr; }

cudaError_t mlp_infer(const float* params, const float* x, uint64_t n, float* y, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  const uint64_t tiles = (n + 63) / 64;
  const unsigned blocks = (unsigned)(tiles < 4096 ? tiles : 4096);
  k_mlp_infer<<<blocks, 128, 0, stream>>>(params, x, n, y);
  count_launches(1);
  return cudaGetLastError();
}
}  // namespace fkd

namespace {
#define MCUDA(call)                                                                                 \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess)                                                                          \
      return capi_fail(e_ == cudaErrorMemoryAllocation ? FKD_ERR_NOMEM : FKD_ERR_CUDA,              \
                       std::string(#call) + ": " + cudaGetErrorString(e_));                         \
  } while (0)

fkd_status stage(fkd_mlp m, const float* x, const float* t, uint64_t n, int mem, const float** dx, const float** dt) {
  if (mem == FKD_MEM_DEVICE) {
    *dx = x;
    *dt = t;
    return FKD_OK;
  }
  if (n > m->stage_rows) {
    cudaFree(m->stage_x);
    cudaFree(m->stage_t);
    m->stage_x = m->stage_t = nullptr;
    m->stage_rows = 0;
    MCUDA(cudaMalloc(&m->stage_x, n * FKD_MLP_IN * sizeof(float)));
    MCUDA(cudaMalloc(&m->stage_t, n * sizeof(float)));
    m->stage_rows = n;
  }
  MCUDA(cudaMemcpy(m->stage_x, x, n * FKD_MLP_IN * sizeof(float), cudaMemcpyHostToDevice));
  if (t) MCUDA(cudaMemcpy(m->stage_t, t, n * sizeof(float), cudaMemcpyHostToDevice));
  *dx = m->stage_x;
  *dt = m->stage_t;
  return FKD_OK;
}

fkd_status grad_pass(fkd_mlp m, const float* dx, const float* dt, uint64_t n) {
  MCUDA(cudaMemset(m->grad, 0, NPARAM * sizeof(float)));
  MCUDA(cudaMemset(m->dloss, 0, sizeof(float)));
  const uint64_t tiles = (n + 16 * GWARPS_MLP - 1) / (16 * GWARPS_MLP);
  const unsigned blocks = (unsigned)(tiles < 2048 ? tiles : 2048);
  if (n) {
    k_mlp_grad<<<blocks, 32 * GWARPS_MLP>>>(m->params, dx, dt, n, m->grad, m->dloss);
    count_launches(1);
  }
  MCUDA(cudaGetLastError());
  return FKD_OK;
}
}  // namespace

extern "C" {

fkd_status fkd_mlp_create(uint32_t seed, fkd_mlp* out) {
  if (!out) return capi_fail(FKD_ERR_ARG, "null output pointer");
  *out = nullptr;
  fkd_mlp m = new (std::nothrow) fkd_mlp_s();
  if (!m) return capi_fail(FKD_ERR_NOMEM, "host allocation failed");
  std::vector<float> p(NPARAM, 0.f);
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  for (int k = 0; k < FKD_MLP_IN; ++k)
    for (int j = 0; j < MH; ++j) p[OFF_W1 + k * MH + j] = nd(rng) * sqrtf(2.f / FKD_MLP_IN);
  for (int k = 0; k < MH; ++k)
    for (int j = 0; j < MH; ++j) p[OFF_W2 + k * MH + j] = nd(rng) * sqrtf(2.f / MH);
  for (int j = 0; j < MH; ++j) p[OFF_W3 + j] = nd(rng) * sqrtf(1.f / MH);
  p[OFF_B3] = 0.5f;
  cudaError_t e = cudaMalloc(&m->params, NPARAM * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->grad, NPARAM * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->m1, NPARAM * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->m2, NPARAM * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->dloss, sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(m->params, p.data(), NPARAM * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(m->m1, 0, NPARAM * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(m->m2, 0, NPARAM * sizeof(float));
  if (e != cudaSuccess) {
    delete m;
    return capi_fail(FKD_ERR_CUDA, std::string("fkd_mlp_create: ") + cudaGetErrorString(e));
  }
  *out = m;
  return FKD_OK;
}

fkd_status fkd_mlp_destroy(fkd_mlp m) {
  delete m;
  return FKD_OK;
}

uint64_t fkd_mlp_param_count(void) { return NPARAM; }

fkd_status fkd_mlp_get_params(fkd_mlp m, float* p) {
  if (!m || !p) return capi_fail(FKD_ERR_ARG, "null argument");
  MCUDA(cudaMemcpy(p, m->params, NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
  return FKD_OK;
}

fkd_status fkd_mlp_set_params(fkd_mlp m, const float* p) {
  if (!m || !p) return capi_fail(FKD_ERR_ARG, "null argument");
  MCUDA(cudaMemcpy(m->params, p, NPARAM * sizeof(float), cudaMemcpyHostToDevice));
  MCUDA(cudaMemset(m->m1, 0, NPARAM * sizeof(float)));
  MCUDA(cudaMemset(m->m2, 0, NPARAM * sizeof(float)));
  m->steps = 0;
  return FKD_OK;
}

fkd_status fkd_mlp_forward(fkd_mlp m, const float* x, uint64_t n, float* y, int mem) {
  if (!m || (n && (!x || !y))) return capi_fail(FKD_ERR_ARG, "null argument");
  const float *dx = nullptr, *dt = nullptr;
  fkd_status s = stage(m, x, nullptr, n, mem, &dx, &dt);
  if (s != FKD_OK) return s;
  float* dy = y;
  float* tmp = nullptr;
  if (mem == FKD_MEM_HOST) {
    MCUDA(cudaMalloc(&tmp, (n ? n : 1) * sizeof(float)));
    dy = tmp;
  }
  cudaError_t e = mlp_infer(m->params, dx, n, dy, 0);
  if (e == cudaSuccess && mem == FKD_MEM_HOST) e = cudaMemcpy(y, dy, n * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaFree(tmp);
  if (e != cudaSuccess) return capi_fail(FKD_ERR_CUDA, std::string("fkd_mlp_forward: ") + cudaGetErrorString(e));
  return FKD_OK;
}

fkd_status fkd_mlp_grad(fkd_mlp m, const float* x, const float* t, uint64_t n, float* grad, float* loss, int mem) {
  if (!m || !grad || !loss || (n && (!x || !t))) return capi_fail(FKD_ERR_ARG, "null argument");
  const float *dx = nullptr, *dt = nullptr;
  fkd_status s = stage(m, x, t, n, mem, &dx, &dt);
  if (s != FKD_OK) return s;
  if ((s = grad_pass(m, dx, dt, n)) != FKD_OK) return s;
  MCUDA(cudaMemcpy(grad, m->grad, NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
  MCUDA(cudaMemcpy(loss, m->dloss, sizeof(float), cudaMemcpyDeviceToHost));
  return FKD_OK;
}

fkd_status fkd_mlp_train(fkd_mlp m, const float* x, const float* t, uint64_t n, uint32_t epochs, uint32_t batch,
                         float lr, uint32_t seed, float* losses, int mem) {
  if (!m || (n && (!x || !t)) || batch == 0) return capi_fail(FKD_ERR_ARG, "bad argument");
  const float *dx = nullptr, *dt = nullptr;
  fkd_status s = stage(m, x, t, n, mem, &dx, &dt);
  if (s != FKD_OK) return s;
  // mini-batches are contiguous slices of a once-shuffled copy
  float *sx = nullptr, *st = nullptr;
  MCUDA(cudaMalloc(&sx, (n ? n : 1) * FKD_MLP_IN * sizeof(float)));
  MCUDA(cudaMalloc(&st, (n ? n : 1) * sizeof(float)));
  std::vector<uint32_t> perm(n);
  for (uint64_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
  std::mt19937 rng(seed);
  std::vector<float> hx(n * FKD_MLP_IN), ht(n);
  cudaMemcpy(hx.data(), dx, n * FKD_MLP_IN * sizeof(float), cudaMemcpyDeviceToHost);
  cudaMemcpy(ht.data(), dt, n * sizeof(float), cudaMemcpyDeviceToHost);
  std::vector<float> px(n * FKD_MLP_IN), pt(n);
  for (uint32_t ep = 0; ep < epochs; ++ep) {
    for (uint64_t i = n; i > 1; --i) std::swap(perm[i - 1], perm[rng() % i]);
    for (uint64_t i = 0; i < n; ++i) {
      memcpy(&px[i * FKD_MLP_IN], &hx[(uint64_t)perm[i] * FKD_MLP_IN], FKD_MLP_IN * sizeof(float));
      pt[i] = ht[perm[i]];
    }
    cudaMemcpy(sx, px.data(), n * FKD_MLP_IN * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(st, pt.data(), n * sizeof(float), cudaMemcpyHostToDevice);
    double eloss = 0.0;
    uint64_t nb = 0;
    for (uint64_t b0 = 0; b0 < n; b0 += batch, ++nb) {
      const uint64_t bn = (n - b0) < batch ? (n - b0) : batch;
      if ((s = grad_pass(m, sx + b0 * FKD_MLP_IN, st + b0, bn)) != FKD_OK) break;
      ++m->steps;
      const float b1 = 0.9f, b2 = 0.999f;
      const float c1 = 1.f - powf(b1, (float)m->steps), c2 = 1.f - powf(b2, (float)m->steps);
      k_mlp_adam<<<(NPARAM + 255) / 256, 256>>>(m->params, m->grad, m->m1, m->m2, lr, b1, b2, 1e-8f, c1, c2);
      count_launches(1);
      float l = 0.f;
      cudaMemcpy(&l, m->dloss, sizeof(float), cudaMemcpyDeviceToHost);
      eloss += l;
    }
    if (s != FKD_OK) break;
    if (losses) losses[ep] = (float)(eloss / (nb ? nb : 1));
  }
  cudaFree(sx);
  cudaFree(st);
  if (s != FKD_OK) return s;
  MCUDA(cudaGetLastError());
  MCUDA(cudaDeviceSynchronize());
  return FKD_OK;
}

}  // extern "C"
