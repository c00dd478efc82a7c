// Factor and invert one 64x64 diagonal block with four warps.
//
// The block is split 2x2 into 32x32 sub-blocks; warp 0 runs the register
// factorization (warp_factor32) of L11 and L22, and the remaining work is
// spread so that independent pieces overlap:
//
//   1  warp 0          L11 = chol(A11)
//   2  warp 1          L21 = A21 L11^{-T}   (one row per lane)
//      warp 2          T11 = L11^{-1}       (one column per lane)
//   3  all             A22 -= L21 L21^T
//   4  warp 0          L22 = chol(A22)
//   5  warp 1          T22 = L22^{-1}
//      warps 2-3       W   = L21 T11
//   6  all             T21 = -T22 W
//
// Rows and columns at or beyond the block's true width are identity
// padding, so a short last block (w < 64) runs the same code.
#pragma once

#include "tile_engine.cuh"

namespace b2p {

constexpr int kD64Ld = 68;   // row stride of S and T (floats)
constexpr int kD64Threads = 128;

// Barrier used between the engine's phases: the whole CTA, or a named
// barrier over the first N threads (when other warps of the CTA run a
// different role and must not be waited for).
struct CtaBarrier {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
template <int NTHREADS>
struct NamedBarrier1 {
  __device__ __forceinline__ void operator()() const {
    asm volatile("bar.sync 1, %0;" ::"n"(NTHREADS) : "memory");
  }
};

struct Diag64Smem {
  float S[64 * kD64Ld];   // block: A in, L out (lower; upper zero)
  float T[64 * kD64Ld];   // inverse of L (lower; upper zero)
  float lt0[32 * kLtLd];  // L11^T
  float lt1[32 * kLtLd];  // L22^T
  float p21t[32 * kLtLd]; // L21^T
  float w21[32 * kLtLd];  // L21 T11
  float invd[64];
  float colbuf[64];
  int bad[2];
};

// Right-looking triangular solve of one row x (32 wide) against L^T:
// x <- x L^{-T}, with lt = L^T (row stride kLtLd) and invd = 1/diag(L).
__device__ __forceinline__ void row_solve32(float (&x)[32], const float* lt, const float* invd) {
#pragma unroll
  for (int m = 0; m < 32; ++m) {
    x[m] *= invd[m];
#pragma unroll
    for (int j4 = (m + 1) / 4; j4 < 8; ++j4) {
      const float4 c = reinterpret_cast<const float4*>(lt + m * kLtLd)[j4];
      const float cv[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int j = 4 * j4 + e;
        if (j > m) x[j] = fmaf(-x[m], cv[e], x[j]);
      }
    }
  }
}

// Column c of L^{-1} for a 32x32 lower L (lt = L^T, invd = 1/diag):
// forward substitution L y = e_c in right-looking order.
__device__ __forceinline__ void col_inverse32(float (&y)[32], int c, const float* lt, const float* invd) {
#pragma unroll
  for (int j = 0; j < 32; ++j) y[j] = (j == c) ? 1.0f : 0.0f;
#pragma unroll
  for (int m = 0; m < 32; ++m) {
    y[m] *= invd[m];
#pragma unroll
    for (int j4 = (m + 1) / 4; j4 < 8; ++j4) {
      const float4 cc = reinterpret_cast<const float4*>(lt + m * kLtLd)[j4];
      const float cv[4] = {cc.x, cc.y, cc.z, cc.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int j = 4 * j4 + e;
        if (j > m) y[j] = fmaf(-cv[e], y[m], y[j]);
      }
    }
  }
}

// Warp-level factorization of the 32x32 block at S[r0][r0]: writes L back
// (zeros above the diagonal), L^T to lt and 1/diag to invd.  Returns the
// first bad local pivot or -1.
__device__ __forceinline__ int diag64_factor_block(Diag64Smem& sm, int r0, float* lt, float* invd, int lane) {
  float x[32];
  const float* row = sm.S + (r0 + lane) * kD64Ld + r0;
#pragma unroll
  for (int c4 = 0; c4 < 8; ++c4) {
    const float4 v = reinterpret_cast<const float4*>(row)[c4];
    x[4 * c4 + 0] = v.x;
    x[4 * c4 + 1] = v.y;
    x[4 * c4 + 2] = v.z;
    x[4 * c4 + 3] = v.w;
  }
  float ip;
  const int bad = warp_factor32(x, lane, 32, sm.colbuf, ip);
  invd[lane] = ip;
  float* wrow = sm.S + (r0 + lane) * kD64Ld + r0;
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    const float v = (j <= lane) ? x[j] : 0.0f;
    wrow[j] = v;
    lt[j * kLtLd + lane] = v;
  }
  return bad;
}

// Full 64x64 factor + inverse.  The caller has filled sm.S (lower triangle
// and diagonal; identity padding beyond the true width) and synchronised.
// Returns the first bad pivot (0..63) or -1, uniform across the CTA.  Every
// thread of the CTA must call it; threads beyond the first kD64Threads only
// take part in the barriers.
template <class Bar = CtaBarrier>
__device__ __forceinline__ int diag64_factor_invert(Diag64Smem& sm, Bar bar = Bar()) {
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const bool active = tid < kD64Threads;
  // T starts at zero (its upper-right block stays zero).
  if (active)
    for (int e = tid; e < 64 * kD64Ld; e += kD64Threads) sm.T[e] = 0.0f;
  if (warp == 0) {
    const int b = diag64_factor_block(sm, 0, sm.lt0, sm.invd, lane);
    if (lane == 0) sm.bad[0] = b;
  }
  bar();
  if (warp == 1) {
    float x[32];
    const float* row = sm.S + (32 + lane) * kD64Ld;
#pragma unroll
    for (int c4 = 0; c4 < 8; ++c4) {
      const float4 v = reinterpret_cast<const float4*>(row)[c4];
      x[4 * c4 + 0] = v.x;
      x[4 * c4 + 1] = v.y;
      x[4 * c4 + 2] = v.z;
      x[4 * c4 + 3] = v.w;
    }
    row_solve32(x, sm.lt0, sm.invd);
    float* wrow = sm.S + (32 + lane) * kD64Ld;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      wrow[j] = x[j];
      sm.p21t[j * kLtLd + lane] = x[j];
    }
  } else if (warp == 2) {
    float y[32];
    col_inverse32(y, lane, sm.lt0, sm.invd);
#pragma unroll
    for (int j = 0; j < 32; ++j) sm.T[j * kD64Ld + lane] = y[j];
  }
  bar();
  if (active) {
    // A22 -= L21 L21^T (lower part): thread -> row i, 8 columns.
    const int i = tid >> 2, c0 = (tid & 3) * 8;
    float s[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) s[q] = 0.0f;
#pragma unroll 8
    for (int m = 0; m < 32; ++m) {
      const float a = sm.p21t[m * kLtLd + i];
      const float4 b0 = *reinterpret_cast<const float4*>(sm.p21t + m * kLtLd + c0);
      const float4 b1 = *reinterpret_cast<const float4*>(sm.p21t + m * kLtLd + c0 + 4);
      s[0] = fmaf(a, b0.x, s[0]);
      s[1] = fmaf(a, b0.y, s[1]);
      s[2] = fmaf(a, b0.z, s[2]);
      s[3] = fmaf(a, b0.w, s[3]);
      s[4] = fmaf(a, b1.x, s[4]);
      s[5] = fmaf(a, b1.y, s[5]);
      s[6] = fmaf(a, b1.z, s[6]);
      s[7] = fmaf(a, b1.w, s[7]);
    }
    float* row = sm.S + (32 + i) * kD64Ld + 32 + c0;
#pragma unroll
    for (int q = 0; q < 8; ++q)
      if (c0 + q <= i) row[q] -= s[q];
  }
  bar();
  if (warp == 0) {
    const int b = diag64_factor_block(sm, 32, sm.lt1, sm.invd + 32, lane);
    if (lane == 0) sm.bad[1] = b;
  }
  bar();
  if (warp == 1) {
    float y[32];
    col_inverse32(y, lane, sm.lt1, sm.invd + 32);
#pragma unroll
    for (int j = 0; j < 32; ++j) sm.T[(32 + j) * kD64Ld + 32 + lane] = y[j];
  } else if (warp == 2 || warp == 3) {
    // W = L21 T11: thread -> row i, 16 columns; T11 rows are in sm.T.
    const int t = tid - 64;
    const int i = t >> 1, c0 = (t & 1) * 16;
    float s[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) s[q] = 0.0f;
#pragma unroll 4
    for (int m = 0; m < 32; ++m) {
      const float a = sm.p21t[m * kLtLd + i];
      const float* trow = sm.T + m * kD64Ld + c0;
#pragma unroll
      for (int q4 = 0; q4 < 4; ++q4) {
        const float4 b = reinterpret_cast<const float4*>(trow)[q4];
        s[4 * q4 + 0] = fmaf(a, b.x, s[4 * q4 + 0]);
        s[4 * q4 + 1] = fmaf(a, b.y, s[4 * q4 + 1]);
        s[4 * q4 + 2] = fmaf(a, b.z, s[4 * q4 + 2]);
        s[4 * q4 + 3] = fmaf(a, b.w, s[4 * q4 + 3]);
      }
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) sm.w21[i * kLtLd + c0 + q] = s[q];
  }
  bar();
  if (active) {
    // T21 = -T22 W: thread -> row i, 8 columns.
    const int i = tid >> 2, c0 = (tid & 3) * 8;
    float s[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) s[q] = 0.0f;
    const float* trow = sm.T + (32 + i) * kD64Ld + 32;
    for (int m = 0; m <= i; ++m) {
      const float a = trow[m];
      const float4 b0 = *reinterpret_cast<const float4*>(sm.w21 + m * kLtLd + c0);
      const float4 b1 = *reinterpret_cast<const float4*>(sm.w21 + m * kLtLd + c0 + 4);
      s[0] = fmaf(a, b0.x, s[0]);
      s[1] = fmaf(a, b0.y, s[1]);
      s[2] = fmaf(a, b0.z, s[2]);
      s[3] = fmaf(a, b0.w, s[3]);
      s[4] = fmaf(a, b1.x, s[4]);
      s[5] = fmaf(a, b1.y, s[5]);
      s[6] = fmaf(a, b1.z, s[6]);
      s[7] = fmaf(a, b1.w, s[7]);
    }
    float* out = sm.T + (32 + i) * kD64Ld + c0;
#pragma unroll
    for (int q = 0; q < 8; ++q) out[q] = -s[q];
  }
  bar();
  const int b0 = sm.bad[0], b1 = sm.bad[1];
  return b0 >= 0 ? b0 : (b1 >= 0 ? 32 + b1 : -1);
}

// Inverse only: T = L^{-1} of the lower-triangular 64x64 block already in
// sm.S (diagonal and lower part valid; identity padding beyond the true
// width).  Uses lt0/lt1/p21t/w21 as scratch.  All threads call it.
template <class Bar = CtaBarrier>
__device__ __forceinline__ void diag64_invert_only(Diag64Smem& sm, Bar bar = Bar()) {
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const bool active = tid < kD64Threads;
  if (active) {
    for (int e = tid; e < 64 * kD64Ld; e += kD64Threads) sm.T[e] = 0.0f;
    // L11^T, L22^T, L21^T and 1/diag.
    for (int e = tid; e < 1024; e += kD64Threads) {
      const int r = e >> 5, c = e & 31;
      sm.lt0[c * kLtLd + r] = (c <= r) ? sm.S[r * kD64Ld + c] : 0.0f;
      sm.lt1[c * kLtLd + r] = (c <= r) ? sm.S[(32 + r) * kD64Ld + 32 + c] : 0.0f;
      sm.p21t[c * kLtLd + r] = sm.S[(32 + r) * kD64Ld + c];
    }
    if (tid < 64) sm.invd[tid] = 1.0f / sm.S[tid * kD64Ld + tid];
  }
  bar();
  if (warp == 0) {
    float y[32];
    col_inverse32(y, lane, sm.lt0, sm.invd);
#pragma unroll
    for (int j = 0; j < 32; ++j) sm.T[j * kD64Ld + lane] = y[j];
  } else if (warp == 1) {
    float y[32];
    col_inverse32(y, lane, sm.lt1, sm.invd + 32);
#pragma unroll
    for (int j = 0; j < 32; ++j) sm.T[(32 + j) * kD64Ld + 32 + lane] = y[j];
  }
  bar();
  if (active) {
    // W = L21 T11: thread -> row i, 8 columns.
    const int i = tid >> 2, c0 = (tid & 3) * 8;
    float sacc[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) sacc[q] = 0.0f;
    for (int m = 0; m < 32; ++m) {
      const float a = sm.p21t[m * kLtLd + i];
      const float* trow = sm.T + m * kD64Ld + c0;
#pragma unroll
      for (int q = 0; q < 8; ++q) sacc[q] = fmaf(a, trow[q], sacc[q]);
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) sm.w21[i * kLtLd + c0 + q] = sacc[q];
  }
  bar();
  if (active) {
    // T21 = -T22 W.
    const int i = tid >> 2, c0 = (tid & 3) * 8;
    float sacc[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) sacc[q] = 0.0f;
    const float* trow = sm.T + (32 + i) * kD64Ld + 32;
    for (int m = 0; m <= i; ++m) {
      const float a = trow[m];
#pragma unroll
      for (int q = 0; q < 8; ++q) sacc[q] = fmaf(a, sm.w21[m * kLtLd + c0 + q], sacc[q]);
    }
    float* out = sm.T + (32 + i) * kD64Ld + c0;
#pragma unroll
    for (int q = 0; q < 8; ++q) out[q] = -sacc[q];
  }
  bar();
}

}  // namespace b2p
