// Pivot guard of the mixed-precision modes (B2P_FLAG_GUARD).
//
// In the tensor modes the update of block column k, D = L[:, 0:k0] L[k-block,
// 0:k0]^T, is accumulated on the tensor core from rounded operands, so every
// entry of D carries an error of about
//     delta(k) * sum_c L_jc^2  <=  delta(k) * A_jj,
//     delta(k) = 2^-16 (BF16x3: the operand split hi + lo keeps 16 bits)
//              | 2^-12 (FP8: E4M3 cross terms, panel_copy.cuh)
//              | 2^-10 (TF32: 11-bit operands, product error 2^-10)
//                + (MMAs accumulated so far) * 2^-23 (the accumulator does
//                  not round to nearest: one FP32 ulp per accumulation step),
// and the pivot d_j = A_jj - D_jj - (within the block) inherits it.  When
// d_j is not well above that error its sign and size are noise: this is how
// the mixed modes fail on matrices whose Schur complements sink to the level
// of a jitter term (Gaussian-process kernels) while the plain FP32 path
// factors them.
//
// The guard therefore audits every computed pivot against
//     d_j = L_jj^2  >  kGuardMargin * delta(k) * A_jj     (k = j / 64)
// (non-finite or non-positive pivots fail too); a matrix's first failing
// block column is its guard state.  The tensor-mode kernels record
// (L_jj, A_jj) for each pivot next to writing L_kk, L_jj as their own
// diagonal block produced it, and audit a matrix's record once they have
// finished it (guard_audit_matrix), outside the diagonal engine's column
// loop.  A matrix that fails is refactored from its first column in FP32 on
// the SIMT cores (potrf_rescue.cu: one launch after the path, which exits
// at once when no matrix failed).  Recomputing only from the failing column
// on is not enough: the mixed columns before it already carry a backward error of
// about delta * |A|, which can exceed the smallest eigenvalues of the
// remaining Schur complement (on the Gaussian-process kernels of order 2048
// an FP32 recompute from the failing column on still met a negative pivot,
// while a restart from column 0 gave the FP32 residual).  The reference's
// closest analogue is the accurate retry of its 256-order kernel, triggered
// when a pivot falls under 1e-2 of the input's diagonal
// (submission.py:866-868, 883-886, 1004-1031), which likewise refactors the
// whole matrix in FP32.
#pragma once

#include <stdint.h>

#include "launch.h"

namespace b2p {

constexpr float kGuardMargin = 2.0f;
constexpr int kGuardStageLd = 36;  // floats per staged row of the FP32 update
constexpr int kGuardStageFloats = 64 * kGuardStageLd;

// Pivot threshold (relative to A_jj) for block column k of a tensor mode;
// 0 for column 0, which no update precedes.
__device__ __forceinline__ float guard_tau(int mode, int k) {
  if (k == 0) return 0.0f;
  const int m = mode & B2P_MODE_MASK;
  // Operand rounding: 2^-10 (TF32), 2^-12 (FP8: E4M3 cross terms), 2^-16 (BF16x3).
  const float rep = m == B2P_MODE_TF32 ? 9.765625e-4f : m == B2P_MODE_FP8 ? 2.44140625e-4f : 1.52587890625e-5f;
  const float steps = m == B2P_MODE_BF16X3 ? 12.0f : 8.0f;  // MMAs per 64-wide chunk
  return kGuardMargin * (rep + steps * (float)k * 1.1920928955078125e-7f);  // 2^-23 per step
}

// The audit of one finished matrix: the first block column whose recorded
// pivot (L_jj, A_jj) fails L_jj^2 > guard_tau * A_jj (or is not finite), or
// -1.  piv is the matrix's record (n pairs; column 0 has no update and is
// not tested), written earlier by threads of this CTA or by earlier
// launches.  Collective over the NT threads that call it (barrier functor
// `bar`); smin is one int of shared memory, free until the call returns.
template <int NT, class Bar>
__device__ __forceinline__ int guard_audit_matrix(const float2* piv, int n, int mode, int* smin, int tid, Bar bar) {
  if (tid == 0) *smin = 0x7fffffff;
  bar();
  int first = 0x7fffffff;
  for (int j = 64 + tid; j < n; j += NT) {
    const float2 p = __ldcg(piv + j);
    if (!(p.x * p.x > guard_tau(mode, j >> 6) * p.y)) first = min(first, j >> 6);
  }
  if (first != 0x7fffffff) atomicMin(smin, first);
  bar();
  const int f = *smin;
  bar();
  return f == 0x7fffffff ? -1 : f;
}

// FP32 update of one row against 32 columns of block column k, computed on
// the SIMT cores: d[q] = sum_{j < k0} L[row][j] * L[k0 + c0 + q][j], each
// 32-wide piece of j summed on its own (fused multiply-adds in order of j)
// and added to d, so that no rounding chain runs over more than 32 + k0/32
// additions.  L is read through L2 only: other
// CTAs of the same launch write it.  Collective over the NT threads
// that call it (barrier functor `bar`): each passes its own row (-1 for
// none; d is then 0) and c0 (0 or 32, uniform within a warp); `stage` holds
// kGuardStageFloats floats of shared memory, free until the call returns.
template <int NT, class Bar>
__device__ __forceinline__ void guard_update_row(float (&d)[32], const float* __restrict__ L, int64_t n, int k0,
                                                 int64_t row, int c0, float* stage, int tid, Bar bar) {
#pragma unroll
  for (int q = 0; q < 32; ++q) d[q] = 0.0f;
  for (int j0 = 0; j0 < k0; j0 += 32) {
    bar();  // the previous chunk's stage has been read
    for (int e = tid; e < 64 * 8; e += NT) {
      const int c = e >> 3, q4 = e & 7;
      *reinterpret_cast<float4*>(stage + c * kGuardStageLd + 4 * q4) =
          __ldcg(reinterpret_cast<const float4*>(L + (size_t)(k0 + c) * n + j0 + 4 * q4));
    }
    bar();
    if (row >= 0) {
      float x[32];
      const float4* src = reinterpret_cast<const float4*>(L + (size_t)row * n + j0);
#pragma unroll
      for (int q4 = 0; q4 < 8; ++q4) {
        const float4 v = __ldcg(src + q4);
        x[4 * q4 + 0] = v.x;
        x[4 * q4 + 1] = v.y;
        x[4 * q4 + 2] = v.z;
        x[4 * q4 + 3] = v.w;
      }
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        const float4* b = reinterpret_cast<const float4*>(stage + (c0 + q) * kGuardStageLd);
        float s = 0.0f;
#pragma unroll
        for (int j4 = 0; j4 < 8; ++j4) {
          const float4 v = b[j4];
          s = fmaf(x[4 * j4 + 0], v.x, s);
          s = fmaf(x[4 * j4 + 1], v.y, s);
          s = fmaf(x[4 * j4 + 2], v.z, s);
          s = fmaf(x[4 * j4 + 3], v.w, s);
        }
        d[q] += s;
      }
    }
  }
  bar();  // the stage may be reused once every thread is done with it
}

// One thread's share of the FP32 recompute of P = A - D for its row `row`
// (-1: none) and columns k0 + c0 .. + 31 of block column k: D in FP32 from
// L (guard_update_row), P into dst[0..31] (shared memory).  Collective over
// NT threads.
template <int NT, class Bar>
__device__ __forceinline__ void guard_row_p(const float* __restrict__ L, const float* __restrict__ A, int64_t n,
                                            int k0, int64_t row, int c0, float* dst, float* stage, int tid,
                                            Bar bar) {
  float d[32];
  guard_update_row<NT>(d, L, n, k0, row, c0, stage, tid, bar);
  if (row >= 0) {
    const float4* src = reinterpret_cast<const float4*>(A + (size_t)row * n + k0 + c0);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float4 v = src[q];
      reinterpret_cast<float4*>(dst)[q] =
          make_float4(v.x - d[4 * q], v.y - d[4 * q + 1], v.z - d[4 * q + 2], v.w - d[4 * q + 3]);
    }
  }
}

}  // namespace b2p
