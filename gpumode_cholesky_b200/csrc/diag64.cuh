// Factor (and invert) one 64x64 diagonal block with four warps.
//
// Factorization (diag64_factor): the block is split 2x2 into 32x32 pieces
// and three warps run concurrently, handing columns to each other through
// shared memory:
//
//   warp 0   rows 0..31:                 pivots 0..31 (look-ahead warp factor)
//   warp 1   rows 32..63, columns < 32:  L21 = A21 L11^{-T}, column by column
//            behind warp 0
//   warp 2   rows 32..63, columns >= 32: A22 -= L21 L21^T column by column
//            behind warp 1, then pivots 32..63
//
// so that L21 and the A22 update hide behind the pivot chain.  A producer
// advances a progress counter (release store) after every group of
// kDiagGroup published columns; a consumer polls it with plain volatile loads
// once per group and fences after success.  Every poll is bounded.
//
// Inverse (diag64_factor_invert): after the factorization, T11 = L11^{-1}
// and T22 = L22^{-1} (one column per lane, warps 0 and 1), then
// W^T = T11^T L21^T and T21^T = -W^T T22^T (all four warps), written
// straight into the transposed layout the panel multiply reads.
//
// Rows and columns at or beyond the block's true width are identity
// padding, so a short last block (w < 64) runs the same code.
#pragma once

#include "tile_engine.cuh"

namespace b2p {

constexpr int kD64Ld = 68;   // row stride of S, T and the L^T view (floats)
constexpr int kD64Threads = 128;
constexpr int kDiagTimeout = -2;   // returned when a bounded wait gave up
constexpr int kDiagGroup = 4;      // columns per hand-off between warps
constexpr uint32_t kProgPolls = 1u << 22;

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

// The same over barrier 2 (a second group of warps that runs its own
// barrier 1 at the same time must not share the id).
template <int NTHREADS>
struct NamedBarrier2 {
  __device__ __forceinline__ void operator()() const {
    asm volatile("bar.sync 2, %0;" ::"n"(NTHREADS) : "memory");
  }
};

struct Diag64Smem {
  float S[64 * kD64Ld];   // block: A in, L out (lower part)
  float T[64 * kD64Ld];   // diag64_factor_invert: T^T, T = L^{-1} (T[c][j] = L^{-1}[j][c])
  // diag64_factor: L^T viewed as 64 x kD64Ld floats (diag64_lt).
  // diag64_invert_only: L11^T, L22^T, L21^T and L21 T11 (stride kLtLd).
  float lt0[32 * kLtLd];
  float lt1[32 * kLtLd];
  float p21t[32 * kLtLd];
  float w21[32 * kLtLd];
  float invd[64];         // 1 / diag(L)
  int bad[2];
  int prog[4];            // columns published by warps 0, 1, 2
  int err;                // a bounded wait gave up
};

__device__ __forceinline__ float* diag64_lt(Diag64Smem& sm) { return sm.lt0; }
__device__ __forceinline__ const float* diag64_lt(const Diag64Smem& sm) { return sm.lt0; }
static_assert(4 * 32 * kLtLd >= 64 * kD64Ld, "the L^T view must fit lt0..w21");

// ---- progress counters -------------------------------------------------------
__device__ __forceinline__ void prog_store(int* p, int v) {
  asm volatile("st.release.cta.shared.b32 [%0], %1;" ::"r"((uint32_t)__cvta_generic_to_shared(p)), "r"(v) : "memory");
}
// Called by all lanes at every column k of a consumer loop: at the first
// column of each group, wait (bounded) until the producer has published the
// whole group (its counter exceeds min(k + kDiagGroup - 1, last)).
__device__ __forceinline__ bool prog_wait_group(const int* p, int k, int last) {
  if (k % kDiagGroup != 0) return true;
  const int want = min(k + kDiagGroup - 1, last);
  const volatile int* vp = p;
  for (uint32_t i = 0; i < kProgPolls; ++i) {
    if (*vp > want) {
      __threadfence_block();
      return true;
    }
  }
  return false;
}
// Producer side: after column k (of `last`), publish the group if complete.
__device__ __forceinline__ void prog_publish(int* p, int k, int last, int lane) {
  if (k % kDiagGroup == kDiagGroup - 1 || k == last) {
    __syncwarp();
    if (lane == 0) prog_store(p, k + 1);
  }
}

// One warp factors the 32x32 block x (row `lane`) with the look-ahead update
// of warp_factor32, publishing column k into lt[k * kD64Ld + lane] (0 above
// the diagonal) and 1/L[k][k] into invd[k]; *prog counts published columns.
// Returns the first bad local pivot or -1.
//
// The rank-1 update of column k beyond column k+1 is deferred by one step:
// step k first shuffles pivot k out, then applies column k-1 (read back from
// its publication) to columns k+1.., which fills the latency of pivot k's
// reciprocal square root, and only then updates column k+1 with column k
// (the look-ahead) and publishes column k.  Every element receives the same
// fused multiply-adds in the same order as with the update done at once.
// On B200 this took the 64x64 factorization from 16.4k to 12.7k cycles.
__device__ __forceinline__ int warp_factor32_publish(float (&x)[32], int lane, float* lt, float* invd, int* prog) {
  int bad = -1;
  float lprev = 0.0f;  // this lane's L[lane][k-1]
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    const float d = __shfl_sync(kFullMask, x[k], k);
    const float e = (k + 1 < 32) ? __shfl_sync(kFullMask, x[k], k + 1) : 0.0f;
    // Column k-1's update of columns k+1.. (column k had it by look-ahead).
    if (k >= 1 && k + 1 < 32) {
      const float* col = lt + (k - 1) * kD64Ld;
#pragma unroll
      for (int j4 = (k + 1) / 4; j4 < 8; ++j4) {
        const float4 c = reinterpret_cast<const float4*>(col)[j4];
        const float cv[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int j = 4 * j4 + q;
          if (j > k) x[j] = fmaf(-lprev, cv[q], x[j]);
        }
      }
    }
    if (bad < 0 && pivot_bad(d)) bad = k;
    const float y = rsqrt_refined(d);
    const float l = (lane == k) ? d * y : x[k] * y;
    x[k] = l;
    if (k + 1 < 32) x[k + 1] = fmaf(-l, e * y, x[k + 1]);
    lt[k * kD64Ld + lane] = (lane >= k) ? l : 0.0f;
    if (lane == k) invd[k] = y;
    lprev = l;
    // The column is read back by every lane next step, and by warp 1 / 2.
    __syncwarp();
    prog_publish(prog, k, 31, lane);
  }
  return bad;
}

__device__ __forceinline__ void load_row32(float (&x)[32], const float* src) {
#pragma unroll
  for (int c4 = 0; c4 < 8; ++c4) {
    const float4 v = reinterpret_cast<const float4*>(src)[c4];
    x[4 * c4] = v.x, x[4 * c4 + 1] = v.y, x[4 * c4 + 2] = v.z, x[4 * c4 + 3] = v.w;
  }
}
// Row of 32 to shared memory, zeros right of column `diag` (all if diag >= 31).
__device__ __forceinline__ void store_row32(float* dst, const float (&x)[32], int diag) {
#pragma unroll
  for (int c4 = 0; c4 < 8; ++c4) {
    float v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = (4 * c4 + q <= diag) ? x[4 * c4 + q] : 0.0f;
    reinterpret_cast<float4*>(dst)[c4] = make_float4(v[0], v[1], v[2], v[3]);
  }
}

// Factor the block in sm.S (lower triangle and diagonal read; the caller has
// filled it and synchronised).  On return sm.S holds L in its lower triangle
// (the upper-right 32x32 block is left as it was), the L^T view holds
// Lt[m][j] = L[j][m] for j >= m (other entries unspecified) and sm.invd
// 1/diag(L).  Returns the first bad pivot, -1, or kDiagTimeout.  Every thread
// of the CTA calls it; threads beyond the first three warps only take part
// in the barriers.
template <class Bar = CtaBarrier>
__device__ __forceinline__ int diag64_factor(Diag64Smem& sm, Bar bar = Bar()) {
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  float* Lt = diag64_lt(sm);
  if (tid < 4) sm.prog[tid] = 0;
  if (tid == 0) sm.err = 0;
  bar();
  if (warp == 0) {
    float x[32];
    load_row32(x, sm.S + lane * kD64Ld);
    const int b = warp_factor32_publish(x, lane, Lt, sm.invd, &sm.prog[0]);
    if (lane == 0) sm.bad[0] = b;
    store_row32(sm.S + lane * kD64Ld, x, lane);
  } else if (warp == 1) {
    // L21 row 32 + lane.
    float x[32];
    load_row32(x, sm.S + (32 + lane) * kD64Ld);
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      if (ok && !prog_wait_group(&sm.prog[0], k, 31)) ok = false;
      const float l = x[k] * sm.invd[k];
      x[k] = l;
      Lt[k * kD64Ld + 32 + lane] = l;
      prog_publish(&sm.prog[1], k, 31, lane);
      if (k + 1 < 32) {
        const float* col = Lt + k * kD64Ld;
#pragma unroll
        for (int j4 = (k + 1) / 4; j4 < 8; ++j4) {
          const float4 c = reinterpret_cast<const float4*>(col)[j4];
          const float cv[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int j = 4 * j4 + q;
            if (j > k) x[j] = fmaf(-l, cv[q], x[j]);
          }
        }
      }
    }
    store_row32(sm.S + (32 + lane) * kD64Ld, x, 31);
    if (!ok) sm.err = 1;
  } else if (warp == 2) {
    // A22 row 32 + lane (columns 32..63): update, then factor.
    float x[32];
    load_row32(x, sm.S + (32 + lane) * kD64Ld + 32);
    bool ok = true;
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
      if (ok && !prog_wait_group(&sm.prog[1], k, 31)) ok = false;
      const float* col = Lt + k * kD64Ld + 32;
      const float l = col[lane];
#pragma unroll
      for (int j4 = 0; j4 < 8; ++j4) {
        const float4 c = reinterpret_cast<const float4*>(col)[j4];
        x[4 * j4 + 0] = fmaf(-l, c.x, x[4 * j4 + 0]);
        x[4 * j4 + 1] = fmaf(-l, c.y, x[4 * j4 + 1]);
        x[4 * j4 + 2] = fmaf(-l, c.z, x[4 * j4 + 2]);
        x[4 * j4 + 3] = fmaf(-l, c.w, x[4 * j4 + 3]);
      }
    }
    const int b = warp_factor32_publish(x, lane, Lt + 32 * kD64Ld + 32, sm.invd + 32, &sm.prog[2]);
    if (lane == 0) sm.bad[1] = b;
    store_row32(sm.S + (32 + lane) * kD64Ld + 32, x, lane);
    if (!ok) sm.err = 1;
  }
  bar();
  if (sm.err) return kDiagTimeout;
  const int b0 = sm.bad[0], b1 = sm.bad[1];
  return b0 >= 0 ? b0 : (b1 >= 0 ? 32 + b1 : -1);
}

// diag64_factor's result as every thread of the CTA can read it back once
// the factorization's last barrier has been passed by all of them.
__device__ __forceinline__ int diag64_status(const Diag64Smem& sm) {
  if (sm.err) return kDiagTimeout;
  return sm.bad[0] >= 0 ? sm.bad[0] : (sm.bad[1] >= 0 ? 32 + sm.bad[1] : -1);
}

// Column c of L^{-1} for a 32x32 lower L given as lt = L^T (row stride LD)
// and invd = 1/diag: forward substitution L y = e_c in right-looking order.
template <int LD>
__device__ __forceinline__ void col_inverse32(float (&y)[32], int c, const float* lt, const float* invd) {
#pragma unroll
  for (int j = 0; j < 32; ++j) y[j] = (j == c) ? 1.0f : 0.0f;
#pragma unroll
  for (int m = 0; m < 32; ++m) {
    y[m] *= invd[m];
#pragma unroll
    for (int j4 = (m + 1) / 4; j4 < 8; ++j4) {
      const float4 cc = reinterpret_cast<const float4*>(lt + m * LD)[j4];
      const float cv[4] = {cc.x, cc.y, cc.z, cc.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int j = 4 * j4 + e;
        if (j > m) y[j] = fmaf(-cv[e], y[m], y[j]);
      }
    }
  }
}

// diag64_factor, then T = L^{-1} stored transposed in sm.T:
// sm.T[c * kD64Ld + j] = T[j][c] (0 for j < c).  W^T is staged in the
// (zero) lower-left quarter of sm.T and cleared again.
template <class Bar = CtaBarrier>
__device__ __forceinline__ int diag64_factor_invert(Diag64Smem& sm, Bar bar = Bar()) {
  const int bad = diag64_factor(sm, bar);
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const bool active = tid < kD64Threads;
  const float* Lt = diag64_lt(sm);
  float* TT = sm.T;
  if (warp < 2) {
    // T11 (warp 0) / T22 (warp 1) column `lane` -> row of T^T.
    float y[32];
    col_inverse32<kD64Ld>(y, lane, Lt + warp * 32 * (kD64Ld + 1), sm.invd + 32 * warp);
    float* row = TT + (32 * warp + lane) * kD64Ld + 32 * warp;
#pragma unroll
    for (int c4 = 0; c4 < 8; ++c4)
      reinterpret_cast<float4*>(row)[c4] = make_float4(y[4 * c4], y[4 * c4 + 1], y[4 * c4 + 2], y[4 * c4 + 3]);
  }
  bar();
  const int c = tid >> 2, i0 = (tid & 3) * 8;
  if (active) {
    // W^T[c][i] = sum_m T11[m][c] L21[i][m]  (W = L21 T11), into TT[32 + c][i].
    float acc[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[q] = 0.0f;
#pragma unroll 8
    for (int m = 0; m < 32; ++m) {
      const float a = TT[c * kD64Ld + m];
      const float4 b0 = *reinterpret_cast<const float4*>(Lt + m * kD64Ld + 32 + i0);
      const float4 b1 = *reinterpret_cast<const float4*>(Lt + m * kD64Ld + 36 + i0);
      acc[0] = fmaf(a, b0.x, acc[0]);
      acc[1] = fmaf(a, b0.y, acc[1]);
      acc[2] = fmaf(a, b0.z, acc[2]);
      acc[3] = fmaf(a, b0.w, acc[3]);
      acc[4] = fmaf(a, b1.x, acc[4]);
      acc[5] = fmaf(a, b1.y, acc[5]);
      acc[6] = fmaf(a, b1.z, acc[6]);
      acc[7] = fmaf(a, b1.w, acc[7]);
    }
    float* w = TT + (32 + c) * kD64Ld + i0;
    reinterpret_cast<float4*>(w)[0] = make_float4(acc[0], acc[1], acc[2], acc[3]);
    reinterpret_cast<float4*>(w)[1] = make_float4(acc[4], acc[5], acc[6], acc[7]);
  }
  bar();
  if (active) {
    // T21^T[c][i] = -sum_p W^T[c][p] T22^T[p][i]  (T21 = -T22 W), into TT[c][32 + i].
    float acc[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[q] = 0.0f;
#pragma unroll 8
    for (int p = 0; p < 32; ++p) {
      const float a = TT[(32 + c) * kD64Ld + p];
      const float4 b0 = *reinterpret_cast<const float4*>(TT + (32 + p) * kD64Ld + 32 + i0);
      const float4 b1 = *reinterpret_cast<const float4*>(TT + (32 + p) * kD64Ld + 36 + i0);
      acc[0] = fmaf(a, b0.x, acc[0]);
      acc[1] = fmaf(a, b0.y, acc[1]);
      acc[2] = fmaf(a, b0.z, acc[2]);
      acc[3] = fmaf(a, b0.w, acc[3]);
      acc[4] = fmaf(a, b1.x, acc[4]);
      acc[5] = fmaf(a, b1.y, acc[5]);
      acc[6] = fmaf(a, b1.z, acc[6]);
      acc[7] = fmaf(a, b1.w, acc[7]);
    }
    float* o = TT + c * kD64Ld + 32 + i0;
    reinterpret_cast<float4*>(o)[0] = make_float4(-acc[0], -acc[1], -acc[2], -acc[3]);
    reinterpret_cast<float4*>(o)[1] = make_float4(-acc[4], -acc[5], -acc[6], -acc[7]);
  }
  bar();
  if (active) {
    float* z = TT + (32 + c) * kD64Ld + i0;
    reinterpret_cast<float4*>(z)[0] = make_float4(0.f, 0.f, 0.f, 0.f);
    reinterpret_cast<float4*>(z)[1] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  bar();
  return bad;
}

// Solve one panel row against the factored 64x64 block: x <- x L^{-T}
// (forward substitution, FP32, right-looking over the columns), with L^T as
// diag64_factor leaves it.  2080 FMAs per row; every shared-memory read is a
// warp-wide broadcast.
__device__ __forceinline__ void panel_solve64(float (&x)[64], const Diag64Smem& sm) {
  const float* Lt = diag64_lt(sm);
#pragma unroll
  for (int m = 0; m < 64; ++m) {
    x[m] *= sm.invd[m];
#pragma unroll
    for (int j4 = (m + 1) / 4; j4 < 16; ++j4) {
      const float4 c = reinterpret_cast<const float4*>(Lt + m * kD64Ld)[j4];
      const float cv[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = 4 * j4 + q;
        if (j > m) x[j] = fmaf(-x[m], cv[q], x[j]);
      }
    }
  }
}

// Inverse only: T = L^{-1} (row-major in sm.T) of the lower-triangular 64x64
// block already in sm.S (diagonal and lower part valid; identity padding
// beyond the true width).  Uses lt0/lt1/p21t/w21 as scratch.  All threads
// call it.
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
    col_inverse32<kLtLd>(y, lane, sm.lt0, sm.invd);
#pragma unroll
    for (int j = 0; j < 32; ++j) sm.T[j * kD64Ld + lane] = y[j];
  } else if (warp == 1) {
    float y[32];
    col_inverse32<kLtLd>(y, lane, sm.lt1, sm.invd + 32);
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
