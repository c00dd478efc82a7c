// Register/shared-memory Cholesky building blocks shared by every path.
//
//  * warp_factor32: one warp factors a 32x32 block held one row per lane in
//    registers (right-looking, column by column).  The pivot column crosses
//    lanes through a double-buffered 32-float shared array, so one
//    __syncwarp per pivot orders it.
//  * smem_potrf:    a CTA factors an n x n (n <= 128) matrix resident in
//    shared memory, blocked by 32: warp 0 factors the diagonal block, every
//    thread solves one panel row against it, then 4x4 register tiles apply
//    the rank-32 trailing update to the lower triangle.
//
// The algorithm is the textbook right-looking Cholesky that LAPACK's potrf
// (called by the reference's ref_kernel, reference/reference.py:129-130, and
// its cuSOLVER routes, submission.py:4268) computes; pivots use a refined
// reciprocal square root instead of a divide.
#pragma once

#include "common.cuh"

namespace b2p {

// Transposed 32x32 copy of the current diagonal block's L, row stride 36.
constexpr int kLtLd = 36;

// Factor the 32x32 block x[] (row `lane`), columns >= w / rows >= w are
// identity padding.  On return x holds L (lower part valid, upper part is
// don't-care) and inv_pivot holds 1/L[lane][lane].  Returns the first local
// pivot index that was not positive, or -1.  All 32 lanes must call.
//
// Step k takes the pivot d = x[k] of lane k and, in the same round of
// shuffles, lane k+1's unscaled column-k value e; every lane then forms
// L[k+1][k] = e / sqrt(d) itself and updates its column k+1 at once, so the
// next pivot depends only on shuffles and registers.  The rest of the rank-1
// update (columns k+2..31) goes through a double-buffered shared-memory copy
// of column k and is deferred by one step: step k+1 applies it right after
// shuffling out its own pivot, in the shadow of that pivot's reciprocal
// square root.  The arithmetic is the same as the textbook right-looking
// update, value for value and in the same order.
__device__ __forceinline__ int warp_factor32(float (&x)[32], int lane, int w, float* colbuf,
                                             float& inv_pivot) {
  int bad = -1;
  inv_pivot = 1.0f;
  float lprev = 0.0f;  // this lane's L[lane][k-1]
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    if (k < w) {  // warp-uniform
      const float d = __shfl_sync(kFullMask, x[k], k);
      const float e = (k + 1 < 32) ? __shfl_sync(kFullMask, x[k], k + 1) : 0.0f;
      // Column k-1's update of columns k+1.. (column k had it by look-ahead).
      if (k >= 1 && k + 1 < 32) {
        const float* cb = colbuf + ((k - 1) & 1) * 32;
#pragma unroll
        for (int j4 = (k + 1) / 4; j4 < 8; ++j4) {
          const float4 c = reinterpret_cast<const float4*>(cb)[j4];
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
      if (lane == k) inv_pivot = y;
      x[k] = (lane == k) ? d * y : x[k] * y;
      if (k + 1 < 32) x[k + 1] = fmaf(-x[k], e * y, x[k + 1]);
      lprev = x[k];
      if (k + 2 < 32) {
        colbuf[(k & 1) * 32 + lane] = x[k];
        __syncwarp();
      }
    }
  }
  return bad;
}

// Scratch layout for smem_potrf (floats).
struct TileScratch {
  float* lt;      // [32][kLtLd]   transposed L of the current diagonal block
  float* invd;    // [128]         1/L[i][i]
  float* pt;      // [32][ldpt]    transposed panel below the diagonal block
  float* colbuf;  // [64]          warp_factor32 pivot column (double buffer)
  int* flag;      // [1]           first bad pivot (global index) or -1
  int ldpt;
};

__host__ __device__ constexpr int tile_scratch_floats(int ldpt) {
  return 32 * kLtLd + 128 + 32 * ldpt + 64 + 4;
}

__device__ __forceinline__ TileScratch make_scratch(float* base, int ldpt) {
  TileScratch s;
  s.lt = base;
  s.invd = s.lt + 32 * kLtLd;
  s.pt = s.invd + 128;
  s.colbuf = s.pt + 32 * ldpt;
  s.flag = reinterpret_cast<int*>(s.colbuf + 64);
  s.ldpt = ldpt;
  return s;
}

// Factor the n x n SPD matrix in shared memory S (row stride lds, a multiple
// of 4; lower triangle read, L written to the lower triangle, zeros written
// to the upper part of each diagonal block only).  n <= 128.  All NT threads
// call it; returns the first bad pivot (0-based) or -1, uniform across the CTA.
template <int NT>
__device__ int smem_potrf(float* S, int n, int lds, const TileScratch& sc) {
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  if (tid == 0) *sc.flag = -1;
  for (int kb = 0; kb < n; kb += 32) {
    const int w = min(32, n - kb);
    if (warp == 0) {
      float x[32];
      const float* row = S + (size_t)(kb + lane) * lds + kb;
#pragma unroll
      for (int c4 = 0; c4 < 8; ++c4) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (lane < w && 4 * c4 < w) v = reinterpret_cast<const float4*>(row)[c4];
        x[4 * c4 + 0] = v.x;
        x[4 * c4 + 1] = v.y;
        x[4 * c4 + 2] = v.z;
        x[4 * c4 + 3] = v.w;
      }
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        if (lane >= w || j >= w) x[j] = (lane == j) ? 1.0f : 0.0f;
      }
      float ip;
      const int bad = warp_factor32(x, lane, w, sc.colbuf, ip);
      if (lane == 0 && bad >= 0 && *sc.flag < 0) *sc.flag = kb + bad;
      sc.invd[kb + lane] = ip;
      float* srow = S + (size_t)(kb + lane) * lds + kb;
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const float v = (j <= lane) ? x[j] : 0.0f;
        if (lane < w && j < w) srow[j] = v;
        sc.lt[j * kLtLd + lane] = (lane < w) ? v : 0.0f;
      }
    }
    __syncthreads();
    const int r0 = kb + 32;
    const int R = n - r0;
    if (R > 0) {
      // Panel solve X * L_kk^T = P, one row per thread.
      for (int t = tid; t < R; t += NT) {
        float x[32];
        const float* row = S + (size_t)(r0 + t) * lds + kb;
#pragma unroll
        for (int c4 = 0; c4 < 8; ++c4) {
          float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
          if (4 * c4 < w) v = reinterpret_cast<const float4*>(row)[c4];
          x[4 * c4 + 0] = v.x;
          x[4 * c4 + 1] = v.y;
          x[4 * c4 + 2] = v.z;
          x[4 * c4 + 3] = v.w;
        }
#pragma unroll
        for (int j = 0; j < 32; ++j)
          if (j >= w) x[j] = 0.0f;
#pragma unroll
        for (int m = 0; m < 32; ++m) {
          x[m] *= sc.invd[kb + m];
#pragma unroll
          for (int j4 = (m + 1) / 4; j4 < 8; ++j4) {
            const float4 c = reinterpret_cast<const float4*>(sc.lt + m * kLtLd)[j4];
            const float cv[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const int j = 4 * j4 + e;
              if (j > m) x[j] = fmaf(-x[m], cv[e], x[j]);
            }
          }
        }
        float* wrow = S + (size_t)(r0 + t) * lds + kb;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          if (j < w) wrow[j] = x[j];
          sc.pt[j * sc.ldpt + t] = x[j];
        }
      }
      // Zero the transposed-panel padding so 4-wide tiles read finite values.
      for (int t = R + tid; t < ((R + 3) & ~3); t += NT) {
#pragma unroll
        for (int j = 0; j < 32; ++j) sc.pt[j * sc.ldpt + t] = 0.0f;
      }
      __syncthreads();
      // Trailing update S[i][j] -= sum_m P[i][m] P[j][m], i >= j >= r0.
      const int T4 = (R + 3) >> 2;
      const int ntiles = T4 * (T4 + 1) / 2;
      for (int q = tid; q < ntiles; q += NT) {
        int ti = (int)((sqrtf(8.0f * q + 1.0f) - 1.0f) * 0.5f);
        while ((ti + 1) * (ti + 2) / 2 <= q) ++ti;
        while (ti * (ti + 1) / 2 > q) --ti;
        const int tj = q - ti * (ti + 1) / 2;
        float acc[4][4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 4; ++c) acc[r][c] = 0.0f;
        for (int m = 0; m < w; ++m) {
          const float4 a = reinterpret_cast<const float4*>(sc.pt + m * sc.ldpt)[ti];
          const float4 b = reinterpret_cast<const float4*>(sc.pt + m * sc.ldpt)[tj];
          const float av[4] = {a.x, a.y, a.z, a.w};
          const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
          for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[r][c] = fmaf(av[r], bv[c], acc[r][c]);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int i = 4 * ti + r;
          if (i < R) {
            float* srow = S + (size_t)(r0 + i) * lds + r0;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              const int j = 4 * tj + c;
              if (j <= i) srow[j] -= acc[r][c];
            }
          }
        }
      }
      __syncthreads();
    }
  }
  __syncthreads();
  return *sc.flag;
}

}  // namespace b2p
