// Blocked right-looking factorization for n > 128 (plain FP32 SIMT form).
//
// The output buffer holds the working matrix.  One copy pass writes tril(A)
// into L (zeros above the diagonal), then for each 64-wide block column k0:
//
//   diag   one CTA per matrix: factor L[k0:k0+64, k0:k0+64] in shared memory
//          (smem_potrf), invert it (smem_trtri), write L_kk back and
//          T^T = inv(L_kk)^T to the workspace;
//   panel  L[i, k0:k0+64] <- L[i, k0:k0+64] * T^T for the rows below
//          (the TRSM as a GEMM against the explicit inverse);
//   trail  L[i, j] -= sum_m L[i, k0+m] L[j, k0+m] over the lower 64x64
//          tiles of the trailing matrix (the SYRK).
//
// The reference reaches the same blocked schedule through cuSOLVER / cuBLAS
// and Triton (submission.py:2375-2661 split32, 3217-3251 right-looking TF32,
// 5152-5196 e62 diagonal block + inverse panel multiply); here every step is
// a kernel of this library.
#include <algorithm>

#include "launch.h"
#include "tile_engine.cuh"

namespace b2p {

constexpr int kNB = 64;            // block column width
constexpr int kTile = 64;          // panel rows / trailing tile edge per CTA
constexpr int kBlkThreads = 256;
constexpr int kDiagLd = kNB + 4;   // 68
constexpr int kGemmLd = kTile + 4; // 68
constexpr int kMaxGridY = 65535;

// -------------------------------------------------------------------------
// tril copy: L[i][j] = (j <= i) ? A[i][j] : 0, info[b] = 0.  One row per CTA
// iteration, float4 columns when rows are 16-byte aligned.
__global__ void __launch_bounds__(256) copy_lower_kernel(const float* __restrict__ a,
                                                         float* __restrict__ l, int64_t batch,
                                                         int n, int32_t* __restrict__ info) {
  const int64_t rows = batch * (int64_t)n;
  const bool vec = (n & 3) == 0;
  for (int64_t g = blockIdx.x; g < rows; g += gridDim.x) {
    const int64_t b = g / n;
    const int r = (int)(g - b * n);
    const float* src = a + g * n;
    float* dst = l + g * n;
    if (vec) {
      const int n4 = n >> 2;
      for (int q = threadIdx.x; q < n4; q += blockDim.x) {
        const int c = q * 4;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c <= r) {
          v = __ldg(reinterpret_cast<const float4*>(src) + q);
          if (c + 1 > r) v.y = 0.0f;
          if (c + 2 > r) v.z = 0.0f;
          if (c + 3 > r) v.w = 0.0f;
        }
        reinterpret_cast<float4*>(dst)[q] = v;
      }
    } else {
      for (int c = threadIdx.x; c < n; c += blockDim.x) dst[c] = (c <= r) ? __ldg(src + c) : 0.0f;
    }
    if (info != nullptr && r == 0 && threadIdx.x == 0) info[b] = 0;
  }
}

// -------------------------------------------------------------------------
constexpr size_t diag_smem_floats() {
  return (size_t)2 * kNB * kDiagLd + tile_scratch_floats(kDiagLd) + 3 * 32 * 33;
}

__global__ void __launch_bounds__(kBlkThreads, 1)
    diag_kernel(float* __restrict__ l, int64_t batch, int n, int k0, float* __restrict__ tws,
                int32_t* __restrict__ info) {
  extern __shared__ __align__(16) float smem[];
  float* S = smem;
  float* Tm = S + kNB * kDiagLd;
  const TileScratch sc = make_scratch(Tm + kNB * kDiagLd, kDiagLd);
  float* work = smem + 2 * kNB * kDiagLd + tile_scratch_floats(kDiagLd);
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int w = min(kNB, n - k0);
  for (int64_t b = blockIdx.x; b < batch; b += gridDim.x) {
    float* base = l + b * (int64_t)n * n + (int64_t)k0 * n + k0;
    for (int r = warp; r < w; r += kBlkThreads / 32)
      for (int c = lane; c <= r; c += 32) S[r * kDiagLd + c] = base[(size_t)r * n + c];
    __syncthreads();
    const int bad = smem_potrf<kBlkThreads>(S, w, kDiagLd, sc);
    smem_trtri<kBlkThreads>(S, w, kDiagLd, Tm, kDiagLd, sc, work);
    __syncthreads();
    for (int r = warp; r < w; r += kBlkThreads / 32)
      for (int c = lane; c <= r; c += 32) base[(size_t)r * n + c] = S[r * kDiagLd + c];
    float* tb = tws + b * kNB * kNB;
    for (int e = tid; e < kNB * kNB; e += kBlkThreads) {
      const int m = e / kNB, c = e - (e / kNB) * kNB;
      tb[e] = (m < w && c < w) ? Tm[c * kDiagLd + m] : 0.0f;  // T^T[m][c] = T[c][m]
    }
    if (info != nullptr && tid == 0 && bad >= 0 && info[b] == 0) info[b] = k0 + bad + 1;
    __syncthreads();
  }
}

// -------------------------------------------------------------------------
// Load a kTile x kNB block of rows (row0.., cols col0..col0+kNB) of an n x n
// matrix into dst[m][i] (transposed, row stride kGemmLd).  Rows >= n load 0.
__device__ __forceinline__ void load_rows_t(const float* __restrict__ mat, int n, int row0,
                                            int col0, float* dst) {
  const int tid = threadIdx.x;
  if ((n & 3) == 0) {
    constexpr int kQ = kNB / 4;
    for (int e = tid; e < kTile * kQ; e += kBlkThreads) {
      const int i = e / kQ, q = e - (e / kQ) * kQ;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (row0 + i < n)
        v = reinterpret_cast<const float4*>(mat + (size_t)(row0 + i) * n + col0)[q];
      dst[(4 * q + 0) * kGemmLd + i] = v.x;
      dst[(4 * q + 1) * kGemmLd + i] = v.y;
      dst[(4 * q + 2) * kGemmLd + i] = v.z;
      dst[(4 * q + 3) * kGemmLd + i] = v.w;
    }
  } else {
    for (int e = tid; e < kTile * kNB; e += kBlkThreads) {
      const int i = e / kNB, m = e - (e / kNB) * kNB;
      dst[m * kGemmLd + i] = (row0 + i < n) ? mat[(size_t)(row0 + i) * n + col0 + m] : 0.0f;
    }
  }
}

// acc[r][c] = sum_m As[m][4ty+r] * Bs[m][4tx+c]
__device__ __forceinline__ void tile_mma_4x4(const float* As, const float* Bs, int ty, int tx,
                                             float (&acc)[4][4]) {
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = 0.0f;
#pragma unroll 8
  for (int m = 0; m < kNB; ++m) {
    const float4 av = *reinterpret_cast<const float4*>(As + m * kGemmLd + 4 * ty);
    const float4 bv = *reinterpret_cast<const float4*>(Bs + m * kGemmLd + 4 * tx);
    const float a4[4] = {av.x, av.y, av.z, av.w};
    const float b4[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[r][c] = fmaf(a4[r], b4[c], acc[r][c]);
  }
}

__global__ void __launch_bounds__(kBlkThreads)
    panel_kernel(float* __restrict__ l, int64_t batch, int n, int k0,
                 const float* __restrict__ tws) {
  __shared__ __align__(16) float Ps[kNB * kGemmLd];
  __shared__ __align__(16) float Ts[kNB * kGemmLd];
  const int tid = threadIdx.x;
  const int ty = tid >> 4, tx = tid & 15;
  const int row0 = k0 + kNB + blockIdx.x * kTile;
  for (int64_t b = blockIdx.y; b < batch; b += gridDim.y) {
    float* mat = l + b * (int64_t)n * n;
    load_rows_t(mat, n, row0, k0, Ps);
    const float* tb = tws + b * kNB * kNB;
    for (int e = tid; e < kNB * kNB / 4; e += kBlkThreads) {
      const int m = e / (kNB / 4), q = e - (e / (kNB / 4)) * (kNB / 4);
      *reinterpret_cast<float4*>(Ts + m * kGemmLd + 4 * q) =
          __ldg(reinterpret_cast<const float4*>(tb + m * kNB) + q);
    }
    __syncthreads();
    float acc[4][4];
    tile_mma_4x4(Ps, Ts, ty, tx, acc);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int i = row0 + 4 * ty + r;
      if (i < n) {
        float* dst = mat + (size_t)i * n + k0 + 4 * tx;
#pragma unroll
        for (int c = 0; c < 4; ++c) dst[c] = acc[r][c];
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kBlkThreads)
    trail_kernel(float* __restrict__ l, int64_t batch, int n, int k0) {
  __shared__ __align__(16) float As[kNB * kGemmLd];
  __shared__ __align__(16) float Bs[kNB * kGemmLd];
  const int tid = threadIdx.x;
  const int ty = tid >> 4, tx = tid & 15;
  const int q = blockIdx.x;
  int ti = (int)((sqrtf(8.0f * q + 1.0f) - 1.0f) * 0.5f);
  while ((ti + 1) * (ti + 2) / 2 <= q) ++ti;
  while (ti * (ti + 1) / 2 > q) --ti;
  const int tj = q - ti * (ti + 1) / 2;
  const int t0 = k0 + kNB;
  const int i0 = t0 + ti * kTile, j0 = t0 + tj * kTile;
  for (int64_t b = blockIdx.y; b < batch; b += gridDim.y) {
    float* mat = l + b * (int64_t)n * n;
    load_rows_t(mat, n, i0, k0, As);
    if (ti != tj) load_rows_t(mat, n, j0, k0, Bs);
    __syncthreads();
    float acc[4][4];
    tile_mma_4x4(As, ti != tj ? Bs : As, ty, tx, acc);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int i = i0 + 4 * ty + r;
      if (i < n) {
        float* dst = mat + (size_t)i * n + j0 + 4 * tx;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int j = j0 + 4 * tx + c;
          if (j <= i) dst[c] -= acc[r][c];
        }
      }
    }
    __syncthreads();
  }
}

// -------------------------------------------------------------------------
size_t blocked_workspace_bytes(int64_t batch, int64_t n, int mode) {
  (void)n;
  (void)mode;
  return (size_t)batch * kNB * kNB * sizeof(float);
}

int potrf_blocked(const float* a, float* l, int64_t batch, int n, int mode, void* ws,
                  size_t ws_bytes, int32_t* info, cudaStream_t s) {
  if ((mode & B2P_MODE_MASK) != B2P_MODE_FP32)
    return set_error(B2P_ERR_UNSUPPORTED, "mode %d not available for n=%d", mode, n);
  const size_t need = blocked_workspace_bytes(batch, n, mode);
  if (ws == nullptr || ws_bytes < need)
    return set_error(B2P_ERR_WORKSPACE, "workspace of %zu bytes required, %zu given", need, ws_bytes);
  float* tws = static_cast<float*>(ws);
  const int sms = device_sms();
  {
    const int64_t rows = batch * (int64_t)n;
    const int grid = (int)std::min<int64_t>(rows, (int64_t)sms * 32);
    {
      TraceScope ts(kKCopyLower, s);
      copy_lower_kernel<<<grid, 256, 0, s>>>(a, l, batch, n, info);
    }
    if (int st = check_launch("copy_lower_kernel")) return st;
  }
  const size_t dsmem = diag_smem_floats() * sizeof(float);
  if (int st = ensure_smem_attr((const void*)diag_kernel, dsmem, kSlotDiag)) return st;
  const int gy = (int)std::min<int64_t>(batch, kMaxGridY);
  for (int k0 = 0; k0 < n; k0 += kNB) {
    const int dgrid = (int)std::min<int64_t>(batch, (int64_t)sms * 16);
    {
      TraceScope ts(kKDiag, s);
      diag_kernel<<<dgrid, kBlkThreads, dsmem, s>>>(l, batch, n, k0, tws, info);
    }
    if (int st = check_launch("diag_kernel")) return st;
    const int R = n - k0 - kNB;
    if (R <= 0) break;
    const int T = (R + kTile - 1) / kTile;
    {
      TraceScope ts(kKPanel, s);
      panel_kernel<<<dim3(T, gy), kBlkThreads, 0, s>>>(l, batch, n, k0, tws);
    }
    if (int st = check_launch("panel_kernel")) return st;
    {
      TraceScope ts(kKTrail, s);
      trail_kernel<<<dim3(T * (T + 1) / 2, gy), kBlkThreads, 0, s>>>(l, batch, n, k0);
    }
    if (int st = check_launch("trail_kernel")) return st;
  }
  return B2P_OK;
}

}  // namespace b2p
