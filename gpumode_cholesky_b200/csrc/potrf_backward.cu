// Cholesky adjoint: Abar = dLoss/dA from L and Lbar = dLoss/dL.
//
//   U  = L^{-1}                      block inverse: 64x64 diagonal blocks in
//                                    shared memory, then a recursive
//                                    U21 = -U22 (L21 U11) over block halves
//   P  = Phi(tril(L^T Lbar))         lower triangle, diagonal halved
//   Z  = P U                         lower x lower = lower
//   S  = U^T Z                       ( = L^{-T} P L^{-1} )
//   Abar = (S + S^T) / 2
//
// For n > 128 every product runs on the tensor cores through gemm_tc.cu
// (BF16x3 or TF32 operands, FP32 accumulation) with triangular K ranges.
// For n <= 128 one CTA per matrix does all of it in shared memory in FP32
// (bwd_small_kernel), which is both exact to FP32 and one launch instead of
// eight.  The upper part of Lbar is ignored: tril(L^T triu(Lbar, 1)) = 0.
//
// The reference has no backward; the oracle is torch.linalg.cholesky's
// autograd (same formula) and FP64 finite differences.
#include <algorithm>

#include "diag64.cuh"
#include "launch.h"
#include "tile_engine.cuh"

namespace b2p {


// Inverse of every 64x64 diagonal block of L into the same block of U.
__global__ void __launch_bounds__(kD64Threads) trtri_diag_kernel(const float* __restrict__ l, float* __restrict__ u,
                                                                 int64_t batch, int n) {
  extern __shared__ __align__(16) unsigned char raw[];
  Diag64Smem& sm = *reinterpret_cast<Diag64Smem*>(raw);
  const int tid = threadIdx.x;
  const int k0 = blockIdx.x * 64;
  const int w = min(64, n - k0);
  for (int64_t b = blockIdx.y; b < batch; b += gridDim.y) {
    const size_t off = (size_t)b * n * n + (size_t)k0 * n + k0;
    for (int e = tid; e < 4096; e += kD64Threads) {
      const int r = e >> 6, c = e & 63;
      float v = (r == c) ? 1.0f : 0.0f;
      if (r < w && c < w) v = (c <= r) ? l[off + (size_t)r * n + c] : 0.0f;
      sm.S[r * kD64Ld + c] = v;
    }
    __syncthreads();
    diag64_invert_only(sm);
    for (int e = tid; e < 4096; e += kD64Threads) {
      const int r = e >> 6, c = e & 63;
      if (r < w && c < w) u[off + (size_t)r * n + c] = sm.T[r * kD64Ld + c];
    }
    __syncthreads();
  }
}

// out = (s + s^T) / 2 by 32 x 32 tile pairs: tiles (bi, bj) and (bj, bi),
// bi >= bj, both read row-wise (coalesced) into shared memory, both written
// row-wise.  256 threads: 32 columns x 8 rows per pass.
constexpr int kSymThreads = 256;

__global__ void __launch_bounds__(kSymThreads) sym_kernel(const float* __restrict__ s, float* __restrict__ out,
                                                          int64_t batch, int n) {
  __shared__ float t1[32][33], t2[32][33];
  const int nt = (n + 31) / 32;
  const int64_t pairs = (int64_t)nt * (nt + 1) / 2;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int64_t item = blockIdx.x; item < batch * pairs; item += gridDim.x) {
    const int64_t b = item / pairs;
    const int q = (int)(item - b * pairs);
    int bi = (int)((sqrtf(8.0f * q + 1.0f) - 1.0f) * 0.5f);
    while ((bi + 1) * (bi + 2) / 2 <= q) ++bi;
    while (bi * (bi + 1) / 2 > q) --bi;
    const int bj = q - bi * (bi + 1) / 2;
    const float* sb = s + b * (int64_t)n * n;
    float* ob = out + b * (int64_t)n * n;
    for (int r = ty; r < 32; r += kSymThreads / 32) {
      const int i1 = 32 * bi + r, j1 = 32 * bj + tx;  // tile (bi, bj)
      const int i2 = 32 * bj + r, j2 = 32 * bi + tx;  // tile (bj, bi)
      t1[r][tx] = (i1 < n && j1 < n) ? sb[(size_t)i1 * n + j1] : 0.0f;
      t2[r][tx] = (i2 < n && j2 < n) ? sb[(size_t)i2 * n + j2] : 0.0f;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += kSymThreads / 32) {
      const int i1 = 32 * bi + r, j1 = 32 * bj + tx;
      if (i1 < n && j1 < n) ob[(size_t)i1 * n + j1] = 0.5f * (t1[r][tx] + t2[tx][r]);
      const int i2 = 32 * bj + r, j2 = 32 * bi + tx;
      if (bi != bj && i2 < n && j2 < n) ob[(size_t)i2 * n + j2] = 0.5f * (t2[r][tx] + t1[tx][r]);
    }
    __syncthreads();
  }
}

// ---- n <= 128: one CTA per matrix ------------------------------------------
constexpr int kBsThreads = 512;  // 16 warps: 8 x 4 register tiles over the 128 x 128 products
constexpr int kBsLd = 132;                      // row stride of the three 128x128 buffers
constexpr int kBsBuf = 128 * kBsLd;             // floats per buffer
constexpr int kBsWork = 64 * 64;                // trtri128's scratch W
constexpr size_t kBsSmemBytes = sizeof(float) * (size_t)(3 * kBsBuf + kBsWork + 128 + 4);

// acc[r][c] = sum_{k in [k0, k1)} X[k][8ti + r] * Y[k][4tj + c] (X, Y row-major
// in shared memory, row stride kBsLd): the X^T Y tile of this thread.
__device__ __forceinline__ void bs_tile(const float* X, const float* Y, int ti, int tj, int k0, int k1,
                                        float (&acc)[8][4]) {
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = 0.0f;
#pragma unroll 2
  for (int k = k0; k < k1; ++k) {
    const float4 x0 = *reinterpret_cast<const float4*>(X + k * kBsLd + 8 * ti);
    const float4 x1 = *reinterpret_cast<const float4*>(X + k * kBsLd + 8 * ti + 4);
    const float4 y0 = *reinterpret_cast<const float4*>(Y + k * kBsLd + 4 * tj);
    const float xv[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
    const float yv[4] = {y0.x, y0.y, y0.z, y0.w};
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[r][c] = fmaf(xv[r], yv[c], acc[r][c]);
  }
}

// C = A B (NEG: -(A B)) for 64 x 64 blocks, with register tiles over the
// 512 threads (2 rows x 4 columns each).  A and B are row-major in shared
// memory; the K range of output column group c4 (4 columns) and row pair is
// cut to where both operands can be non-zero: B lower triangular
// (B[k][j] = 0 for k < j) when B_LOWER, A lower triangular (A[i][k] = 0 for
// k > i) when A_LOWER.
template <bool A_LOWER, bool B_LOWER, bool NEG>
__device__ __forceinline__ void product64(const float* A, int lda, const float* B, int ldb, float* C, int ldc) {
  const int t = threadIdx.x;
  const int i0 = 2 * (t >> 4), j0 = 4 * (t & 15);  // rows i0, i0+1; columns j0..j0+3
  float acc[2][4] = {};
  const int k_lo = B_LOWER ? j0 : 0;
  const int k_hi = A_LOWER ? i0 + 2 : 64;
  for (int k = k_lo; k < k_hi; ++k) {
    const float a0 = A[i0 * lda + k], a1 = A[(i0 + 1) * lda + k];
    const float4 b = *reinterpret_cast<const float4*>(B + k * ldb + j0);
    acc[0][0] = fmaf(a0, b.x, acc[0][0]);
    acc[0][1] = fmaf(a0, b.y, acc[0][1]);
    acc[0][2] = fmaf(a0, b.z, acc[0][2]);
    acc[0][3] = fmaf(a0, b.w, acc[0][3]);
    acc[1][0] = fmaf(a1, b.x, acc[1][0]);
    acc[1][1] = fmaf(a1, b.y, acc[1][1]);
    acc[1][2] = fmaf(a1, b.z, acc[1][2]);
    acc[1][3] = fmaf(a1, b.w, acc[1][3]);
  }
  const float sg = NEG ? -1.0f : 1.0f;
#pragma unroll
  for (int r = 0; r < 2; ++r)
    *reinterpret_cast<float4*>(C + (i0 + r) * ldc + j0) =
        make_float4(sg * acc[r][0], sg * acc[r][1], sg * acc[r][2], sg * acc[r][3]);
}

// The same for two independent 32 x 32 products at once: block h = t / 256
// reads A + h a_off and B + h b_off and writes C + h c_off; each thread
// computes 1 row x 4 columns.
template <bool A_LOWER, bool B_LOWER, bool NEG>
__device__ __forceinline__ void product32x2(const float* A, int lda, const float* B, int ldb, float* C, int ldc,
                                                int a_off, int b_off, int c_off) {
  const int t = threadIdx.x;
  const int h = t >> 8, u = t & 255;
  const int i = u >> 3, j0 = 4 * (u & 7);
  const float* Ah = A + h * a_off;
  const float* Bh = B + h * b_off;
  float acc[4] = {};
  const int k_lo = B_LOWER ? j0 : 0;
  const int k_hi = A_LOWER ? i + 1 : 32;
  for (int k = k_lo; k < k_hi; ++k) {
    const float a = Ah[i * lda + k];
    const float4 b = *reinterpret_cast<const float4*>(Bh + k * ldb + j0);
    acc[0] = fmaf(a, b.x, acc[0]);
    acc[1] = fmaf(a, b.y, acc[1]);
    acc[2] = fmaf(a, b.z, acc[2]);
    acc[3] = fmaf(a, b.w, acc[3]);
  }
  const float sg = NEG ? -1.0f : 1.0f;
  *reinterpret_cast<float4*>(C + h * c_off + i * ldc + j0) = make_float4(sg * acc[0], sg * acc[1], sg * acc[2], sg * acc[3]);
}

// U = L^{-1} of the 128 x 128 lower-triangular L in shared memory (row stride
// ld), into U (row stride ld, zero above the diagonal), by block recursion:
//   32 x 32 diagonal blocks by forward substitution (warp b, lane = column);
//   U_10 = -U_11 (L_10 U_00) inside each 64-block (both 64-blocks at once);
//   U_21 = -U_22 (L_21 U_11) for the 64-blocks.
// invd holds 1 / L_ii; W is scratch of 64 x kBsWLd floats.  All 512 threads.
constexpr int kBsWLd = 64;
static_assert(64 * kBsWLd <= kBsWork, "trtri128 scratch fits the work area");
__device__ void trtri128(const float* L, float* U, int ld, const float* invd, float* W) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = tid; e < 128 * ld; e += kBsThreads) U[e] = 0.0f;
  __syncthreads();
  if (warp < 4) {
    const int kb = 32 * warp, c = lane;
    float x[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) x[j] = (j == c) ? 1.0f : 0.0f;
#pragma unroll
    for (int m = 0; m < 32; ++m) {
      x[m] *= invd[kb + m];
#pragma unroll
      for (int j = m + 1; j < 32; ++j) x[j] = fmaf(-L[(kb + j) * ld + kb + m], x[m], x[j]);
    }
#pragma unroll
    for (int j = 0; j < 32; ++j)
      if (j >= c) U[(kb + j) * ld + kb + c] = x[j];
  }
  __syncthreads();
  // Inside each 64-block h: W_h = L_10 U_00 (W rows 32 h ..), then U_10 = -U_11 W_h.
  // Block h covers rows / columns 64 h .. 64 h + 63; its L_10 starts at
  // (64 h + 32, 64 h), U_00 at (64 h, 64 h), U_11 at (64 h + 32, 64 h + 32).
  product32x2<false, true, false>(L + 32 * ld, ld, U, ld, W, kBsWLd, 64 * (ld + 1), 64 * (ld + 1), 32 * kBsWLd);
  __syncthreads();
  product32x2<true, false, true>(U + 32 * ld + 32, ld, W, kBsWLd, U + 32 * ld, ld, 64 * (ld + 1), 32 * kBsWLd,
                                 64 * (ld + 1));
  __syncthreads();
  // W = L_21 U_11 (the first 64-block's inverse), then U_21 = -U_22 W.
  product64<false, true, false>(L + 64 * ld, ld, U, ld, W, kBsWLd);
  __syncthreads();
  product64<true, false, true>(U + 64 * ld + 64, ld, W, kBsWLd, U + 64 * ld, ld);
  __syncthreads();
}

__global__ void __launch_bounds__(kBsThreads, 1)
    bwd_small_kernel(const float* __restrict__ l, const float* __restrict__ lbar, float* __restrict__ abar,
                     int64_t batch, int n) {
  extern __shared__ __align__(16) float bsm[];
  float* bA = bsm;               // L, later S
  float* bB = bsm + kBsBuf;      // Lbar, later P^T, later Z
  float* bC = bsm + 2 * kBsBuf;  // U = L^{-1}
  float* work = bsm + 3 * kBsBuf;
  TileScratch sc{};
  sc.invd = work + kBsWork;
  const int tid = threadIdx.x;
  const int ti = tid >> 5, tj = tid & 31;  // rows 8ti.., columns 4tj..
  float acc[8][4];
  for (int64_t b = blockIdx.x; b < batch; b += gridDim.x) {
    const float* L = l + (size_t)b * n * n;
    const float* G = lbar + (size_t)b * n * n;
    // L (lower, identity beyond n) and Lbar (lower, zero beyond n).
    for (int e = tid; e < 128 * 128; e += kBsThreads) {
      const int i = e >> 7, j = e & 127;
      const bool in = i < n && j < n && j <= i;
      bA[i * kBsLd + j] = in ? L[(size_t)i * n + j] : (i == j ? 1.0f : 0.0f);
      bB[i * kBsLd + j] = in ? G[(size_t)i * n + j] : 0.0f;
    }
    __syncthreads();
    if (tid < 128) sc.invd[tid] = 1.0f / bA[tid * kBsLd + tid];
    // P = Phi(L^T Lbar) (tiles reaching the lower triangle; k >= max(i, j)),
    // kept in registers.
    const bool lower = 4 * tj <= 8 * ti + 7;
    const int kmax = 8 * ti > 4 * tj ? 8 * ti : 4 * tj;  // smallest max(i, j) of the tile
    if (lower) bs_tile(bA, bB, ti, tj, kmax, 128, acc);
    __syncthreads();
    // P^T into bB: per column j of the tile, its 8 rows as two float4.
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int j = 4 * tj + c;
      float v[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int i = 8 * ti + r;
        v[r] = !lower || j > i ? 0.0f : (j == i ? 0.5f * acc[r][c] : acc[r][c]);
      }
      float4* dst = reinterpret_cast<float4*>(bB + j * kBsLd + 8 * ti);
      dst[0] = make_float4(v[0], v[1], v[2], v[3]);
      dst[1] = make_float4(v[4], v[5], v[6], v[7]);
    }
    // U = L^{-1} into bC.
    trtri128(bA, bC, kBsLd, sc.invd, work);
    // Z = P U: Z[i][j] = sum_k P^T[k][i] U[k][j], k in [j, i] (lower tiles).
    if (lower) bs_tile(bB, bC, ti, tj, 4 * tj, 8 * ti + 8, acc);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int i = 8 * ti + r, j = 4 * tj;
      *reinterpret_cast<float4*>(bB + i * kBsLd + j) =
          make_float4((lower && j <= i) ? acc[r][0] : 0.0f, (lower && j + 1 <= i) ? acc[r][1] : 0.0f,
                      (lower && j + 2 <= i) ? acc[r][2] : 0.0f, (lower && j + 3 <= i) ? acc[r][3] : 0.0f);
    }
    __syncthreads();
    // S = U^T Z: S[i][j] = sum_k U[k][i] Z[k][j], k >= max(i, j); into bA.
    bs_tile(bC, bB, ti, tj, kmax, 128, acc);
#pragma unroll
    for (int r = 0; r < 8; ++r)
      *reinterpret_cast<float4*>(bA + (8 * ti + r) * kBsLd + 4 * tj) =
          make_float4(acc[r][0], acc[r][1], acc[r][2], acc[r][3]);
    __syncthreads();
    float* Ab = abar + (size_t)b * n * n;
    for (int i = tid >> 5; i < n; i += kBsThreads / 32)
      for (int j = tid & 31; j < n; j += 32) Ab[(size_t)i * n + j] = 0.5f * (bA[i * kBsLd + j] + bA[j * kBsLd + i]);
    __syncthreads();
  }
}

// Packed-operand scratch of the current call (see GemmArgs::pack_x).
struct PackScratch {
  uint8_t* x = nullptr;
  uint8_t* y = nullptr;
};

static GemmArgs gemm_args(int64_t batch, int n, const PackScratch& ps) {
  GemmArgs g{};
  g.pack_x = ps.x;
  g.pack_y = ps.y;
  g.sx = g.sy = g.sc = (int64_t)n * n;
  g.ldx = g.ldy = g.ldc = n;
  g.alpha = 1.0f;
  g.beta = 0.0f;
  g.batch = batch;
  g.c_in = nullptr;
  return g;
}

// Packing pays once both sides of a product are this large.
constexpr int kPackMin = 256;

// The off-diagonal block of `pairs` block pairs ([lo, mid), [mid, hi), then
// the same shape every 2 (mid - lo) blocks down the diagonal), each of whose
// diagonal halves is already inverted: U21 = -U22 (L21 U11); tmp holds
// L21 U11.  One batched product per step for all pairs.
static int trtri_combine(const float* l, float* u, float* tmp, int64_t batch, int n, int lo, int mid, int hi,
                         int64_t pairs, int mode, int32_t* err, const PackScratch& ps, cudaStream_t s) {
  const int r0 = lo * 64, r1 = mid * 64, r2 = std::min(hi * 64, n);
  const size_t o21 = (size_t)r1 * n + r0, o11 = (size_t)r0 * n + r0, o22 = (size_t)r1 * n + r1;
  const int64_t step = 2LL * (r1 - r0) * (n + 1);  // next pair along the diagonal
  const PackScratch none;
  const PackScratch& pk = (r2 - r1 >= kPackMin && r1 - r0 >= kPackMin) ? ps : none;
  // tmp21 = L21 * U11   (U11 lower: op2(Y)[k][c] nonzero for k >= c)
  GemmArgs g = gemm_args(batch, n, pk);
  g.batch2 = pairs;
  g.sx2 = g.sy2 = g.sc2 = step;
  g.x = l + o21;
  g.y = u + o11;
  g.c = tmp + o21;
  g.m = r2 - r1;
  g.n = r1 - r0;
  g.k = r1 - r0;
  g.y_tri = 1;
  if (int st = launch_gemm_tc(g, mode, err, s)) return st;
  // U21 = -U22 * tmp21   (U22 lower: op1(X)[m][k] nonzero for k <= m)
  g = gemm_args(batch, n, pk);
  g.batch2 = pairs;
  g.sx2 = g.sy2 = g.sc2 = step;
  g.x = u + o22;
  g.y = tmp + o21;
  g.c = u + o21;
  g.m = r2 - r1;
  g.n = r1 - r0;
  g.k = r2 - r1;
  g.x_tri = 1;
  g.alpha = -1.0f;
  return launch_gemm_tc(g, mode, err, s);
}

// U[lo:lo+len, lo:lo+len] for a power-of-two number of 64-wide blocks, bottom
// up: at width h every aligned pair of h-block inverses merges into one of
// 2h blocks, all pairs of a level in one batched product.  A pair that holds
// the last (partial) block of the matrix has its own product.
static int trtri_pow2(const float* l, float* u, float* tmp, int64_t batch, int n, int nblk, int lo, int len, int mode,
                      int32_t* err, const PackScratch& ps, cudaStream_t s) {
  for (int h = 1; 2 * h <= len; h *= 2) {
    const int pairs = len / (2 * h);
    const bool partial = (lo + len == nblk) && (n % 64) != 0;
    const int full = partial ? pairs - 1 : pairs;
    if (full > 0) {
      if (int st = trtri_combine(l, u, tmp, batch, n, lo, lo + h, lo + 2 * h, full, mode, err, ps, s)) return st;
    }
    if (partial) {
      const int j0 = lo + (pairs - 1) * 2 * h;
      if (int st = trtri_combine(l, u, tmp, batch, n, j0, j0 + h, j0 + 2 * h, 1, mode, err, ps, s)) return st;
    }
  }
  return B2P_OK;
}

// U[lo:hi, lo:hi] = inverse of L[lo:hi, lo:hi] (block indices, 64 wide);
// diagonal blocks are already inverted.  Splits off the largest power-of-two
// prefix (batched levels), recurses on the rest, then merges the two.
static int trtri_range(const float* l, float* u, float* tmp, int64_t batch, int n, int nblk, int lo, int hi, int mode,
                       int32_t* err, const PackScratch& ps, cudaStream_t s) {
  const int len = hi - lo;
  if (len <= 1) return B2P_OK;
  if ((len & (len - 1)) == 0) return trtri_pow2(l, u, tmp, batch, n, nblk, lo, len, mode, err, ps, s);
  int p = 1;
  while (2 * p < len) p *= 2;
  if (int st = trtri_pow2(l, u, tmp, batch, n, nblk, lo, p, mode, err, ps, s)) return st;
  if (int st = trtri_range(l, u, tmp, batch, n, nblk, lo + p, hi, mode, err, ps, s)) return st;
  return trtri_combine(l, u, tmp, batch, n, lo, lo + p, hi, 1, mode, err, ps, s);
}

// U and one temporary (batch x n x n FP32 each), then the two packed operands
// of the tensor-core products (1024-byte aligned).
size_t backward_workspace_bytes(int64_t batch, int64_t n) {
  if (n <= 128) return 0;
  const size_t pack = (gemm_pack_bytes(batch, (int)n, (int)n) + 1023) & ~(size_t)1023;
  return (size_t)2 * batch * n * n * sizeof(float) + 2 * pack + 1024;
}

int potrf_backward(const float* l, const float* lbar, float* abar, int64_t batch, int n, int mode, void* ws,
                   size_t ws_bytes, cudaStream_t s) {
  const int m = mode & B2P_MODE_MASK;
  if (m != B2P_MODE_TF32 && m != B2P_MODE_BF16X3)
    return set_error(B2P_ERR_UNSUPPORTED, "backward runs its products in tf32 or bf16x3 (mode 0x%x)", mode);
  if (n <= 128) {
    // One CTA per matrix, everything in shared memory, FP32 in every mode.
    if (int st = ensure_smem_attr((const void*)bwd_small_kernel, kBsSmemBytes, kSlotBwdSmall)) return st;
    TraceScope ts(kKBwdSym, s);
    const int grid = (int)std::min<int64_t>(batch, (int64_t)device_sms());
    bwd_small_kernel<<<grid, kBsThreads, kBsSmemBytes, s>>>(l, lbar, abar, batch, n);
    return check_launch("bwd_small_kernel");
  }
  const size_t need = backward_workspace_bytes(batch, n);
  if (ws == nullptr || ws_bytes < need)
    return set_error(B2P_ERR_WORKSPACE, "workspace of %zu bytes required, %zu given", need, ws_bytes);
  const size_t mat = (size_t)batch * n * n;
  float* u = static_cast<float*>(ws);
  float* w1 = u + mat;
  PackScratch ps;
  {
    const size_t pack = (gemm_pack_bytes(batch, n, n) + 1023) & ~(size_t)1023;
    uint8_t* p0 = reinterpret_cast<uint8_t*>(((reinterpret_cast<uintptr_t>(w1 + mat)) + 1023) & ~(uintptr_t)1023);
    ps.x = p0;
    ps.y = p0 + pack;
  }
  int32_t* err = nullptr;
  // U = L^{-1}: zero (upper part stays zero), diagonal blocks, recursion.
  if (cudaMemsetAsync(u, 0, mat * sizeof(float), s) != cudaSuccess) return check_launch("cudaMemsetAsync");
  const int nblk = (n + 63) / 64;
  if (int st = ensure_smem_attr((const void*)trtri_diag_kernel, sizeof(Diag64Smem), kSlotBwd2)) return st;
  {
    TraceScope ts(kKBwdTrsm, s);
    trtri_diag_kernel<<<dim3(nblk, (unsigned)std::min<int64_t>(batch, 65535)), kD64Threads, sizeof(Diag64Smem), s>>>(
        l, u, batch, n);
  }
  if (int st = check_launch("trtri_diag_kernel")) return st;
  if (int st = trtri_range(l, u, w1, batch, n, nblk, 0, nblk, mode, err, ps, s)) return st;
  const PackScratch none;
  const PackScratch& pbig = n >= kPackMin ? ps : none;
  // P = Phi(tril(L^T Lbar)) into w1 (upper part zero).
  if (cudaMemsetAsync(w1, 0, mat * sizeof(float), s) != cudaSuccess) return check_launch("cudaMemsetAsync");
  GemmArgs g = gemm_args(batch, n, pbig);
  g.x = l;
  g.y = lbar;
  g.c = w1;
  g.m = g.n = g.k = n;
  g.trans_x = 1;  // op1 = L^T: upper (k >= m)
  g.x_tri = 2;
  g.y_tri = 1;    // Lbar lower: k >= column
  g.lower_out = 1;
  g.phi = 1;
  if (int st = launch_gemm_tc(g, mode, err, s)) return st;
  // Z = P U into abar (lower; upper zero).
  if (cudaMemsetAsync(abar, 0, mat * sizeof(float), s) != cudaSuccess) return check_launch("cudaMemsetAsync");
  g = gemm_args(batch, n, pbig);
  g.x = w1;
  g.y = u;
  g.c = abar;
  g.m = g.n = g.k = n;
  g.x_tri = 1;
  g.y_tri = 1;
  g.lower_out = 1;
  if (int st = launch_gemm_tc(g, mode, err, s)) return st;
  // S = U^T Z into w1.
  g = gemm_args(batch, n, pbig);
  g.x = u;
  g.y = abar;
  g.c = w1;
  g.m = g.n = g.k = n;
  g.trans_x = 1;
  g.x_tri = 2;
  g.y_tri = 1;
  if (int st = launch_gemm_tc(g, mode, err, s)) return st;
  {
    TraceScope ts(kKBwdSym, s);
    const int nt = (n + 31) / 32;
    const int64_t items = batch * ((int64_t)nt * (nt + 1) / 2);
    const int grid = (int)std::min<int64_t>(items, (int64_t)device_sms() * 8);
    sym_kernel<<<grid, kSymThreads, 0, s>>>(w1, abar, batch, n);
  }
  return check_launch("sym_kernel");
}

}  // namespace b2p
