// Batched triangular solves with a Cholesky factor, and the Gaussian-process
// log-likelihood built on them.
//
//   trsv_kernel<false, *>   L x = b          (forward substitution)
//   trsv_kernel<true,  *>   L^T x = b        (backward substitution)
//   trsv_kernel<false, GP>  alpha = L^{-1} y and loss = 1/2 alpha^T alpha + sum log L_ii
//   gp_lbar_kernel          Lbar = g (tril(-beta alpha^T) + diag(1 / L_ii)),
//                           beta = L^{-T} alpha (= A^{-1} y), g = dOut/dloss
//
// One matrix per thread-block cluster of C CTAs (C = 1 when the batch fills
// the GPU; up to 8 for a few large matrices), persistent over the batch.  The
// solve walks 32-row blocks, dealt round-robin to the CTAs of the cluster
// (block k belongs to rank k % C; each CTA keeps its own rows of x in shared
// memory).  For each block the owner's warp 0 solves the 32 x 32 diagonal
// block in registers (lane i owns row i, or column i for L^T; one shuffle
// per pivot) and publishes the 32 solved values; after one cluster barrier
// every CTA reads them over distributed shared memory and applies them to
// its own remaining rows (one row per thread and 32 loads in flight for L,
// float4 column groups for L^T).  All FP32.
//
// The reference has no GP path (its task is the forward factorization
// only); these implement the GP-solve step of its roadmap, with torch's
// solve_triangular and autograd in FP64 as the oracle.
#include <algorithm>

#include "launch.h"
#include "umma.cuh"

namespace b2p {

namespace {

constexpr int kTrsvThreads = 256;
constexpr int kTrsvMaxCluster = 8;

__device__ __forceinline__ float ld_cluster_f32(const float* local, uint32_t rank) {
  float v;
  asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(umma::cluster_addr(local, rank)) : "memory");
  return v;
}

// This lane's 32 values of the diagonal block at rows r0 .. r0 + m - 1: row
// `lane` of it, or column `lane` for L^T (zeros outside its lower triangle).
template <bool TRANS>
__device__ __forceinline__ void load_diag_block(const float* __restrict__ L, int n, int r0, int m, float (&e)[32]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    float v = 0.0f;
    if (TRANS) {
      if (j < m && lane < m && j >= lane) v = __ldg(L + (size_t)(r0 + j) * n + r0 + lane);
    } else {
      if (j < m && lane < m && j <= lane) v = __ldg(L + (size_t)(r0 + lane) * n + r0 + j);
    }
    e[j] = v;
  }
}

__device__ __forceinline__ void st_cluster_f32(float* local, uint32_t rank, float v) {
  asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(umma::cluster_addr(local, rank)), "f"(v) : "memory");
}

// Solves the diagonal block at rows r0 .. r0 + m - 1 in place in x (one
// warp), with e from load_diag_block.
template <bool TRANS>
__device__ __forceinline__ void solve_diag_block(const float (&e)[32], int r0, int m, float* x) {
  const int lane = threadIdx.x & 31;
  float r = lane < m ? x[r0 + lane] : 0.0f;
  float inv = 0.0f;  // 1 / L_ii of this lane's row (e[lane] is the diagonal)
#pragma unroll
  for (int j = 0; j < 32; ++j)
    if (j == lane) inv = lane < m ? 1.0f / e[j] : 0.0f;
  if (!TRANS) {
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      if (j < m) {
        const float xj = __shfl_sync(0xffffffffu, r * inv, j);
        if (lane == j) r = xj;
        if (lane > j) r -= e[j] * xj;
      }
    }
  } else {
#pragma unroll
    for (int j = 31; j >= 0; --j) {
      if (j < m) {
        const float xj = __shfl_sync(0xffffffffu, r * inv, j);
        if (lane == j) r = xj;
        if (lane < j) r -= e[j] * xj;
      }
    }
  }
  if (lane < m) x[r0 + lane] = r;
}

// L[i, r0:r0+32] . xb (32 loads in flight).
__device__ __forceinline__ float row_dot32(const float* __restrict__ row, const float* xb, bool vec) {
  float v[32];
  if (vec) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float4 t = __ldg(reinterpret_cast<const float4*>(row) + q);
      v[4 * q] = t.x;
      v[4 * q + 1] = t.y;
      v[4 * q + 2] = t.z;
      v[4 * q + 3] = t.w;
    }
  } else {
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __ldg(row + j);
  }
  float acc = 0.0f;
#pragma unroll
  for (int j = 0; j < 32; ++j) acc = fmaf(v[j], xb[j], acc);
  return acc;
}

// Shared memory of one CTA besides x (n floats, dynamic).
struct TrsvShared {
  float bcast[2][32];  // the owner's solved block, by block parity
  float xb[32];        // this CTA's copy of the solved block
  float red[kTrsvThreads / 32];
  float part[2];       // this CTA's partial loss sums (GP)
};

// x (this CTA's rows, holding b on entry) <- L^{-1} x or L^{-T} x.
template <bool TRANS>
__device__ void cluster_trsv(const float* __restrict__ L, int n, float* x, TrsvShared& sh, int C, int rank) {
  const int tid = threadIdx.x;
  const int nb = (n + 31) / 32;
  const bool vec = (n & 3) == 0;
  for (int s = 0; s < nb; ++s) {
    const int blk = TRANS ? nb - 1 - s : s;
    const int r0 = 32 * blk, m = min(32, n - r0);
    const int owner = blk % C;
    if (rank == owner && tid < 32) {
      float e[32];
      load_diag_block<TRANS>(L, n, r0, m, e);
      solve_diag_block<TRANS>(e, r0, m, x);
      if (tid < m) sh.bcast[s & 1][tid] = x[r0 + tid];
    }
    // The slot written at block s is rewritten at s + 2, after every CTA
    // has passed the barrier of s + 1, i.e. finished reading it.
    if (C > 1)
      umma::cluster_sync();
    else
      __syncthreads();
    if (tid < 32) {
      float v = 0.0f;
      if (tid < m) v = (C > 1) ? ld_cluster_f32(&sh.bcast[s & 1][tid], (uint32_t)owner) : sh.bcast[s & 1][tid];
      sh.xb[tid] = v;
    }
    __syncthreads();
    if (!TRANS) {
      // own rows below the block (only the last block is partial, and it
      // has none below): x[i] -= L[i, r0:r0+32] . xb
      const int first = blk + 1 + ((rank - (blk + 1) % C) % C + C) % C;
      const int nown = first < nb ? (nb - 1 - first) / C + 1 : 0;
      const int rows = 32 * nown;
      for (int idx = tid; idx < rows; idx += 2 * kTrsvThreads) {
        const int idx2 = idx + kTrsvThreads;
        const int i = 32 * (first + (idx >> 5) * C) + (idx & 31);
        const int i2 = 32 * (first + (idx2 >> 5) * C) + (idx2 & 31);
        const bool ok1 = i < n, ok2 = idx2 < rows && i2 < n;
        float a1 = 0.0f, a2 = 0.0f;
        if (ok1) a1 = row_dot32(L + (size_t)i * n + r0, sh.xb, vec);
        if (ok2) a2 = row_dot32(L + (size_t)i2 * n + r0, sh.xb, vec);
        if (ok1) x[i] -= a1;
        if (ok2) x[i2] -= a2;
      }
    } else {
      // own rows above the block: x[i] -= sum_j L[r0+j, i] xb[j] (column
      // reads, coalesced across threads)
      const int nown = blk > rank ? (blk - 1 - rank) / C + 1 : 0;
      if (vec) {
        for (int idx = tid; idx < 8 * nown; idx += kTrsvThreads) {
          const int i = 32 * (rank + (idx >> 3) * C) + 4 * (idx & 7);
          float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll 8
          for (int j = 0; j < m; ++j) {
            const float4 v = __ldg(reinterpret_cast<const float4*>(L + (size_t)(r0 + j) * n + i));
            const float w = sh.xb[j];
            acc.x = fmaf(v.x, w, acc.x);
            acc.y = fmaf(v.y, w, acc.y);
            acc.z = fmaf(v.z, w, acc.z);
            acc.w = fmaf(v.w, w, acc.w);
          }
          x[i] -= acc.x;
          x[i + 1] -= acc.y;
          x[i + 2] -= acc.z;
          x[i + 3] -= acc.w;
        }
      } else {
        for (int idx = tid; idx < 32 * nown; idx += kTrsvThreads) {
          const int i = 32 * (rank + (idx >> 5) * C) + (idx & 31);
          float acc = 0.0f;
#pragma unroll 8
          for (int j = 0; j < m; ++j) acc = fmaf(__ldg(L + (size_t)(r0 + j) * n + i), sh.xb[j], acc);
          x[i] -= acc;
        }
      }
    }
    __syncthreads();
  }
}

// The same solve for n % 4 == 0 with the loads of L issued one step ahead:
// the next step's diagonal block (by its owner's warp 0) while this step's
// update runs, and this thread's first operands of the next update right
// after this one, so that a step's critical path is the diagonal block's
// shuffles, the barriers and the FMAs rather than two round trips to
// memory.  With C > 1 the next block's owner is idle during this step's
// diagonal block and loads its own at the start of the step, and the owner
// stores the 32 solved values into every CTA's shared memory ahead of the
// cluster barrier (whose release / acquire makes them visible), so that no
// CTA reads them remotely behind it.  Same barriers in the same order as
// cluster_trsv.  The update of
// L^T runs as (column group of 4, group of 4 of the block's 32 rows) tasks,
// eight per column group in consecutive lanes, summed by shuffles.
template <bool TRANS>
__device__ void cluster_trsv_ahead(const float* __restrict__ L, int n, float* x, TrsvShared& sh, int C, int rank) {
  const int tid = threadIdx.x;
  const int nb = (n + 31) / 32;
  float e[32];         // the diagonal block of the current step (its owner's warp 0)
  float v[32];         // L: this thread's first row of the update
  float4 w[2][4];      // L^T: this thread's first two tasks of the update
  // Own rows below block blk (L): 32 nown rows from own block `first` on.
  auto rows_below = [&](int blk, int& first) {
    first = blk + 1 + ((rank - (blk + 1) % C) % C + C) % C;
    return first < nb ? 32 * ((nb - 1 - first) / C + 1) : 0;
  };
  auto row_of = [&](int first, int idx) { return 32 * (first + (idx >> 5) * C) + (idx & 31); };
  // Tasks above block blk (L^T): 8 per column group of this CTA's own rows.
  auto tasks_above = [&](int blk) { return blk > rank ? 64 * ((blk - 1 - rank) / C + 1) : 0; };
  auto col_of = [&](int t) {
    const int cg = t >> 3;
    return 32 * (rank + (cg >> 3) * C) + 4 * (cg & 7);
  };
  auto load_task = [&](int r0, int m, int t, int tasks, float4 (&q)[4]) {
    const int jg = t & 7;
    const int i = col_of(t);
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int j = 4 * jg + jj;
      q[jj] = (t < tasks && j < m) ? __ldg(reinterpret_cast<const float4*>(L + (size_t)(r0 + j) * n + i))
                                   : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };
  auto prefetch = [&](int s) {
    if (s >= nb) return;
    const int blk = TRANS ? nb - 1 - s : s;
    const int r0 = 32 * blk, m = min(32, n - r0);
    if (TRANS) {
      const int tasks = tasks_above(blk);
#pragma unroll
      for (int q = 0; q < 2; ++q) load_task(r0, m, tid + q * kTrsvThreads, tasks, w[q]);
    } else {
      int first;
      const int rows = rows_below(blk, first);
      const int i = row_of(first, tid);
      if (tid < rows && i < n) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const float4 t = __ldg(reinterpret_cast<const float4*>(L + (size_t)i * n + r0) + c);
          v[4 * c] = t.x;
          v[4 * c + 1] = t.y;
          v[4 * c + 2] = t.z;
          v[4 * c + 3] = t.w;
        }
      }
    }
  };
  {
    const int blk0 = TRANS ? nb - 1 : 0;
    if (rank == blk0 % C && tid < 32) load_diag_block<TRANS>(L, n, 32 * blk0, min(32, n - 32 * blk0), e);
  }
  prefetch(0);
  for (int s = 0; s < nb; ++s) {
    const int blk = TRANS ? nb - 1 - s : s;
    const int r0 = 32 * blk, m = min(32, n - r0);
    const int owner = blk % C;
    // With C > 1 the next step's owner differs from this one: its e is free.
    if (C > 1 && s + 1 < nb) {
      const int nblk = TRANS ? blk - 1 : blk + 1;
      if (rank == nblk % C && tid < 32) load_diag_block<TRANS>(L, n, 32 * nblk, min(32, n - 32 * nblk), e);
    }
    if (rank == owner && tid < 32) {
      solve_diag_block<TRANS>(e, r0, m, x);
      // All 32 entries (zeros past a partial block), so that no value of an
      // earlier matrix reaches the update.
      const float val = tid < m ? x[r0 + tid] : 0.0f;
      if (C > 1) {
        for (int q = 0; q < C; ++q) st_cluster_f32(&sh.bcast[s & 1][tid], (uint32_t)q, val);
      } else {
        sh.bcast[s & 1][tid] = val;
      }
    }
    // Barrier: the solved values are visible to every thread after it.
    if (C > 1)
      umma::cluster_sync();
    else
      __syncthreads();
    const float* xb = sh.bcast[s & 1];
    // The next step's diagonal block (C == 1: e is free again only now).
    if (C == 1 && s + 1 < nb) {
      const int nblk = TRANS ? blk - 1 : blk + 1;
      if (rank == nblk % C && tid < 32) load_diag_block<TRANS>(L, n, 32 * nblk, min(32, n - 32 * nblk), e);
    }
    if (!TRANS) {
      int first;
      const int rows = rows_below(blk, first);
      for (int idx = tid; idx < rows; idx += kTrsvThreads) {
        const int i = row_of(first, idx);
        if (i >= n) continue;
        float a = 0.0f;
        if (idx == tid) {
          // The prefetched row.
#pragma unroll
          for (int j = 0; j < 32; ++j) a = fmaf(v[j], xb[j], a);
        } else {
          a = row_dot32(L + (size_t)i * n + r0, xb, true);
        }
        x[i] -= a;
      }
    } else {
      const int tasks = tasks_above(blk);
      for (int t = tid; t - tid < tasks; t += kTrsvThreads) {
        float4 q[4];
        const int pass = (t - tid) / kTrsvThreads;
        if (pass == 0) {
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) q[jj] = w[0][jj];
        } else if (pass == 1) {
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) q[jj] = w[1][jj];
        } else {
          load_task(r0, m, t, tasks, q);
        }
        const int jg = t & 7;
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const float xv = xb[4 * jg + jj];
          acc.x = fmaf(q[jj].x, xv, acc.x);
          acc.y = fmaf(q[jj].y, xv, acc.y);
          acc.z = fmaf(q[jj].z, xv, acc.z);
          acc.w = fmaf(q[jj].w, xv, acc.w);
        }
        // Sum over the eight tasks of the column group (lanes 8g .. 8g + 7).
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
          acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
          acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
          acc.z += __shfl_xor_sync(0xffffffffu, acc.z, o);
          acc.w += __shfl_xor_sync(0xffffffffu, acc.w, o);
        }
        if (jg == 0 && t < tasks) {
          const int i = col_of(t);
          x[i] -= acc.x;
          x[i + 1] -= acc.y;
          x[i + 2] -= acc.z;
          x[i + 3] -= acc.w;
        }
      }
    }
    prefetch(s + 1);
    __syncthreads();
  }
}

// Sum over the CTA; the result is valid in thread 0.
__device__ __forceinline__ float cta_sum(float v, float* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  float t = 0.0f;
  if (threadIdx.x < 32) {
    t = lane < kTrsvThreads / 32 ? red[lane] : 0.0f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  __syncthreads();
  return t;
}

// One matrix per cluster of C CTAs (launched with that cluster size).  GP:
// b = y, xout = alpha, and loss[m] receives the log-likelihood terms.
template <bool TRANS, bool GP>
__global__ void __launch_bounds__(kTrsvThreads, 2) trsv_kernel(const float* __restrict__ l, const float* b, float* xout,
                                                            float* __restrict__ loss, int64_t batch, int n, int C) {
  extern __shared__ float xs[];
  __shared__ TrsvShared sh;
  const int rank = C > 1 ? (int)umma::cluster_rank() : 0;
  const int tid = threadIdx.x;
  const int nb = (n + 31) / 32;
  const int nown = rank < nb ? (nb - 1 - rank) / C + 1 : 0;  // blocks of this rank
  for (int64_t m = blockIdx.x / C; m < batch; m += gridDim.x / C) {
    const float* L = l + (size_t)m * n * n;
    for (int idx = tid; idx < 32 * nown; idx += kTrsvThreads) {
      const int i = 32 * (rank + (idx >> 5) * C) + (idx & 31);
      if (i < n) xs[i] = b[(size_t)m * n + i];
    }
    __syncthreads();
    if ((n & 3) == 0)
      cluster_trsv_ahead<TRANS>(L, n, xs, sh, C, rank);
    else
      cluster_trsv<TRANS>(L, n, xs, sh, C, rank);
    float quad = 0.0f, logdet = 0.0f;
    for (int idx = tid; idx < 32 * nown; idx += kTrsvThreads) {
      const int i = 32 * (rank + (idx >> 5) * C) + (idx & 31);
      if (i < n) {
        const float v = xs[i];
        xout[(size_t)m * n + i] = v;
        if (GP) {
          quad = fmaf(v, v, quad);
          logdet += logf(__ldg(L + (size_t)i * n + i));
        }
      }
    }
    if (GP) {
      const float q = cta_sum(quad, sh.red);
      const float ld = cta_sum(logdet, sh.red);
      if (tid == 0) {
        sh.part[0] = q;
        sh.part[1] = ld;
      }
      if (C > 1) {
        umma::cluster_sync();
        if (rank == 0 && tid == 0) {
          float qs = 0.0f, ls = 0.0f;
          for (int r = 0; r < C; ++r) {
            qs += ld_cluster_f32(&sh.part[0], (uint32_t)r);
            ls += ld_cluster_f32(&sh.part[1], (uint32_t)r);
          }
          loss[m] = 0.5f * qs + ls;
        }
      } else if (tid == 0) {
        loss[m] = 0.5f * q + ld;
      }
    }
    // No CTA moves on (or leaves) while another may still read its shared memory.
    if (C > 1)
      umma::cluster_sync();
    else
      __syncthreads();
  }
}

// Lbar, one warp per row (matrix, i); float4 stores when n % 4 == 0.
__global__ void __launch_bounds__(kTrsvThreads) gp_lbar_kernel(const float* __restrict__ l,
                                                               const float* __restrict__ alpha,
                                                               const float* __restrict__ beta,
                                                               const float* __restrict__ gloss,
                                                               float* __restrict__ lbar, int64_t batch, int n) {
  const int lane = threadIdx.x & 31;
  const int64_t rows = batch * (int64_t)n;
  const int64_t warps = (int64_t)gridDim.x * (kTrsvThreads / 32);
  for (int64_t row = ((int64_t)blockIdx.x * kTrsvThreads + threadIdx.x) >> 5; row < rows; row += warps) {
    const int64_t m = row / n;
    const int i = (int)(row - m * n);
    const float g = __ldg(gloss + m);
    const float bi = g * __ldg(beta + (size_t)m * n + i);
    const float dinv = g / __ldg(l + (size_t)m * n * n + (size_t)i * n + i);
    const float* a = alpha + (size_t)m * n;
    float* out = lbar + (size_t)m * n * n + (size_t)i * n;
    auto val = [&](int j) -> float {
      if (j > i) return 0.0f;
      const float v = -bi * __ldg(a + j);
      return j == i ? v + dinv : v;
    };
    if ((n & 3) == 0) {
      for (int j = 4 * lane; j < n; j += 128)
        *reinterpret_cast<float4*>(out + j) = make_float4(val(j), val(j + 1), val(j + 2), val(j + 3));
    } else {
      for (int j = lane; j < n; j += 32) out[j] = val(j);
    }
  }
}

int check_trsv_args(const void* p0, const void* p1, const void* p2, int64_t batch, int64_t n) {
  if (batch < 0 || n < 0 || n > kTrsvMaxN)
    return set_error(B2P_ERR_INVALID_ARG, "bad shape batch=%lld n=%lld (n <= %d)", (long long)batch, (long long)n,
                     kTrsvMaxN);
  if (batch > 0 && n > 0 && (p0 == nullptr || p1 == nullptr || p2 == nullptr))
    return set_error(B2P_ERR_INVALID_ARG, "null pointer");
  return B2P_OK;
}

// CTAs per matrix: more while the batch leaves SMs idle (each CTA keeps at
// least four 32-row blocks).
int trsv_cluster(int64_t batch, int n) {
  const int64_t sms = device_sms();
  const int nb = (n + 31) / 32;
  int c = 1;
  while (c < kTrsvMaxCluster && batch * c * 2 <= sms && c * 8 <= nb) c *= 2;
  return c;
}

template <bool TRANS, bool GP>
int launch_trsv_kernel(const float* l, const float* b, float* x, float* loss, int64_t batch, int n, int slot,
                       int kid, const char* what, cudaStream_t s) {
  const size_t smem = (size_t)n * sizeof(float);
  auto kern = trsv_kernel<TRANS, GP>;
  if (int st = ensure_smem_attr((const void*)kern, smem, slot)) return st;
  const int C = trsv_cluster(batch, n);
  const int64_t per_sm = 2048 / kTrsvThreads;
  const int64_t clusters = std::max<int64_t>(1, std::min<int64_t>(batch, (int64_t)device_sms() * per_sm / C));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(clusters * C), 1, 1);
  cfg.blockDim = dim3(kTrsvThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  TraceScope ts(kid, s);
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, l, b, x, loss, batch, n, C);
  if (e != cudaSuccess) return set_error(B2P_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return B2P_OK;
}

}  // namespace

int launch_trsv(const float* l, const float* b, float* x, int64_t batch, int n, bool trans, cudaStream_t s) {
  if (trans) return launch_trsv_kernel<true, false>(l, b, x, nullptr, batch, n, kSlotTrsv1, kKTrsv, "trsv_kernel", s);
  return launch_trsv_kernel<false, false>(l, b, x, nullptr, batch, n, kSlotTrsv0, kKTrsv, "trsv_kernel", s);
}

}  // namespace b2p

using namespace b2p;

extern "C" {

int b2p_trsv_batched(const float* l, const float* b, float* x, int64_t batch, int64_t n, int trans, void* stream) {
  if (int st = check_trsv_args(l, b, x, batch, n)) return st;
  if (batch == 0 || n == 0) return B2P_OK;
  return launch_trsv(l, b, x, batch, (int)n, trans != 0, static_cast<cudaStream_t>(stream));
}

int b2p_gp_nll_forward(const float* l, const float* y, float* alpha, float* loss, int64_t batch, int64_t n,
                       void* stream) {
  if (int st = check_trsv_args(l, y, alpha, batch, n)) return st;
  if (batch > 0 && loss == nullptr) return set_error(B2P_ERR_INVALID_ARG, "null loss pointer");
  if (batch == 0) return B2P_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n == 0) {
    const cudaError_t e = cudaMemsetAsync(loss, 0, (size_t)batch * sizeof(float), s);
    return e == cudaSuccess ? B2P_OK : set_error(B2P_ERR_CUDA, "cudaMemsetAsync: %s", cudaGetErrorString(e));
  }
  return launch_trsv_kernel<false, true>(l, y, alpha, loss, batch, (int)n, kSlotGpForward, kKGpForward,
                                         "gp_forward_kernel", s);
}

int b2p_gp_nll_backward(const float* l, const float* alpha, const float* gloss, float* beta, float* lbar,
                        int64_t batch, int64_t n, void* stream) {
  if (int st = check_trsv_args(l, alpha, beta, batch, n)) return st;
  if (batch > 0 && n > 0 && (gloss == nullptr || lbar == nullptr))
    return set_error(B2P_ERR_INVALID_ARG, "null pointer");
  if (batch == 0 || n == 0) return B2P_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (int st = launch_trsv(l, alpha, beta, batch, (int)n, true, s)) return st;
  const int64_t rows = batch * n;
  const int64_t per_cta = kTrsvThreads / 32;
  const int grid =
      (int)std::max<int64_t>(1, std::min<int64_t>((rows + per_cta - 1) / per_cta, (int64_t)device_sms() * 8));
  TraceScope ts(kKGpLbar, s);
  gp_lbar_kernel<<<grid, kTrsvThreads, 0, s>>>(l, alpha, beta, gloss, lbar, batch, (int)n);
  return check_launch("gp_lbar_kernel");
}

}  // extern "C"
