// Blocked right-looking factorization for n > 128 (plain FP32 SIMT form).
//
// The output buffer holds the working matrix.  For each 64-wide block column
// k0 three kernels run:
//
//   diag   one CTA per matrix: factor the 64x64 diagonal block and invert it
//          in shared memory (diag64.cuh); write L_kk (zeros above its
//          diagonal) and store T = inv(L_kk) (row-major) in the workspace;
//   panel  L[i, k0:k0+64] <- A[i, k0:k0+64] * T^T for the rows below
//          (the TRSM as a GEMM against the explicit inverse); CTA t also
//          zeroes the 64x64 block t of the strictly-upper strip to the right
//          of the diagonal block, so the strip is cleared by the whole grid;
//   trail  C[i, j] -= sum_m L[i, k0+m] L[j, k0+m] over the lower 64x64 tiles
//          of the trailing matrix (the SYRK).
//
// The first block column reads the caller's A directly (its diagonal block,
// its panel and, in the first trailing update, every lower tile), so A's
// lower triangle is read once and no separate copy pass runs; later steps
// work in place on L.  Every element of L is written exactly once by the
// step that finalises it, except the trailing tiles that later steps update.
//
// The reference reaches the same blocked schedule through cuSOLVER / cuBLAS
// and Triton (submission.py:2375-2661 split32, 3217-3251 right-looking TF32,
// 5152-5196 e62 diagonal block + inverse panel multiply); here every step is
// a kernel of this library.
#include <algorithm>
#include <mutex>

#include "diag64.cuh"
#include "launch.h"
#include "sched.cuh"

namespace b2p {

constexpr int kNB = 64;             // block column width
constexpr int kTile = 64;           // panel rows / trailing tile edge per CTA
constexpr int kGemmLd = kTile + 4;  // 68
constexpr int kMaxGridY = 65535;
constexpr int kOuterNB = 256;  // outer block column of the two-level schedule
// Orders that use the two-level schedule (tensor modes).  Its K = 256 update
// runs through gemm_tc_kernel, whose per-chunk staging is not yet faster
// than the single-level tcgen05 SYRK on any measured order (1x8192: 10.9 vs
// 10.3 ms), so the threshold is above every order the library accepts until
// that kernel streams its operands.
constexpr int kTwoLevelMin = 1 << 21;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// -------------------------------------------------------------------------
// diag: factor + invert the 64x64 diagonal block of every matrix.
template <bool RAGGED>
__global__ void __launch_bounds__(kD64Threads, 3)
    diag_kernel(const float* __restrict__ src, float* __restrict__ l, Sched sch, int k0,
                float* __restrict__ tws, int32_t* __restrict__ info) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Diag64Smem& sm = *reinterpret_cast<Diag64Smem*>(smem_raw);
  const int tid = threadIdx.x;
  for (int64_t it = blockIdx.x; it < sch.count; it += gridDim.x) {
    const Target tg = resolve_matrix<RAGGED>(sch, it);
    const int n = tg.n;
    const int64_t b = tg.pos;
    const int w = min(kNB, n - k0);
    const bool vec = (n & 3) == 0;  // then w is a multiple of 4 as well
    const size_t moff = tg.off + (size_t)k0 * n + k0;
    const float* in = src + moff;
    float* base = l + moff;
    if (vec) {
      float4 v[8];
#pragma unroll
      for (int it = 0; it < 8; ++it) {
        const int e4 = tid + kD64Threads * it;
        const int r = e4 >> 4, c = (e4 & 15) * 4;
        v[it] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (r < w && c <= r) v[it] = *reinterpret_cast<const float4*>(in + (size_t)r * n + c);
      }
#pragma unroll
      for (int it = 0; it < 8; ++it) {
        const int e4 = tid + kD64Threads * it;
        const int r = e4 >> 4, c = (e4 & 15) * 4;
        float e[4] = {v[it].x, v[it].y, v[it].z, v[it].w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (c + q > r) e[q] = 0.0f;
          if (r >= w) e[q] = (r == c + q) ? 1.0f : 0.0f;
        }
        *reinterpret_cast<float4*>(sm.S + r * kD64Ld + c) = make_float4(e[0], e[1], e[2], e[3]);
      }
    } else {
      float v[32];
#pragma unroll
      for (int it = 0; it < 32; ++it) {
        const int e = tid + kD64Threads * it;
        const int r = e >> 6, c = e & 63;
        v[it] = (r == c) ? 1.0f : 0.0f;
        if (r < w && c <= r) v[it] = in[(size_t)r * n + c];
        else if (r < w) v[it] = 0.0f;
      }
#pragma unroll
      for (int it = 0; it < 32; ++it) {
        const int e = tid + kD64Threads * it;
        sm.S[(e >> 6) * kD64Ld + (e & 63)] = v[it];
      }
    }
    __syncthreads();
    const int bad = diag64_factor_invert(sm);
    // L_kk (zeros above its diagonal; the engine leaves them in S).
    if (vec) {
#pragma unroll
      for (int it = 0; it < 8; ++it) {
        const int e4 = tid + kD64Threads * it;
        const int r = e4 >> 4, c = (e4 & 15) * 4;
        if (r < w && c < w) {
          const float* sr = sm.S + r * kD64Ld + c;
          *reinterpret_cast<float4*>(base + (size_t)r * n + c) =
              make_float4(c <= r ? sr[0] : 0.f, c + 1 <= r ? sr[1] : 0.f, c + 2 <= r ? sr[2] : 0.f,
                          c + 3 <= r ? sr[3] : 0.f);
        }
      }
    } else {
      for (int e = tid; e < 64 * 64; e += kD64Threads) {
        const int r = e >> 6, c = e & 63;
        if (r < w && c < w) base[(size_t)r * n + c] = (c <= r) ? sm.S[r * kD64Ld + c] : 0.0f;
      }
    }
    // T^T (T = inv(L_kk)) as the engine leaves it: tws[m][c] = T[c][m].
    float* tb = tws + b * kNB * kNB;
#pragma unroll
    for (int it = 0; it < 8; ++it) {
      const int e4 = tid + kD64Threads * it;
      const int r = e4 >> 4, c = (e4 & 15) * 4;
      const float* tr = sm.T + r * kD64Ld + c;
      float4 v = make_float4(tr[0], tr[1], tr[2], tr[3]);
      if (r >= w) v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (c + 0 >= w) v.x = 0.f;
      if (c + 1 >= w) v.y = 0.f;
      if (c + 2 >= w) v.z = 0.f;
      if (c + 3 >= w) v.w = 0.f;
      reinterpret_cast<float4*>(tb)[e4] = v;
    }
    if (info != nullptr && tid == 0) {
      if (bad == kDiagTimeout)
        info[tg.mat] = -1;
      else if (k0 == 0)
        info[tg.mat] = bad >= 0 ? bad + 1 : 0;
      else if (bad >= 0 && info[tg.mat] == 0)
        info[tg.mat] = k0 + bad + 1;
    }
    __syncthreads();
  }
}

// -------------------------------------------------------------------------
// The panel multiply and the trailing update run 256 threads per 64x64 tile
// (4x4 outputs per thread: four times the warps of the 8x8 layout, for
// latency hiding at the same shared-memory footprint).  Each output still
// accumulates m = 0..63 in order with one fmaf per step, so results equal the
// 8x8 layout's bit for bit.
constexpr int kTrailThreads = 256;

// load_rows_t with 256 threads: thread (row t % 64, quarter t / 64) moves 16 values.
__device__ __forceinline__ void load_rows_t256(const float* __restrict__ mat, int n, int row0, int col0,
                                               float* dst) {
  const int i = threadIdx.x & 63, q4 = threadIdx.x >> 6;
  const bool ok = row0 + i < n;
  if ((n & 3) == 0) {
    const float4* src = reinterpret_cast<const float4*>(mat + (size_t)(ok ? row0 + i : 0) * n + col0) + 4 * q4;
    float4 v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = ok ? src[q] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int m = 16 * q4 + 4 * q;
      dst[(m + 0) * kGemmLd + i] = v[q].x;
      dst[(m + 1) * kGemmLd + i] = v[q].y;
      dst[(m + 2) * kGemmLd + i] = v[q].z;
      dst[(m + 3) * kGemmLd + i] = v[q].w;
    }
  } else {
    const float* src = mat + (size_t)(ok ? row0 + i : 0) * n + col0;
#pragma unroll 16
    for (int m = 16 * q4; m < 16 * q4 + 16; ++m) dst[m * kGemmLd + i] = ok ? src[m] : 0.0f;
  }
}

// acc[r][c] = sum_m As[m][4ty + r] * Bs[m][4tx + c]
__device__ __forceinline__ void tile_mma_4x4(const float* As, const float* Bs, int ty, int tx, float (&acc)[4][4]) {
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = 0.0f;
#pragma unroll 8
  for (int m = 0; m < kNB; ++m) {
    const float4 a = *reinterpret_cast<const float4*>(As + m * kGemmLd + 4 * ty);
    const float4 b = *reinterpret_cast<const float4*>(Bs + m * kGemmLd + 4 * tx);
    const float a4[4] = {a.x, a.y, a.z, a.w};
    const float b4[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[r][c] = fmaf(a4[r], b4[c], acc[r][c]);
  }
}

template <bool RAGGED>
__global__ void __launch_bounds__(kTrailThreads)
    panel_kernel(const float* __restrict__ src, float* __restrict__ l, Sched sch, int k0,
                 const float* __restrict__ tws) {
  __shared__ __align__(16) float Ps[kNB * kGemmLd];
  __shared__ __align__(16) float Ts[kNB * kGemmLd];
  const int tid = threadIdx.x;
  const int ty = tid >> 4, tx = tid & 15;
  const int64_t start = RAGGED ? blockIdx.x : blockIdx.y;
  const int64_t stride = RAGGED ? gridDim.x : gridDim.y;
  for (int64_t it = start; it < sch.count; it += stride) {
    const Target tg = resolve_tile<RAGGED>(sch, it);
    const int n = tg.n;
    const int row0 = k0 + kNB + tg.ti * kTile;
    const size_t moff = tg.off;
    const float* tb = tws + tg.pos * kNB * kNB;
    // Ts[m][c] = T[c][m]: the diagonal kernel stored T^T row-major.
    {
      float4 tv[4];
#pragma unroll
      for (int it = 0; it < 4; ++it) tv[it] = __ldg(reinterpret_cast<const float4*>(tb) + tid + kTrailThreads * it);
      load_rows_t256(src + moff, n, row0, k0, Ps);
#pragma unroll
      for (int it = 0; it < 4; ++it) {
        const int e = tid + kTrailThreads * it;
        *reinterpret_cast<float4*>(Ts + (e >> 4) * kGemmLd + (e & 15) * 4) = tv[it];
      }
    }
    __syncthreads();
    float acc[4][4];
    tile_mma_4x4(Ps, Ts, ty, tx, acc);
    float* mat = l + moff;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int i = row0 + 4 * ty + r;
      if (i < n) {
        float* dst = mat + (size_t)i * n + k0;
        if ((n & 3) == 0) {
          reinterpret_cast<float4*>(dst + 4 * tx)[0] = make_float4(acc[r][0], acc[r][1], acc[r][2], acc[r][3]);
        } else {
#pragma unroll
          for (int c = 0; c < 4; ++c) dst[4 * tx + c] = acc[r][c];
        }
      }
    }
    // Zero block ti of the strip: rows k0..k0+63, cols k0+64+64*ti .. +63.
    {
      const int c0 = k0 + kNB + tg.ti * kTile;
      const int cw = min(kTile, n - c0);
      float* zb = mat + (size_t)k0 * n + c0;
      if ((n & 3) == 0) {
        const int q4 = cw >> 2;
        for (int e = tid; e < kNB * q4; e += kTrailThreads) {
          const int r = e / q4, q = e - (e / q4) * q4;
          reinterpret_cast<float4*>(zb + (size_t)r * n)[q] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
      } else {
        for (int e = tid; e < kNB * cw; e += kTrailThreads) {
          const int r = e / cw, c = e - (e / cw) * cw;
          zb[(size_t)r * n + c] = 0.0f;
        }
      }
    }
    __syncthreads();
  }
}

// Trailing SYRK on lower 64x64 tiles.  The C tile is prefetched into shared
// memory with cp.async while the panel tiles load and multiply; `csrc` is A
// for the first block column and L afterwards, the result always goes to L.
template <bool RAGGED>
__global__ void __launch_bounds__(kTrailThreads)
    trail_kernel(const float* __restrict__ csrc, float* __restrict__ l, Sched sch, int k0, int part) {
  extern __shared__ __align__(16) float tsm[];
  float* As = tsm;
  float* Bs = As + kNB * kGemmLd;
  float* Cs = Bs + kNB * kGemmLd;  // [64][kGemmLd], row-major C tile
  const int tid = threadIdx.x;
  const int ty = tid >> 4, tx = tid & 15;
  const int64_t start = RAGGED ? blockIdx.x : blockIdx.y;
  const int64_t stride = RAGGED ? gridDim.x : gridDim.y;
  for (int64_t it = start; it < sch.count; it += stride) {
    const Target tg = resolve_tile<RAGGED>(sch, it);
    const int n = tg.n;
    int ti = tg.ti, tj = tg.tj;
    if (!RAGGED) {
      // part 0: every lower tile; 1: the first tile column only (the next
      // block column, for the look-ahead); 2: every lower tile but those.
      const int q = blockIdx.x;
      if (part == 1) {
        ti = q;
        tj = 0;
      } else {
        ti = (int)((sqrtf(8.0f * q + 1.0f) - 1.0f) * 0.5f);
        while ((ti + 1) * (ti + 2) / 2 <= q) ++ti;
        while (ti * (ti + 1) / 2 > q) --ti;
        tj = q - ti * (ti + 1) / 2;
        if (part == 2) {
          ++ti;
          ++tj;
        }
      }
    }
    const int t0 = k0 + kNB;
    const int i0 = t0 + ti * kTile, j0 = t0 + tj * kTile;
    const bool vec = (n & 3) == 0 && j0 + 64 <= n;
    const size_t moff = tg.off;
    if (vec) {
#pragma unroll
      for (int it = 0; it < 4; ++it) {
        const int e = tid + kTrailThreads * it;
        const int r = e >> 4, c4 = e & 15;
        if (i0 + r < n) cp_async16(Cs + r * kGemmLd + 4 * c4, csrc + moff + (size_t)(i0 + r) * n + j0 + 4 * c4);
      }
      cp_async_commit();
    }
    float* mat = l + moff;
    load_rows_t256(mat, n, i0, k0, As);
    if (ti != tj) load_rows_t256(mat, n, j0, k0, Bs);
    __syncthreads();
    float acc[4][4];
    tile_mma_4x4(As, ti != tj ? Bs : As, ty, tx, acc);
    if (vec) cp_async_wait_all();
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int rl = 4 * ty + r;
      const int i = i0 + rl;
      if (i < n) {
        float* row = mat + (size_t)i * n + j0;
        if (vec && ti != tj) {
          float4 c = *reinterpret_cast<const float4*>(Cs + rl * kGemmLd + 4 * tx);
          c.x -= acc[r][0];
          c.y -= acc[r][1];
          c.z -= acc[r][2];
          c.w -= acc[r][3];
          *reinterpret_cast<float4*>(row + 4 * tx) = c;
        } else {
          const float* crow = csrc + moff + (size_t)i * n + j0;
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            const int jl = 4 * tx + c;
            if (j0 + jl <= i && j0 + jl < n) row[jl] = (vec ? Cs[rl * kGemmLd + jl] : crow[jl]) - acc[r][c];
          }
        }
      }
    }
    __syncthreads();
  }
}

// -------------------------------------------------------------------------
// B2P_FLAG_FP64_DIAG: the diagonal step in FP64.  Same contract as
// diag_kernel (dense batches): the block's lower triangle (identity beyond
// w = min(64, n - k0)) is factored right-looking in FP64 shared memory, the
// inverse T = L_kk^{-1} follows by column substitution (thread c: column c),
// and L_kk (zeros above) and T^T go out rounded to FP32; info takes the first
// pivot that is not positive.  One CTA per matrix, 128 threads.
constexpr int kD64fLd = 65;
constexpr size_t kDiagF64Smem = 2 * 64 * kD64fLd * sizeof(double);

__global__ void __launch_bounds__(kD64Threads) diag_kernel_f64(const float* __restrict__ src, float* __restrict__ l,
                                                               Sched sch, int k0, float* __restrict__ tws,
                                                               int32_t* __restrict__ info) {
  extern __shared__ __align__(16) double dsm[];
  double* S = dsm;               // [64][kD64fLd]: the block, then L_kk
  double* Tm = dsm + 64 * kD64fLd;  // [64][kD64fLd]: T = L_kk^{-1} (lower)
  __shared__ int sbad;
  const int tid = threadIdx.x;
  for (int64_t it = blockIdx.x; it < sch.count; it += gridDim.x) {
    const Target tg = resolve_matrix<false>(sch, it);
    const int n = tg.n;
    const int64_t b = tg.pos;
    const int w = min(kNB, n - k0);
    const size_t moff = tg.off + (size_t)k0 * n + k0;
    const float* in = src + moff;
    float* base = l + moff;
    for (int e = tid; e < 64 * 64; e += kD64Threads) {
      const int r = e >> 6, c = e & 63;
      double v = (r == c) ? 1.0 : 0.0;
      if (r < w) v = (c <= r) ? (double)in[(size_t)r * n + c] : 0.0;
      S[r * kD64fLd + c] = v;
    }
    if (tid == 0) sbad = -1;
    __syncthreads();
    for (int k = 0; k < 64; ++k) {
      if (tid == 0) {
        const double d = S[k * kD64fLd + k];
        if (!(d > 0.0) && sbad < 0) sbad = k;
        S[k * kD64fLd + k] = sqrt(d);
      }
      __syncthreads();
      const double piv = S[k * kD64fLd + k];
      for (int i = k + 1 + tid; i < 64; i += kD64Threads) S[i * kD64fLd + k] /= piv;
      __syncthreads();
      // S[i][j] -= S[i][k] S[j][k] for k < j <= i
      const int m = 63 - k;
      for (int e = tid; e < m * m; e += kD64Threads) {
        const int i = k + 1 + e / m, j = k + 1 + e % m;
        if (j <= i) S[i * kD64fLd + j] -= S[i * kD64fLd + k] * S[j * kD64fLd + k];
      }
      __syncthreads();
    }
    if (tid < 64) {
      const int c = tid;
      for (int i = 0; i < c; ++i) Tm[i * kD64fLd + c] = 0.0;
      for (int i = c; i < 64; ++i) {
        double acc = (i == c) ? 1.0 : 0.0;
        for (int k = c; k < i; ++k) acc -= S[i * kD64fLd + k] * Tm[k * kD64fLd + c];
        Tm[i * kD64fLd + c] = acc / S[i * kD64fLd + i];
      }
    }
    __syncthreads();
    for (int e = tid; e < 64 * 64; e += kD64Threads) {
      const int r = e >> 6, c = e & 63;
      if (r < w && c < w) base[(size_t)r * n + c] = (c <= r) ? (float)S[r * kD64fLd + c] : 0.0f;
    }
    // tws[m][c] = T[c][m]
    float* tb = tws + b * kNB * kNB;
    for (int e = tid; e < 64 * 64; e += kD64Threads) {
      const int mm = e >> 6, c = e & 63;
      tb[e] = (mm < w && c < w) ? (float)Tm[c * kD64fLd + mm] : 0.0f;
    }
    if (info != nullptr && tid == 0) {
      const int bad = sbad;
      if (k0 == 0)
        info[tg.mat] = bad >= 0 ? bad + 1 : 0;
      else if (bad >= 0 && info[tg.mat] == 0)
        info[tg.mat] = k0 + bad + 1;
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

namespace {
// Per device: the stream the FP32 look-ahead runs the bulk of each trailing
// update on, with the events that fork it from and join it to the caller's.
struct TrailStream {
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  cudaEvent_t join = nullptr;
  int priority = 0;  // the device's greatest (numerically lowest) launch priority
};
constexpr int kTrailDevices = 64;
TrailStream g_trail[kTrailDevices];
std::mutex g_trail_mu;

int trail_stream(TrailStream** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kTrailDevices)
    return set_error(B2P_ERR_CUDA, "no usable current device");
  std::lock_guard<std::mutex> lock(g_trail_mu);
  TrailStream& t = g_trail[dev];
  if (t.stream == nullptr) {
    cudaError_t e = cudaStreamCreateWithFlags(&t.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t.fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t.join, cudaEventDisableTiming);
    int least = 0, greatest = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e != cudaSuccess) return set_error(B2P_ERR_CUDA, "trail stream set-up: %s", cudaGetErrorString(e));
    t.priority = greatest;
  }
  *out = &t;
  return B2P_OK;
}

// Launches `k` on `s`.  With `prio` set its CTAs take that launch priority,
// so they go first when the look-ahead's side-stream update holds the SMs
// (a CUDA graph's kernel node keeps the priority too).
template <typename... KArgs, typename... Args>
int launch_prio(const char* what, void (*k)(KArgs...), dim3 grid, int threads, size_t smem, cudaStream_t s,
                const int* prio, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3((unsigned)threads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  if (prio != nullptr) {
    attr[0].id = cudaLaunchAttributePriority;
    attr[0].val.priority = *prio;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
  const cudaError_t e = cudaLaunchKernelEx(&cfg, k, args...);
  return e == cudaSuccess ? B2P_OK : set_error(B2P_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}
}  // namespace

int potrf_blocked(const float* a, float* l, int64_t batch, int n, int mode, void* ws,
                  size_t ws_bytes, int32_t* info, cudaStream_t s) {
  const int m = mode & B2P_MODE_MASK;
  if (m == B2P_MODE_FP8) return set_error(B2P_ERR_UNSUPPORTED, "mode 0x%x not available for n=%d", mode, n);
  const bool f64diag = (mode & B2P_FLAG_FP64_DIAG) != 0;
  const bool tensor = (m == B2P_MODE_TF32 || m == B2P_MODE_BF16X3);
  const size_t need = blocked_workspace_bytes(batch, n, mode);
  if (ws == nullptr || ws_bytes < need)
    return set_error(B2P_ERR_WORKSPACE, "workspace of %zu bytes required, %zu given", need, ws_bytes);
  float* tws = static_cast<float*>(ws);
  const int sms = device_sms();
  const size_t dsmem = sizeof(Diag64Smem);
  if (int st = ensure_smem_attr((const void*)diag_kernel<false>, dsmem, kSlotDiag)) return st;
  if (f64diag) {
    if (int st = ensure_smem_attr((const void*)diag_kernel_f64, kDiagF64Smem, kSlotDiagF64)) return st;
  }
  const size_t tsmem = (size_t)3 * kNB * kGemmLd * sizeof(float);
  if (int st = ensure_smem_attr((const void*)trail_kernel<false>, tsmem, kSlotTrail)) return st;
  const int gy = (int)std::min<int64_t>(batch, kMaxGridY);
  const Sched sch = dense_sched(batch, n);
  // Tensor modes on large orders: two-level blocking.  Inner 64-wide steps
  // factor a 256-wide block column (their trailing updates limited to its
  // columns); one tcgen05 SYRK with K = 256 then updates the rest.
  const int outer = (tensor && n >= kTwoLevelMin) ? kOuterNB : n;
  // FP32 look-ahead: diag, panel and the next column's update carry the
  // critical path, so they launch at the device's greatest priority.
  const int* prio = nullptr;
  if (!tensor && n > kNB) {
    TrailStream* ts0 = nullptr;
    if (int st = trail_stream(&ts0)) return st;
    prio = &ts0->priority;
  }
  for (int K0 = 0; K0 < n; K0 += outer) {
    const int jmax = std::min(n, K0 + outer);
    for (int k0 = K0; k0 < jmax; k0 += kNB) {
      const float* src = (k0 == 0) ? a : l;
      const int dgrid = (int)std::min<int64_t>(batch, (int64_t)sms * 16);
      {
        TraceScope ts(kKDiag, s);
        const int st = f64diag ? launch_prio("diag_kernel_f64", diag_kernel_f64, dim3(dgrid), kD64Threads,
                                             kDiagF64Smem, s, prio, src, l, sch, k0, tws, info)
                               : launch_prio("diag_kernel", diag_kernel<false>, dim3(dgrid), kD64Threads, dsmem, s,
                                             prio, src, l, sch, k0, tws, info);
        if (st) return st;
      }
      const int R = n - k0 - kNB;
      if (R <= 0) {
        // The FP32 look-ahead's stream rejoins the caller's before the end.
        if (!tensor && k0 > K0) {
          TrailStream* ts2 = nullptr;
          if (int st = trail_stream(&ts2)) return st;
          const cudaError_t e = cudaStreamWaitEvent(s, ts2->join, 0);
          if (e != cudaSuccess) return set_error(B2P_ERR_CUDA, "cudaStreamWaitEvent: %s", cudaGetErrorString(e));
        }
        return B2P_OK;
      }
      const int T = (R + kTile - 1) / kTile;
      {
        TraceScope ts(kKPanel, s);
        if (int st = launch_prio("panel_kernel", panel_kernel<false>, dim3(T, gy), kTrailThreads, 0, s, prio, src, l,
                                 sch, k0, tws))
          return st;
      }
      if (k0 + kNB >= jmax) continue;
      if (tensor) {
        if (int st = launch_syrk_tc(src, l, sch, false, T_tc(n, k0), k0, mode, info, s, jmax < n ? jmax : 0))
          return st;
        continue;
      }
      // FP32 look-ahead: the tiles of the next block column first (they are
      // all diag and panel of step k+1 read), the rest on the side stream
      // beside that step; step k+1's own update waits for the rest.
      TrailStream* ts2 = nullptr;
      if (int st = trail_stream(&ts2)) return st;
      auto check = [](cudaError_t e, const char* what) -> int {
        return e == cudaSuccess ? B2P_OK : set_error(B2P_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
      };
      if (k0 > K0) {
        if (int st = check(cudaStreamWaitEvent(s, ts2->join, 0), "cudaStreamWaitEvent")) return st;
      }
      {
        TraceScope ts(kKTrail, s);
        if (int st = launch_prio("trail_kernel", trail_kernel<false>, dim3(T, gy), kTrailThreads, tsmem, s, prio, src,
                                 l, sch, k0, 1))
          return st;
      }
      if (int st = check(cudaEventRecord(ts2->fork, s), "cudaEventRecord")) return st;
      if (int st = check(cudaStreamWaitEvent(ts2->stream, ts2->fork, 0), "cudaStreamWaitEvent")) return st;
      if (T > 1) {
        TraceScope ts(kKTrail, ts2->stream);
        trail_kernel<false><<<dim3(T * (T - 1) / 2, gy), kTrailThreads, tsmem, ts2->stream>>>(src, l, sch, k0, 2);
        if (int st = check_launch("trail_kernel")) return st;
      }
      if (int st = check(cudaEventRecord(ts2->join, ts2->stream), "cudaEventRecord")) return st;
    }
    if (jmax < n) {
      // C[jmax:, jmax:] -= X X^T, X = L[jmax:, K0:jmax] (lower triangle only).
      const size_t nn = (size_t)n;
      GemmArgs g{};
      g.x = l + (size_t)jmax * nn + K0;
      g.y = g.x;
      g.c = l + (size_t)jmax * nn + jmax;
      g.c_in = ((K0 == 0) ? a : l) + (size_t)jmax * nn + jmax;
      g.sx = g.sy = g.sc = (int64_t)n * n;
      g.ldx = g.ldy = g.ldc = n;
      g.m = g.n = n - jmax;
      g.k = jmax - K0;
      g.trans_y = 1;
      g.lower_out = 1;
      g.alpha = -1.0f;
      g.beta = 1.0f;
      g.batch = batch;
      if (int st = launch_gemm_tc(g, mode, nullptr, s)) return st;
    }
  }
  return B2P_OK;
}

// One block-column step of the ragged schedule (potrf_ragged.cu builds it):
// the first `ndiag` positions of the big-matrix list are active, `panel`
// and `trail` are item lists on the device.
int ragged_blocked_step(const float* a, float* l, const RaggedTables& t, const RaggedStep& st, int k0, int mode,
                        float* tws, int32_t* info, cudaStream_t s) {
  const int m = mode & B2P_MODE_MASK;
  const bool tensor = (m == B2P_MODE_TF32 || m == B2P_MODE_BF16X3);
  const float* src = (k0 == 0) ? a : l;
  const int sms = device_sms();
  const size_t dsmem = sizeof(Diag64Smem);
  if (int e = ensure_smem_attr((const void*)diag_kernel<true>, dsmem, kSlotDiagR)) return e;
  const size_t tsmem = (size_t)3 * kNB * kGemmLd * sizeof(float);
  if (int e = ensure_smem_attr((const void*)trail_kernel<true>, tsmem, kSlotTrailR)) return e;
  Sched sd = ragged_sched(t, nullptr, st.ndiag);
  if (st.ndiag > 0) {
    TraceScope ts(kKDiag, s);
    diag_kernel<true><<<(int)std::min<int64_t>(st.ndiag, (int64_t)sms * 16), kD64Threads, dsmem, s>>>(
        src, l, sd, k0, tws, info);
  }
  if (int e = check_launch("diag_kernel<ragged>")) return e;
  if (st.npanel > 0) {
    Sched sp = ragged_sched(t, t.items + st.panel_beg, st.npanel);
    TraceScope ts(kKPanel, s);
    panel_kernel<true><<<(int)std::min<int64_t>(st.npanel, 1 << 30), kTrailThreads, 0, s>>>(src, l, sp, k0, tws);
  }
  if (int e = check_launch("panel_kernel<ragged>")) return e;
  if (st.ntrail > 0) {
    Sched sr = ragged_sched(t, t.items + st.trail_beg, st.ntrail);
    if (tensor) return launch_syrk_tc(src, l, sr, true, 0, k0, mode, info, s);
    TraceScope ts(kKTrail, s);
    trail_kernel<true><<<(int)std::min<int64_t>(st.ntrail, 1 << 30), kTrailThreads, tsmem, s>>>(src, l, sr, k0, 0);
  }
  return check_launch("trail_kernel<ragged>");
}

}  // namespace b2p
