// Trailing (Schur complement) update on the tcgen05 tensor cores.
//
// C[i, j] -= sum_m X[i, m] X[j, m]  for the lower 128x128 tiles of the
// trailing matrix, X = L[:, k0:k0+64] the freshly solved panel (FP32).
// One 128-thread CTA per tile:
//   1. warp 0 allocates 128 TMEM columns (the 128x128 FP32 accumulator);
//   2. every thread stages one row of each operand into shared memory in
//      the 128B-swizzled K-major layout, converting on the way:
//        TF32   : the value rounded to TF32 (cvt.rna), 2 swizzle atoms per row;
//        BF16x3 : hi = bf16(x) and lo = bf16(x - hi) in two separate tiles;
//   3. thread 0 issues the MMAs (TF32: 8 x K=8; BF16x3: 4 x K=16 for each of
//      hi*hi, hi*lo, lo*hi) and commits them to an mbarrier;
//   4. each warp reads its 32 accumulator rows from TMEM (tcgen05.ld) and
//      writes C - D to L for the lower-triangular part.
// All waits are bounded; on timeout the kernel records B2P_ERR_TIMEOUT in
// the error word, waits a bounded time again, frees TMEM and returns.
//
// The reference runs this update through cuBLAS TF32 GEMMs (baddbmm_/addmm_,
// submission.py:2529-2534,3319-3409) and Triton `_trailing_nb`
// (submission.py:2201-2252).
#include <algorithm>

#include "launch.h"
#include "sched.cuh"
#include "umma.cuh"

namespace b2p {

constexpr int kTcTile = 128;
constexpr int kTcK = 64;  // block column width of the blocked path
constexpr int kTcThreads = 128;
constexpr uint32_t kTcMaxPolls = 1u << 24;
constexpr size_t kTcOperandBytes = 32768;  // one operand: 128 rows x 64 K (fp32 or bf16 hi+lo)
constexpr size_t kTcSmemBytes = 2 * kTcOperandBytes + 1024 /*alignment slack*/ + 64;

__device__ __forceinline__ float round_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Stage row r (64 FP32 values at src, or zeros when src is null) of one operand.
template <int MODE>
__device__ __forceinline__ void stage_row(const float* src, bool vec, uint8_t* op, int r) {
  float4 v[16];
  if (src != nullptr) {
    if (vec) {
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = reinterpret_cast<const float4*>(src)[q];
    } else {
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = make_float4(src[4 * q], src[4 * q + 1], src[4 * q + 2], src[4 * q + 3]);
    }
  } else {
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  if (MODE == B2P_MODE_TF32) {
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      float4 t = make_float4(round_tf32(v[q].x), round_tf32(v[q].y), round_tf32(v[q].z), round_tf32(v[q].w));
      const int atom = q >> 3, c = q & 7;
      *reinterpret_cast<float4*>(op + atom * 16384 + umma::sw128_offset(r, c)) = t;
    }
  } else {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const float x[8] = {v[2 * c].x, v[2 * c].y, v[2 * c].z, v[2 * c].w,
                          v[2 * c + 1].x, v[2 * c + 1].y, v[2 * c + 1].z, v[2 * c + 1].w};
      uint32_t hi[4], lo[4];
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        __nv_bfloat16 h0, l0, h1, l1;
        umma::split_bf16(x[2 * p], h0, l0);
        umma::split_bf16(x[2 * p + 1], h1, l1);
        hi[p] = umma::pack_bf16(h0, h1);
        lo[p] = umma::pack_bf16(l0, l1);
      }
      const uint32_t off = umma::sw128_offset(r, c);
      *reinterpret_cast<uint4*>(op + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
      *reinterpret_cast<uint4*>(op + 16384 + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    }
  }
}

// D = A * B^T over K = 64 (issued by one thread).
template <int MODE>
__device__ __forceinline__ void issue_mmas(uint32_t tmem, const uint8_t* opA, const uint8_t* opB) {
  const uint32_t a = umma::smem_u32(opA), b = umma::smem_u32(opB);
  if (MODE == B2P_MODE_TF32) {
    constexpr uint32_t idesc = umma::idesc_f32acc(2, kTcTile, kTcTile);
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      const uint32_t off = (uint32_t)((s >> 2) * 16384 + (s & 3) * 32);
      umma::mma_tf32(tmem, umma::desc_k_sw128(a + off), umma::desc_k_sw128(b + off), idesc, s > 0 ? 1u : 0u);
    }
  } else {
    constexpr uint32_t idesc = umma::idesc_f32acc(1, kTcTile, kTcTile);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const uint32_t off = (uint32_t)(s * 32);
      const uint64_t ah = umma::desc_k_sw128(a + off), al = umma::desc_k_sw128(a + 16384 + off);
      const uint64_t bh = umma::desc_k_sw128(b + off), bl = umma::desc_k_sw128(b + 16384 + off);
      umma::mma_bf16(tmem, al, bh, idesc, s > 0 ? 1u : 0u);
      umma::mma_bf16(tmem, ah, bl, idesc, 1u);
      umma::mma_bf16(tmem, ah, bh, idesc, 1u);
    }
  }
}

struct TcShared {
  uint8_t* opA;
  uint8_t* opB;
  uint64_t* mbar;
  uint32_t* tslot;
  int* flag;
  uint64_t* stall;  // an mbarrier nothing arrives on (the diagnostic's timed-out wait)
};

__device__ __forceinline__ TcShared tc_layout(unsigned char* raw) {
  TcShared s;
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(raw) + 1023) & ~(uintptr_t)1023);
  s.opA = base;
  s.opB = base + kTcOperandBytes;
  s.mbar = reinterpret_cast<uint64_t*>(base + 2 * kTcOperandBytes);
  s.tslot = reinterpret_cast<uint32_t*>(base + 2 * kTcOperandBytes + 8);
  s.flag = reinterpret_cast<int*>(base + 2 * kTcOperandBytes + 16);
  s.stall = reinterpret_cast<uint64_t*>(base + 2 * kTcOperandBytes + 24);
  return s;
}

__device__ __forceinline__ void tc_setup(const TcShared& sh) {
  const int warp = threadIdx.x >> 5;
  if (warp == 0) {
    umma::tmem_alloc(sh.tslot, kTcTile);
    umma::tmem_relinquish();
  }
  if (threadIdx.x == 32) {
    umma::mbar_init(sh.mbar, 1);
    umma::mbar_init(sh.stall, 1);
    umma::mbar_fence_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
}

// Issue the MMAs for the staged operands and wait for them.  Returns false
// (uniformly) if the bounded wait gave up.
template <int MODE>
__device__ __forceinline__ bool tc_run(const TcShared& sh, uint32_t tmem, bool same_operand, uint32_t parity) {
  umma::fence_proxy_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  if (threadIdx.x == 0) {
    umma::fence_after_sync();
    issue_mmas<MODE>(tmem, sh.opA, same_operand ? sh.opA : sh.opB);
    umma::mma_commit(sh.mbar);
  }
  const bool ok = umma::mbar_wait_bounded(sh.mbar, parity, kTcMaxPolls);
  umma::fence_after_sync();
  if (!ok) *sh.flag = 1;
  __syncthreads();
  return *sh.flag == 0;
}

__device__ __forceinline__ void tc_teardown(const TcShared& sh, uint32_t tmem, bool ok, uint32_t parity) {
  if (!ok) {
    // Give the tensor core one more bounded chance to finish before the
    // accumulator is released.
    umma::mbar_wait_bounded(sh.mbar, parity, kTcMaxPolls);
  }
  umma::fence_before_sync();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) umma::tmem_dealloc(tmem, kTcTile);
}

template <int MODE, bool RAGGED>
__global__ void __launch_bounds__(kTcThreads, 1)
    syrk_tc_kernel(const float* __restrict__ csrc, float* __restrict__ l, Sched sch, int k0,
                   int32_t* __restrict__ info, int jmax, int tiles_i, int tiles_j) {
  extern __shared__ unsigned char tc_raw[];
  const TcShared sh = tc_layout(tc_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) *sh.flag = 0;
  tc_setup(sh);
  const uint32_t tmem = *sh.tslot;
  uint32_t parity = 0;
  bool ok = true;
  const int64_t start = RAGGED ? blockIdx.x : blockIdx.y;
  const int64_t stride = RAGGED ? gridDim.x : gridDim.y;
  int64_t it = start;
  int64_t cur_mat = -1;
  for (; it < sch.count && ok; it += stride) {
    const Target tg = resolve_tile<RAGGED>(sch, it);
    cur_mat = tg.mat;
    const int n = tg.n;
    int ti = tg.ti, tj = tg.tj;
    if (!RAGGED) {
      const int q = blockIdx.x;
      if (tiles_j >= tiles_i) {
        ti = (int)((sqrtf(8.0f * q + 1.0f) - 1.0f) * 0.5f);
        while ((ti + 1) * (ti + 2) / 2 <= q) ++ti;
        while (ti * (ti + 1) / 2 > q) --ti;
        tj = q - ti * (ti + 1) / 2;
      } else {
        // Columns limited to the first tiles_j tile columns: column tj holds
        // tiles ti = tj .. tiles_i-1.
        int rem = q;
        tj = 0;
        while (rem >= tiles_i - tj) {
          rem -= tiles_i - tj;
          ++tj;
        }
        ti = tj + rem;
      }
    }
    const int t0 = k0 + kTcK;
    const int i0 = t0 + ti * kTcTile, j0 = t0 + tj * kTcTile;
    const bool vec = (n & 3) == 0;
    const int jlim = (RAGGED || jmax <= 0) ? n : jmax;
    const size_t moff = tg.off;
    const float* mat = l + moff;
    {
      const int ia = i0 + tid;
      stage_row<MODE>(ia < n ? mat + (size_t)ia * n + k0 : nullptr, vec, sh.opA, tid);
      if (ti != tj) {
        const int jb = j0 + tid;
        stage_row<MODE>(jb < n ? mat + (size_t)jb * n + k0 : nullptr, vec, sh.opB, tid);
      }
    }
    ok = tc_run<MODE>(sh, tmem, ti == tj, parity);
    if (!ok) break;
    parity ^= 1u;
    // Epilogue: row i = i0 + 32*warp + lane, 4 chunks of 32 columns.
    const int i = i0 + 32 * warp + lane;
    const float* crow = csrc + moff + (size_t)i * n;
    float* lrow = l + moff + (size_t)i * n;
#pragma unroll 1
    for (int ch = 0; ch < 4; ++ch) {
      float v[32];
      umma::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(32 * ch), v);
      const int jc = j0 + 32 * ch;
      if (i < n && jc <= i && jc < jlim) {
        if (vec && jc + 31 <= i && jc + 31 < jlim) {
#pragma unroll
          for (int q4 = 0; q4 < 8; ++q4) {
            float4 c = *reinterpret_cast<const float4*>(crow + jc + 4 * q4);
            c.x -= v[4 * q4 + 0];
            c.y -= v[4 * q4 + 1];
            c.z -= v[4 * q4 + 2];
            c.w -= v[4 * q4 + 3];
            *reinterpret_cast<float4*>(lrow + jc + 4 * q4) = c;
          }
        } else {
#pragma unroll
          for (int e = 0; e < 32; ++e)
            if (jc + e <= i && jc + e < jlim) lrow[jc + e] = crow[jc + e] - v[e];
        }
      }
    }
    umma::fence_before_sync();
    __syncthreads();
  }
  // A timed-out wait marks the matrix it was working on with info = -1.
  if (!ok && tid == 0 && info != nullptr && cur_mat >= 0) info[cur_mat] = -1;
  tc_teardown(sh, tmem, ok, parity);
}

// Diagnostic: D[t] = A[t] * B[t]^T for `count` independent 128x64 FP32 tiles,
// through the same staging and MMA code as the trailing update.
template <int MODE>
__global__ void __launch_bounds__(kTcThreads, 1)
    tc_gemm_test_kernel(const float* __restrict__ a, const float* __restrict__ bmat, float* __restrict__ d,
                        int64_t count, int32_t* __restrict__ err, uint32_t stall_polls) {
  extern __shared__ unsigned char tc_raw[];
  const TcShared sh = tc_layout(tc_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) *sh.flag = 0;
  tc_setup(sh);
  const uint32_t tmem = *sh.tslot;
  uint32_t parity = 0;
  bool ok = true;
  for (int64_t t = blockIdx.x; t < count && ok; t += gridDim.x) {
    stage_row<MODE>(a + (size_t)t * kTcTile * kTcK + (size_t)tid * kTcK, true, sh.opA, tid);
    stage_row<MODE>(bmat + (size_t)t * kTcTile * kTcK + (size_t)tid * kTcK, true, sh.opB, tid);
    ok = tc_run<MODE>(sh, tmem, false, parity);
    if (!ok) break;
    parity ^= 1u;
    float* drow = d + (size_t)t * kTcTile * kTcTile + (size_t)(32 * warp + lane) * kTcTile;
#pragma unroll 1
    for (int ch = 0; ch < 4; ++ch) {
      float v[32];
      umma::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(32 * ch), v);
#pragma unroll
      for (int e = 0; e < 32; ++e) drow[32 * ch + e] = v[e];
    }
    umma::fence_before_sync();
    __syncthreads();
    if (stall_polls != 0) {
      // Diagnostic: a bounded wait on a barrier nothing completes runs out
      // and takes the same error path as a real timeout.  The tile's MMAs
      // have completed, so nothing is in flight and no drain is needed.
      const bool got = umma::mbar_wait_bounded(sh.stall, 0u, stall_polls);
      if (!got) *sh.flag = 1;
      __syncthreads();
      if (*sh.flag) {
        if (tid == 0 && err != nullptr) atomicExch(err, B2P_ERR_TIMEOUT);
        tc_teardown(sh, tmem, true, parity);
        return;
      }
    }
  }
  if (!ok && tid == 0 && err != nullptr) atomicExch(err, B2P_ERR_TIMEOUT);
  tc_teardown(sh, tmem, ok, parity);
}

int T_tc(int n, int k0) {
  const int R = n - k0 - kTcK;
  return R <= 0 ? 0 : (R + kTcTile - 1) / kTcTile;
}

int launch_syrk_tc(const float* csrc, float* l, const Sched& sch, bool ragged, int tiles, int k0, int mode,
                   int32_t* info, cudaStream_t s, int jmax) {
  const bool tf32 = (mode & B2P_MODE_MASK) == B2P_MODE_TF32;
  const void* fn;
  int slot;
  if (ragged) {
    fn = tf32 ? (const void*)syrk_tc_kernel<B2P_MODE_TF32, true> : (const void*)syrk_tc_kernel<B2P_MODE_BF16X3, true>;
    slot = tf32 ? kSlotTcR0 : kSlotTcR1;
  } else {
    fn = tf32 ? (const void*)syrk_tc_kernel<B2P_MODE_TF32, false>
              : (const void*)syrk_tc_kernel<B2P_MODE_BF16X3, false>;
    slot = tf32 ? kSlotTc0 : kSlotTc1;
  }
  if (int st = ensure_smem_attr(fn, kTcSmemBytes, slot)) return st;
  dim3 grid;
  int tiles_i = 0, tiles_j = 0;
  if (ragged) {
    if (sch.count <= 0) return B2P_OK;
    grid = dim3((unsigned)std::min<int64_t>(sch.count, 1 << 30), 1);
  } else {
    if (tiles <= 0 || sch.count <= 0) return B2P_OK;
    int tj = tiles;
    if (jmax > 0) tj = std::min(tiles, (jmax - (k0 + kTcK) + kTcTile - 1) / kTcTile);
    if (tj <= 0) return B2P_OK;
    const int count = (tj >= tiles) ? tiles * (tiles + 1) / 2 : tj * tiles - tj * (tj - 1) / 2;
    grid = dim3(count, (unsigned)std::min<int64_t>(sch.count, 65535));
    tiles_i = tiles;
    tiles_j = tj;
  }
  TraceScope ts(kKTrailTc, s);
  if (ragged) {
    if (tf32) syrk_tc_kernel<B2P_MODE_TF32, true><<<grid, kTcThreads, kTcSmemBytes, s>>>(csrc, l, sch, k0, info, jmax, tiles_i, tiles_j);
    else syrk_tc_kernel<B2P_MODE_BF16X3, true><<<grid, kTcThreads, kTcSmemBytes, s>>>(csrc, l, sch, k0, info, jmax, tiles_i, tiles_j);
  } else {
    if (tf32) syrk_tc_kernel<B2P_MODE_TF32, false><<<grid, kTcThreads, kTcSmemBytes, s>>>(csrc, l, sch, k0, info, jmax, tiles_i, tiles_j);
    else syrk_tc_kernel<B2P_MODE_BF16X3, false><<<grid, kTcThreads, kTcSmemBytes, s>>>(csrc, l, sch, k0, info, jmax, tiles_i, tiles_j);
  }
  return check_launch("syrk_tc_kernel");
}

}  // namespace b2p

using namespace b2p;

extern "C" int b2p_debug_tc_gemm(const float* a, const float* bmat, float* d, int64_t count, int mode,
                                 int32_t* err, void* stream) {
  return b2p_debug_tc_gemm_stall(a, bmat, d, count, mode, 0u, err, stream);
}

extern "C" int b2p_debug_tc_gemm_stall(const float* a, const float* bmat, float* d, int64_t count, int mode,
                                       uint32_t stall_polls, int32_t* err, void* stream) {
  if (count < 0 || a == nullptr || bmat == nullptr || d == nullptr)
    return set_error(B2P_ERR_INVALID_ARG, "bad arguments to b2p_debug_tc_gemm");
  if (count == 0) return B2P_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int grid = (int)std::min<int64_t>(count, (int64_t)device_sms());
  const int m = mode & B2P_MODE_MASK;
  if (m == B2P_MODE_TF32) {
    if (int st = ensure_smem_attr((const void*)tc_gemm_test_kernel<B2P_MODE_TF32>, kTcSmemBytes, kSlotTc2)) return st;
    tc_gemm_test_kernel<B2P_MODE_TF32><<<grid, kTcThreads, kTcSmemBytes, s>>>(a, bmat, d, count, err, stall_polls);
  } else if (m == B2P_MODE_BF16X3) {
    if (int st = ensure_smem_attr((const void*)tc_gemm_test_kernel<B2P_MODE_BF16X3>, kTcSmemBytes, kSlotTc3)) return st;
    tc_gemm_test_kernel<B2P_MODE_BF16X3><<<grid, kTcThreads, kTcSmemBytes, s>>>(a, bmat, d, count, err,
                                                                                  stall_polls);
  } else {
    return set_error(B2P_ERR_UNSUPPORTED, "b2p_debug_tc_gemm supports tf32 and bf16x3");
  }
  return check_launch("tc_gemm_test_kernel");
}
