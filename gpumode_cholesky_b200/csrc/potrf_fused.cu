// Fused left-looking factorization on the tensor cores: one CTA per matrix.
//
// For 128 < n <= 1024 with n a multiple of 64 and a tensor mode (TF32 or
// BF16x3), a persistent CTA factors whole matrices.  Block column k
// (k0 = 64k) is produced in three phases:
//
//   1. update   D = L[k0:n, 0:k0] * L[k0:k0+64, 0:k0]^T on tcgen05, one
//               128x64 FP32 accumulator in TMEM per 128-row tile.  The
//               operands are the earlier panels' tensor-core copies in the
//               workspace, already in the 128B-swizzled K-major layout, so a
//               single thread streams them into shared memory with bulk
//               copies (cp.async.bulk, two stages) and issues the MMAs;
//   2. panel    P = A[k0:n, k0:k0+64] - D (A read from HBM exactly once);
//               the top 64x64 block is factored and inverted in shared memory
//               (diag64.cuh, warps 0-3) while warps 4-7 form P of the later
//               row tiles and park it in TMEM in place of D; the rows below
//               are solved as X = P T^T (FP32 SIMT, T = L_kk^{-1});
//   3. output   L_kk, X and the zero strip above go to L (written once);
//               X's tensor-core copy (BF16 hi and lo, or TF32 halves) goes to
//               the workspace for the updates of later block columns.
//
// Compared with the right-looking schedule, the trailing matrix is never
// re-read and re-written through HBM, and the update accumulates in TMEM.
// All mbarrier waits are bounded; a timeout marks the matrix with info = -1.
//
// The reference's left-looking paths run the same schedule through cuBLAS
// and cuSOLVER (submission.py:3319-3409 _left_looking_large, 3606-3676,
// 5152-5196 e62 with a resident diagonal block and inverse panel multiply).
#include <algorithm>

#include "diag64.cuh"
#include "guard.cuh"
#include "launch.h"
#include "panel_copy.cuh"
#include "umma.cuh"
#include "xgemm.cuh"

namespace b2p {

constexpr int kFThreads = 256;
constexpr int kFB = 64;     // block column width = K of each MMA chunk
constexpr int kFM = 128;    // rows per M tile
constexpr int kFPtLd = 132; // P^T in shared memory: [64][kFPtLd]
constexpr uint32_t kFPolls = 1u << 24;

// Phase-1 staging: 2 stages x (A: 2 regions x 16 KB, B: 2 regions x 8 KB).
constexpr uint32_t kFStageA = 32768;
constexpr uint32_t kFStageB = 16384;
constexpr uint32_t kFStage = kFStageA + kFStageB;
constexpr uint32_t kFStaging = 2 * kFStage;
// Phase-2 layout in the same region.  The workspace holds the panel copies
// (panel_copy.cuh).
constexpr uint32_t kFPtOff = ((uint32_t)sizeof(Diag64Smem) + 1023u) & ~1023u;
constexpr uint32_t kFPhase2 = kFPtOff + 64 * kFPtLd * 4;
constexpr uint32_t kFUnion = kFStaging > kFPhase2 ? kFStaging : kFPhase2;
constexpr uint32_t kFZeroOff = kFUnion + 128;  // zeros, source of the strip's bulk stores
constexpr uint32_t kFZeroBytes = 4096;           // >= 4 (n - 64) bytes for n <= 1024
constexpr uint32_t kFSmemBytes = kFZeroOff + kFZeroBytes + 1024;
constexpr uint32_t kFSmemOneCta = 120 * 1024;  // forces one CTA per SM (512 TMEM columns)

constexpr uint32_t kNoTmem = 0xffffffffu;
constexpr int kFStripThread = 128;  // warp 4, free during the diagonal engine

// One thread's 32 values of P = A - D for row r0 + rl (rl < 0: beyond the
// matrix, zeros) and columns k0 + 32 h .. + 31, D from the TMEM columns at
// dcol (lanes of warp quarter w4; kNoTmem: no update yet).  The TMEM load is
// warp-collective, so every lane of the warp calls this.
__device__ __forceinline__ void p_form(float (&p)[32], const float* A, int n, int k0, int r0, int rl, int w4, int h,
                                       uint32_t dcol) {
  float d[32];
  if (dcol != kNoTmem) {
    umma::tmem_ld32(dcol + ((uint32_t)(32 * w4) << 16), d);
  } else {
#pragma unroll
    for (int q = 0; q < 32; ++q) d[q] = 0.0f;
  }
  if (rl >= 0) {
    const float4* src = reinterpret_cast<const float4*>(A + (size_t)(r0 + rl) * n + k0 + 32 * h);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float4 v = src[q];
      p[4 * q + 0] = v.x - d[4 * q + 0];
      p[4 * q + 1] = v.y - d[4 * q + 1];
      p[4 * q + 2] = v.z - d[4 * q + 2];
      p[4 * q + 3] = v.w - d[4 * q + 3];
    }
  } else {
#pragma unroll
    for (int q = 0; q < 32; ++q) p[q] = 0.0f;
  }
}

template <int MODE>
__global__ void __launch_bounds__(kFThreads, 2)
    potrf_fused_kernel(const float* __restrict__ a, float* __restrict__ l, int64_t batch, int n,
                       uint8_t* __restrict__ ws, uint32_t tmem_cols, int32_t* __restrict__ info,
                       GuardRec grd) {
  __shared__ int s_gmin;
  // The rescue's grid barrier starts from zero (it runs after this kernel).
  if (grd.bar != nullptr && blockIdx.x == 0 && threadIdx.x == 0) grd.bar[0] = grd.bar[1] = 0;
  extern __shared__ unsigned char fraw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(fraw) + 1023) & ~(uintptr_t)1023);
  Diag64Smem& dg = *reinterpret_cast<Diag64Smem*>(sm);
  float* PtT = reinterpret_cast<float*>(sm + kFPtOff);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + kFUnion);  // [2]
  uint64_t* empty = full + 2;                                   // [2]
  uint64_t* done = full + 4;                                    // [1]
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kFUnion + 48);
  int* flag = reinterpret_cast<int*>(sm + kFUnion + 56);
  int* badp = flag + 1;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int N = n / kFB;
  const size_t rbytes = panel_copy_region_bytes(n);

  if (tid == 0) *flag = 0;
  for (uint32_t e = tid; e < kFZeroBytes / 16; e += kFThreads)
    reinterpret_cast<float4*>(sm + kFZeroOff)[e] = make_float4(0.f, 0.f, 0.f, 0.f);
  umma::fence_proxy_async_smem();  // the zeros are read by bulk stores
  if (warp == 0) {
    umma::tmem_alloc(tslot, tmem_cols);
    umma::tmem_relinquish();
  }
  if (tid == 32) {
    for (int i = 0; i < 5; ++i) umma::mbar_init(full + i, 1);
    umma::mbar_fence_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;

  // mbarrier phase bookkeeping (thread 0 drives full/empty; all wait on done)
  uint32_t ph_full[2] = {0u, 0u};
  uint32_t n_empty[2] = {0u, 0u};
  uint32_t ph_done = 0u;
  bool ok = true;

  int64_t b = blockIdx.x;
  for (; b < batch && ok; b += gridDim.x) {
    const float* A = a + (size_t)b * n * n;
    float* L = l + (size_t)b * n * n;
    uint8_t* W0 = ws + (size_t)b * 2 * rbytes;
    uint8_t* W1 = W0 + rbytes;
    if (tid == 0) *badp = -1;

    for (int k = 0; k < N; ++k) {
      const int k0 = k * kFB;
      const int mtiles = (n - k0 + kFM - 1) / kFM;
      // ---------------- phase 1: left-looking update into TMEM -------------
      if (k > 0) {
        if (tid == 0) {
          const int iters = mtiles * k;
          auto load = [&](int i, int s) {
            const int mt = i / k, kc = i - (i / k) * k;
            const int r0 = k0 + mt * kFM;
            const uint32_t abytes = (uint32_t)min(kFM, n - r0) * 128u;
            const size_t aoff = panel_copy_row_byte(N, kc, r0);
            const size_t boff = panel_copy_row_byte(N, kc, k0);
            uint8_t* st = sm + s * kFStage;
            umma::mbar_arrive_expect_tx(full + s, 2 * abytes + 2 * 8192u);
            umma::bulk_g2s(st, W0 + aoff, abytes, full + s);
            umma::bulk_g2s(st + 16384, W1 + aoff, abytes, full + s);
            umma::bulk_g2s(st + kFStageA, W0 + boff, 8192u, full + s);
            umma::bulk_g2s(st + kFStageA + 8192, W1 + boff, 8192u, full + s);
          };
          int loaded = 0;
          load(0, 0);
          ++loaded;
          if (iters > 1) {
            load(1, 1);
            ++loaded;
          }
          int waited = 0;
          for (int i = 0; i < iters; ++i) {
            const int s = i & 1;
            if (!umma::mbar_wait_bounded(full + s, ph_full[s], kFPolls)) {
              ok = false;
              break;
            }
            ph_full[s] ^= 1u;
            ++waited;
            umma::fence_after_sync();
            const int mt = i / k, kc = i - (i / k) * k;
            const uint32_t st = umma::smem_u32(sm + s * kFStage);
            panel_copy_mmas<MODE>(tmem + (uint32_t)(kFB * mt), st, st + kFStageA, kc > 0);
            umma::mma_commit(empty + s);
            ++n_empty[s];
            if (i + 2 < iters) {
              if (!umma::mbar_wait_bounded(empty + s, (n_empty[s] - 1u) & 1u, kFPolls)) {
                ok = false;
                break;
              }
              load(i + 2, s);
              ++loaded;
            }
          }
          if (ok) {
            // Retire the last commits on each stage so that every barrier
            // phase is complete at the step boundary.
            for (int s = 0; s < 2; ++s) {
              const int last = iters - 1 - ((iters - 1 - s) & 1);  // last iteration using stage s
              if (last >= 0 && last + 2 >= iters) {
                if (!umma::mbar_wait_bounded(empty + s, (n_empty[s] - 1u) & 1u, kFPolls)) ok = false;
              }
            }
          }
          if (!ok) {
            // Let the copies still in flight land before anything else runs.
            for (int i = waited; i < loaded; ++i) {
              const int s = i & 1;
              if (umma::mbar_wait_bounded(full + s, ph_full[s], kFPolls)) ph_full[s] ^= 1u;
            }
            *flag = 1;
          }
          umma::mma_commit(done);
        }
        const bool got = umma::mbar_wait_bounded(done, ph_done, kFPolls);
        ph_done ^= 1u;
        umma::fence_after_sync();
        if (!got) *flag = 1;
        __syncthreads();
        if (*flag) {
          ok = false;
          break;
        }
      }
      // ---------------- phases 2-3: panel, diagonal block, output ----------
      for (int mt = 0; mt < mtiles; ++mt) {
        const int r0 = k0 + mt * kFM;
        const int vr = min(kFM, n - r0);
        {
          const int w4 = warp & 3, h = warp >> 2;
          const int rl = 32 * w4 + lane;
          float p[32];
          if (mt > 0) {
            // Formed during the diagonal phase (below) and kept in TMEM.
            umma::tmem_ld32(tmem + ((uint32_t)(32 * w4) << 16) + (uint32_t)(kFB * mt + 32 * h), p);
          } else {
            p_form(p, A, n, k0, r0, rl < vr ? rl : -1, w4, h, k > 0 ? tmem + (uint32_t)(32 * h) : kNoTmem);
          }
#pragma unroll
          for (int q = 0; q < 32; ++q) PtT[(32 * h + q) * kFPtLd + rl] = p[q];
          if (mt == 0 && rl < 64) {
#pragma unroll
            for (int q = 0; q < 32; ++q) dg.S[rl * kD64Ld + 32 * h + q] = p[q];
          }
        }
        umma::fence_before_sync();
        __syncthreads();
        if (mt == 0) {
          // L_kk and T^T (T = L_kk^{-1}, in dg.T) from the pipelined engine
          // on warps 0-3.  Meanwhile warps 4-7 form P = A - D of the later
          // row tiles (their loads of A hide behind the diagonal engine) and
          // park it in place of D in TMEM, each warp its lane quarter.
          if (warp < 4) {
            diag64_factor_invert(dg, NamedBarrier1<kD64Threads>());
          } else {
            // Zero strip right of the diagonal block: one bulk store per row
            // from the zero buffer, issued by one thread and left to run.
            const uint32_t strip = 4u * (uint32_t)(n - k0 - kFB);
            if (tid == kFStripThread && strip > 0) {
              for (int r = 0; r < 64; ++r)
                umma::bulk_s2g(L + (size_t)(k0 + r) * n + k0 + kFB, sm + kFZeroOff, strip);
              umma::bulk_commit();
            }
            const int w4 = warp & 3;
            for (int mt2 = 1; mt2 < mtiles; ++mt2) {
              const int r2 = k0 + mt2 * kFM, v2 = min(kFM, n - r2);
              const int rl = 32 * w4 + lane;
#pragma unroll 1
              for (int h = 0; h < 2; ++h) {
                const uint32_t col = tmem + (uint32_t)(kFB * mt2 + 32 * h);
                float p[32];
                p_form(p, A, n, k0, r2, rl < v2 ? rl : -1, w4, h, k > 0 ? col : kNoTmem);
                umma::tmem_st32(col + ((uint32_t)(32 * w4) << 16), p);
              }
            }
            umma::tmem_wait_st();
          }
          umma::fence_before_sync();
          __syncthreads();
          umma::fence_after_sync();
          const int bad = diag64_status(dg);
          if (bad == kDiagTimeout) {
            ok = false;
            break;
          }
          // The pivot record of a guarded call: (L_jj, A_jj).
          if (grd.piv != nullptr && tid < 64)
            grd.piv[(size_t)b * n + k0 + tid] =
                make_float2(dg.S[tid * kD64Ld + tid], __ldg(A + (size_t)(k0 + tid) * (n + 1)));
          if (tid == 0 && bad >= 0 && *badp < 0) *badp = k0 + bad;
          // L_kk (zeros above its diagonal), row-major, float4.
          for (int e = tid; e < 64 * 16; e += kFThreads) {
            const int r = e >> 4, c = (e & 15) * 4;
            const float* srow = dg.S + r * kD64Ld + c;
            float4 v = make_float4(c <= r ? srow[0] : 0.f, c + 1 <= r ? srow[1] : 0.f, c + 2 <= r ? srow[2] : 0.f,
                                   c + 3 <= r ? srow[3] : 0.f);
            *reinterpret_cast<float4*>(L + (size_t)(k0 + r) * n + k0 + c) = v;
          }
          __syncthreads();
        }
        // X = P T^T for the rows below the diagonal block (triangle skipped),
        // then L and the tensor-core copy from X^T.
        xgemm_tri_inplace(PtT, kFPtLd, dg.T, kD64Ld, CtaBarrier());
        for (int item = tid; item < kFM * 8; item += kFThreads) {
          const int rl = item & (kFM - 1), c = item >> 7;
          if (rl >= vr || (mt == 0 && rl < 64)) continue;
          float v[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) v[j] = PtT[(8 * c + j) * kFPtLd + rl];
          const int rg = r0 + rl;
          float4* dst = reinterpret_cast<float4*>(L + (size_t)rg * n + k0 + 8 * c);
          dst[0] = make_float4(v[0], v[1], v[2], v[3]);
          dst[1] = make_float4(v[4], v[5], v[6], v[7]);
          if (k + 1 < N) panel_copy_store<MODE>(W0, W1, N, k, rg, c, v);
        }
        __syncthreads();
      }
      if (!ok) break;
      // Workspace and shared-memory writes above must be ordered before the
      // next step's bulk copies and tensor-core reads (async proxy).
      umma::fence_proxy_async_all();
      umma::fence_before_sync();
      __syncthreads();
      umma::fence_after_sync();
    }
    if (tid == 0 && info != nullptr) info[b] = ok ? (*badp < 0 ? 0 : *badp + 1) : -1;
    if (grd.state != nullptr) {
      const int f = ok ? guard_audit_matrix<kFThreads>(grd.piv + (size_t)b * n, n, MODE, &s_gmin, tid, CtaBarrier())
                       : -1;
      if (tid == 0) grd.state[b] = f;
    }
  }
  // Matrices this CTA did not reach (a bounded wait gave up) are not rescued.
  if (grd.state != nullptr && tid == 0)
    for (; b < batch; b += gridDim.x) grd.state[b] = -1;
  // The strip's bulk stores read the zero buffer until they complete.
  if (tid == kFStripThread) umma::bulk_wait_all();
  // Release TMEM after a last bounded chance for outstanding MMAs.
  if (!ok) {
    umma::mbar_wait_bounded(done, ph_done, kFPolls);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, tmem_cols);
}

// The workspace pointer is rounded up to 1024 bytes inside, hence the slack.
size_t fused_workspace_bytes(int64_t batch, int64_t n) {
  return (size_t)batch * 2 * panel_copy_region_bytes((int)n) + 1024;
}

bool fused_supported(int64_t n, int mode) {
  const int m = mode & B2P_MODE_MASK;
  return (m == B2P_MODE_TF32 || m == B2P_MODE_BF16X3) && !(mode & B2P_FLAG_FP64_DIAG) && n > 128 && n <= 1024 &&
         (n % kFB) == 0;
}

int potrf_fused(const float* a, float* l, int64_t batch, int n, int mode, void* ws, size_t ws_bytes,
                int32_t* info, cudaStream_t s, GuardRec grd) {
  const size_t need = fused_workspace_bytes(batch, n);
  if (ws == nullptr || ws_bytes < need)
    return set_error(B2P_ERR_WORKSPACE, "workspace of %zu bytes required, %zu given", need, ws_bytes);
  uint8_t* wsa = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(ws) + 1023) & ~(uintptr_t)1023);
  const bool two = n <= 512;
  const uint32_t cols = two ? 256u : 512u;
  const size_t smem = two ? kFSmemBytes : std::max<size_t>(kFSmemBytes, kFSmemOneCta);
  const int sms = device_sms();
  const int grid = (int)std::min<int64_t>(batch, (int64_t)sms * (two ? 2 : 1));
  TraceScope ts(kKFused, s, (double)batch * n * n * n / 3.0);
  if ((mode & B2P_MODE_MASK) == B2P_MODE_TF32) {
    if (int st = ensure_smem_attr((const void*)potrf_fused_kernel<B2P_MODE_TF32>, smem, kSlotFused0)) return st;
    potrf_fused_kernel<B2P_MODE_TF32><<<grid, kFThreads, smem, s>>>(a, l, batch, n, wsa, cols, info, grd);
  } else {
    if (int st = ensure_smem_attr((const void*)potrf_fused_kernel<B2P_MODE_BF16X3>, smem, kSlotFused1)) return st;
    potrf_fused_kernel<B2P_MODE_BF16X3><<<grid, kFThreads, smem, s>>>(a, l, batch, n, wsa, cols, info, grd);
  }
  return check_launch("potrf_fused_kernel");
}

}  // namespace b2p
