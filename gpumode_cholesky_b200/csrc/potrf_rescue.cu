// FP32 rescue of the pivot guard (guard.cuh).
//
// The tensor-mode paths (potrf_fused.cu, potrf_fused_ws.cu, potrf_split.cu)
// audit each matrix when they finish it (guard_audit_matrix over the
// (L_jj, A_jj) pairs they recorded next to writing L_kk), write its guard
// state (the first failing block column, or -1) and reset this kernel's grid
// barrier.  Right after, on the same stream, potrf_rescue_kernel reads the
// guard state and returns when no matrix failed (the usual case, one short
// launch); otherwise it refactors every failing matrix from its first column
// in plain FP32 and overwrites its L and info; the others are not touched.
//
// Rescue schedule: one cooperative launch, one CTA per SM (all CTAs
// resident at once), left-looking by 64-wide block columns.  In column k the jobs are
// (flagged matrix, 128-row chunk of the rows below the diagonal block); each
// job recomputes the diagonal block's P = A - L[:, 0:k0] L[k-block, 0:k0]^T
// in FP32 (guard_row_p), factors it with the diagonal engine (diag64_factor),
// then computes and solves its own 128 rows (one row per thread, the same
// forward substitution as the split path).  A bounded grid barrier separates
// the columns, because column k reads the rows other CTAs wrote in earlier
// columns.  All accumulation is in FP32 in a fixed order, so the result does
// not depend on which CTA ran which job.
//
// Matrices are taken in rounds of at most kRList, in order of index.
#include "diag64.cuh"
#include "guard.cuh"
#include "launch.h"

namespace b2p {

constexpr int kRThreads = 128;
constexpr int kRList = 2048;   // flagged matrices per round
constexpr int kRRowLd = 68;    // floats per thread's P row
constexpr uint32_t kRPolls = 1u << 24;

constexpr uint32_t kRDiagOff = 0;
constexpr uint32_t kRStageOff = (((uint32_t)sizeof(Diag64Smem) + 127u) & ~127u);
constexpr uint32_t kRRowsOff = kRStageOff + kGuardStageFloats * 4;
constexpr uint32_t kRListOff = kRRowsOff + kRThreads * kRRowLd * 4;
constexpr uint32_t kRMiscOff = kRListOff + kRList * 8;
constexpr uint32_t kRSmemBytes = kRMiscOff + 64 + 128;

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }
size_t guard_piv_offset(int64_t batch) { return align256((size_t)batch * sizeof(int32_t)); }
size_t guard_ws_bytes(int64_t batch, int64_t n) {
  return guard_piv_offset(batch) + align256((size_t)batch * (size_t)n * sizeof(float2)) + 256;
}

// Grid-wide barrier over the launch's CTAs: bar[0] counts arrivals, bar[1]
// is the generation.  Bounded: false when the generation did not move.
__device__ __forceinline__ bool rescue_grid_sync(int* bar, int* s_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile int* gen = bar + 1;
    const int g = *gen;
    __threadfence();  // this CTA's L writes before its arrival
    int ok = 1;
    if (atomicAdd(bar, 1) == (int)gridDim.x - 1) {
      atomicExch(bar, 0);
      __threadfence();
      atomicAdd(bar + 1, 1);
    } else {
      ok = 0;
      for (uint32_t i = 0; i < kRPolls; ++i) {
        if (*gen != g) {
          ok = 1;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();  // other CTAs' writes before this CTA's next reads
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

__global__ void __launch_bounds__(kRThreads, 1)
    potrf_rescue_kernel(const float* __restrict__ a, float* __restrict__ l, int64_t batch, int n, int mode,
                        int32_t* __restrict__ gstate, int* bar, int32_t* __restrict__ info) {
  extern __shared__ unsigned char rraw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(rraw) + 127) & ~(uintptr_t)127);
  Diag64Smem& dg = *reinterpret_cast<Diag64Smem*>(sm + kRDiagOff);
  float* stage = reinterpret_cast<float*>(sm + kRStageOff);
  float* rows = reinterpret_cast<float*>(sm + kRRowsOff);
  int64_t* list = reinterpret_cast<int64_t*>(sm + kRListOff);
  int* misc = reinterpret_cast<int*>(sm + kRMiscOff);  // [0] list size, [1] barrier verdict, [4..7] warp counts
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int N = n / 64;
  const size_t n2 = (size_t)n * n;

  // 2. Fast exit: nothing flagged (the usual case).
  bool any = false;
  for (int64_t b = tid; b < batch; b += kRThreads) any |= __ldcg(gstate + b) >= 0;
  if (!__syncthreads_or(any)) return;

  int64_t scan = 0;
  while (scan < batch) {
    // Ordered compaction of the next flagged matrices into the list.
    if (tid == 0) misc[0] = 0;
    __syncthreads();
    while (scan < batch && misc[0] + kRThreads <= kRList) {
      const int64_t b = scan + tid;
      const bool f = b < batch && __ldcg(gstate + b) >= 0;
      const unsigned m = __ballot_sync(0xffffffffu, f);
      if (lane == 0) misc[4 + warp] = __popc(m);
      __syncthreads();
      int base = misc[0];
      for (int w = 0; w < warp; ++w) base += misc[4 + w];
      if (f) list[base + __popc(m & ((1u << lane) - 1u))] = b;
      int total = misc[0];
      for (int w = 0; w < kRThreads / 32; ++w) total += misc[4 + w];
      __syncthreads();
      if (tid == 0) misc[0] = total;
      __syncthreads();
      scan += kRThreads;
    }
    const int nf = misc[0];
    if (nf == 0) continue;  // (only when the scan has reached the end)

    for (int k = 0; k < N; ++k) {
      const int k0 = 64 * k;
      const int chunks = (n - k0 - 64 + kRThreads - 1) / kRThreads;
      const int G = chunks > 0 ? chunks : 1;
      const int64_t jobs = (int64_t)nf * G;
      for (int64_t job = blockIdx.x; job < jobs; job += gridDim.x) {
        const int f = (int)(job / G), q = (int)(job - (int64_t)f * G);
        const int64_t b = list[f];
        const float* A = a + (size_t)b * n2;
        float* L = l + (size_t)b * n2;
        // Diagonal block: P_kk in FP32 (rows k0 .. k0 + 63, one per thread).
        for (int h = 0; h < 2; ++h)
          guard_row_p<kRThreads>(L, A, n, k0, tid < 64 ? (int64_t)(k0 + tid) : -1, 32 * h,
                                 dg.S + (tid & 63) * kD64Ld + 32 * h, stage, tid, CtaBarrier());
        __syncthreads();
        const int bad = diag64_factor(dg);
        if (q == 0) {
          for (int e = tid; e < 64 * 16; e += kRThreads) {
            const int r = e >> 4, c = (e & 15) * 4;
            const float* srow = dg.S + r * kD64Ld + c;
            *reinterpret_cast<float4*>(L + (size_t)(k0 + r) * n + k0 + c) =
                make_float4(c <= r ? srow[0] : 0.f, c + 1 <= r ? srow[1] : 0.f, c + 2 <= r ? srow[2] : 0.f,
                            c + 3 <= r ? srow[3] : 0.f);
          }
          if (tid == 0 && info != nullptr) {
            if (bad == kDiagTimeout)
              info[b] = -1;
            else if (k == 0)
              info[b] = bad >= 0 ? bad + 1 : 0;
            else if (bad >= 0 && info[b] == 0)
              info[b] = k0 + bad + 1;
          }
        }
        // Zeros right of the diagonal block: rows q, q + G, ... of it.
        for (int r = q; r < 64; r += G)
          for (int c = k0 + 64 + 4 * tid; c < n; c += 4 * kRThreads)
            *reinterpret_cast<float4*>(L + (size_t)(k0 + r) * n + c) = make_float4(0.f, 0.f, 0.f, 0.f);
        // The chunk's rows: P in FP32, then X L_kk^T = P.
        if (chunks > 0) {
          const int r = k0 + 64 + q * kRThreads + tid;
          float* xs = rows + tid * kRRowLd;
          for (int h = 0; h < 2; ++h)
            guard_row_p<kRThreads>(L, A, n, k0, r < n ? (int64_t)r : -1, 32 * h, xs + 32 * h, stage, tid,
                                   CtaBarrier());
          if (r < n) {
            float x[64];
#pragma unroll
            for (int c = 0; c < 64; ++c) x[c] = xs[c];
            panel_solve64(x, dg);
            float4* dst = reinterpret_cast<float4*>(L + (size_t)r * n + k0);
#pragma unroll
            for (int c4 = 0; c4 < 16; ++c4)
              dst[c4] = make_float4(x[4 * c4], x[4 * c4 + 1], x[4 * c4 + 2], x[4 * c4 + 3]);
          }
        }
        __syncthreads();  // dg, the stage and the rows are reused by the next job
      }
      if (!rescue_grid_sync(bar, misc + 1)) {
        // A CTA did not arrive: mark this round's matrices incomplete.
        for (int f = tid; f < nf; f += kRThreads)
          if (info != nullptr) info[list[f]] = -1;
        return;
      }
    }
  }
}

int guard_rescue(const float* a, float* l, int64_t batch, int n, int mode, const GuardRec& grd, int32_t* info,
                 cudaStream_t s) {
  if (batch == 0) return B2P_OK;
  if (int st = ensure_smem_attr((const void*)potrf_rescue_kernel, kRSmemBytes, kSlotRescue)) return st;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)device_sms(), 1, 1);
  cfg.blockDim = dim3(kRThreads, 1, 1);
  cfg.dynamicSmemBytes = kRSmemBytes;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  TraceScope ts(kKRescue, s);
  const cudaError_t e =
      cudaLaunchKernelEx(&cfg, potrf_rescue_kernel, a, l, batch, n, mode, grd.state, grd.bar, info);
  if (e != cudaSuccess) return set_error(B2P_ERR_CUDA, "potrf_rescue_kernel: %s", cudaGetErrorString(e));
  return B2P_OK;
}

}  // namespace b2p
