// Host-side declarations shared by the translation units of the library.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/b200_potrf.h"
#include "matrix_list.cuh"
#include "sched.cuh"

namespace b2p {

int set_error(int status, const char* fmt, ...);
int check_launch(const char* what);

// Multiprocessor count of the current device (cached per device).
int device_sms();

// Raises a kernel's dynamic shared-memory limit once per device.
int ensure_smem_attr(const void* func, size_t bytes, int slot);

// Whole-matrix kernels (potrf_small.cu).
int launch_warp32(const float* a, float* l, const MatrixList& ml, int32_t* info, cudaStream_t s);
int launch_cta128(const float* a, float* l, const MatrixList& ml, int32_t* info, cudaStream_t s);

// Blocked right-looking path for n > 128 (potrf_blocked.cu).
size_t blocked_workspace_bytes(int64_t batch, int64_t n, int mode);
int potrf_blocked(const float* a, float* l, int64_t batch, int n, int mode, void* ws,
                  size_t ws_bytes, int32_t* info, cudaStream_t s);

// tcgen05 trailing update, TF32 or BF16x3 (syrk_tc.cu).  Dense: `tiles`
// lower 128x128 tiles per matrix; ragged: one CTA per item of `sch`.
int T_tc(int n, int k0);
int launch_syrk_tc(const float* csrc, float* l, const Sched& sch, bool ragged, int tiles, int k0, int mode,
                   int32_t* info, cudaStream_t s, int jmax = 0);
int ragged_blocked_step(const float* a, float* l, const RaggedTables& t, const RaggedStep& st, int k0, int mode,
                        float* tws, int32_t* info, cudaStream_t s);

// Fused left-looking tensor-core path for 128 < n <= 1024, n % 64 == 0 (potrf_fused.cu).
bool fused_supported(int64_t n, int mode);
size_t fused_workspace_bytes(int64_t batch, int64_t n);
// The pivot guard's device state for one guarded call (all null otherwise):
// the pivot record, (L_jj, A_jj) per pivot (batch x n), written next to L_kk;
// the first failing block column per matrix (-1 for none), which the path
// writes when it finishes a matrix (the audit); the rescue's two grid-barrier
// words, which the path resets.
struct GuardRec {
  float2* piv = nullptr;
  int32_t* state = nullptr;
  int* bar = nullptr;
};
int potrf_fused(const float* a, float* l, int64_t batch, int n, int mode, void* ws, size_t ws_bytes,
                int32_t* info, cudaStream_t s, GuardRec grd = GuardRec());
// Warp-specialized variant (potrf_fused_ws.cu), in clusters of up to 8 CTAs
// per matrix for small batches: same workspace and contract.
int potrf_fused_ws(const float* a, float* l, int64_t batch, int n, int mode, void* ws, size_t ws_bytes,
                   int32_t* info, cudaStream_t s, GuardRec grd = GuardRec());
// Orders and batches the warp-specialized kernel can take (n <= 8192, in
// clusters large enough for TMEM), and the subset the dispatcher and the
// forced-path entry point offer (n <= 1024).
bool fused_ws_fits(int64_t batch, int64_t n, int mode);
bool fused_ws_supported(int64_t batch, int64_t n, int mode);

// Pivot guard (guard.cuh, potrf_rescue.cu).  A guarded call keeps, ahead of
// its path's own workspace, guard_ws_bytes(batch, n): the per-matrix guard
// state (int32: first failing block column, -1 for none; the caller's
// fp32_from array takes its place when given), the pivot record
// (guard_piv_offset) and two barrier words, all filled by the path's
// kernels (GuardRec).  guard_rescue then refactors in FP32 every matrix
// whose pivots failed.
size_t guard_ws_bytes(int64_t batch, int64_t n);
size_t guard_piv_offset(int64_t batch);
int guard_rescue(const float* a, float* l, int64_t batch, int n, int mode, const GuardRec& grd, int32_t* info,
                 cudaStream_t s);

// Multi-CTA left-looking tensor-core path (potrf_split.cu): n % 64 == 0,
// n > 128, tensor modes; two launches per 64-wide block column.
bool split_supported(int64_t n, int mode);
size_t split_workspace_bytes(int64_t batch, int64_t n);
int potrf_split(const float* a, float* l, int64_t batch, int n, int mode, void* ws, size_t ws_bytes,
                int32_t* info, cudaStream_t s, GuardRec grd = GuardRec());

// The n > 128 dispatcher (capi.cu): the path for (batch, n, mode), whether a
// path takes a shape, its workspace, and a launch on an explicit path (n > 128;
// the caller has checked path_supported).
int choose_path(int64_t batch, int64_t n, int mode);
bool path_supported(int path, int64_t batch, int64_t n, int mode);
size_t path_workspace_bytes(int path, int64_t batch, int64_t n, int mode);
int potrf_path(const float* a, float* l, int64_t batch, int n, int mode, int path, void* ws, size_t ws_bytes,
               int32_t* info, cudaStream_t s, GuardRec grd = GuardRec());

// Batched triangular solves with L (trsv.cu): x = L^{-1} b, or L^{-T} b.
constexpr int kTrsvMaxN = 32768;  // x is held in shared memory (n floats)
int launch_trsv(const float* l, const float* b, float* x, int64_t batch, int n, bool trans, cudaStream_t s);

// Batched tensor-core GEMM with structure hints (gemm_tc.cu):
// C = alpha * op1(X) op2(Y) + beta * C per batch item.
struct GemmArgs {
  const float* x;
  const float* y;
  float* c;
  int64_t sx, sy, sc;    // batch strides (elements)
  int ldx, ldy, ldc;
  int m, n, k;
  int trans_x, trans_y;  // op1 = X^T / op2 = Y^T
  int x_tri, y_tri;      // 0 none; 1: op(.) lower (op1: k <= m, op2: k >= n); 2: upper
  int lower_out;         // write only C[i][j], j <= i (square M == N); skip tiles above
  int phi;               // epilogue: zero above the diagonal, halve the diagonal
  float alpha, beta;
  int64_t batch;
  const float* c_in;     // C read from here (null: from c); same layout as c
  // Optional scratch (both or neither, gemm_pack_bytes each): op1(X) and
  // op2(Y) are first packed once into the MMA's tile image, and the product
  // streams the tiles with bulk copies instead of converting every operand
  // row in every output tile.
  uint8_t* pack_x;
  uint8_t* pack_y;
  // Optional second batch dimension (0 = none): item (b, b2) of C starts at
  // c + b sc + b2 sc2 (likewise x, y), b2 < batch2.
  int64_t batch2;
  int64_t sx2, sy2, sc2;
};
int launch_gemm_tc(const GemmArgs& g, int mode, int32_t* err, cudaStream_t s);
// Bytes of one packed operand of `rows` x `kdim` per batch item.
size_t gemm_pack_bytes(int64_t batch, int rows, int kdim);

// Cholesky adjoint (potrf_backward.cu).
size_t backward_workspace_bytes(int64_t batch, int64_t n);
int potrf_backward(const float* l, const float* lbar, float* abar, int64_t batch, int n, int mode, void* ws,
                   size_t ws_bytes, cudaStream_t s);

// Kernel ids reported by the launch trace (b2p_kernel_name).
enum KernelId {
  kKWarp32 = 0,
  kKCta128,
  kKCopyLower,
  kKDiag,
  kKPanel,
  kKTrail,
  kKTrailTc,
  kKSplitStep,
  kKSplitUpdate,
  kKRaggedGather,
  kKBwdGemm,
  kKBwdTrsm,
  kKBwdSym,
  kKFused,
  kKFusedWs,
  kKRaggedScatter,
  kKSplitWide,
  kKTrsv,
  kKGpForward,
  kKGpLbar,
  kKRescue,
  kKCount
};

// RAII bracket: records a start/end CUDA event pair around one launch on
// stream `s` while the trace is enabled; a no-op otherwise.  `units` is the
// launch's algorithmic work: n^3/3 flops per matrix for the kernels that
// factor whole matrices, 8 n^2 bytes per matrix for the n <= 32 kernel, the
// product's flops for update kernels; 0 where none is defined.
class TraceScope {
 public:
  TraceScope(int kernel_id, cudaStream_t s, double units = 0.0);
  ~TraceScope();

 private:
  int slot_;
  cudaStream_t s_;
};

// Slots for ensure_smem_attr (one per kernel that needs > 48 KB).
enum SmemSlot {
  kSlotCta128 = 0,
  kSlotDiag,
  kSlotPanel,
  kSlotTrail,
  kSlotBwd0,
  kSlotBwd1,
  kSlotBwd2,
  kSlotTc0,
  kSlotTc1,
  kSlotTc2,
  kSlotTc3,
  kSlotFused0,
  kSlotFused1,
  kSlotDiagR,
  kSlotTrailR,
  kSlotTcR0,
  kSlotTcR1,
  kSlotFusedWs0,
  kSlotFusedWs1,
  kSlotFusedWs2,
  kSlotFusedWs3,
  kSlotFusedWs4,
  kSlotFusedWs5,
  kSlotFusedWs6,
  kSlotFusedWs7,
  kSlotSplitU0,
  kSlotSplitU1,
  kSlotSplitS0,
  kSlotSplitS1,
  kSlotSplitW0,
  kSlotSplitW1,
  kSlotBwdSmall,
  kSlotDiagF64,
  kSlotBwdBulk0,
  kSlotBwdBulk1,
  kSlotTrsv0,
  kSlotTrsv1,
  kSlotGpForward,
  kSlotRescue,
  kSlotSplitU2,
  kSlotSplitS2,
  kSlotSplitW2,
  kSlotCount
};

}  // namespace b2p
