// Shared helpers for the B200 potrf kernels (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/b200_potrf.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "this library targets sm_100a (B200) only"
#endif

namespace b2p {

constexpr unsigned kFullMask = 0xffffffffu;

// Records a detail message for b2p_last_error() and returns `status`.
int set_error(int status, const char* fmt, ...);

// Returns B2P_ERR_CUDA with a message if the last launch failed.
int check_launch(const char* what);

// Reciprocal square root refined by one Newton-Raphson step
// y <- y * (1.5 - 0.5 * d * y * y), starting from the hardware estimate.
// One step brings the MUFU estimate to about one ulp.  A non-positive or NaN
// pivot yields NaN/Inf, which the factorization propagates.
__device__ __forceinline__ float rsqrt_refined(float d) {
  float y = rsqrtf(d);
  float h = 0.5f * d;
  float t = fmaf(-h * y, y, 0.5f);  // 0.5 - 0.5*d*y^2
  return fmaf(y, t, y);             // y + y*(0.5 - 0.5*d*y^2)
}

__device__ __forceinline__ bool pivot_bad(float d) { return !(d > 0.0f); }

// 64-bit element offset of matrix `b` in a contiguous batch of n x n matrices.
__device__ __forceinline__ int64_t mat_offset(int64_t b, int n) { return b * (int64_t)n * n; }

}  // namespace b2p
