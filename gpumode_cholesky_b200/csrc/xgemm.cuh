// Panel solve X = P T^T for one 128-row tile in shared memory (FP32 SIMT),
// skipping the zero half of T^T (T = L_kk^{-1} is lower triangular, so
// T^T[m][c] = 0 for m > c).
//
// Layout: PtT[m][r] = P[r][m] (64 x 128, row stride ld) and TT[m][c] = T[c][m]
// (64 x 64, row stride ldt).  Eight warps; lane -> rows 4*lane..4*lane+3;
// warp w -> the column groups {4w..4w+3} (m < 4w+4) and {60-4w..63-4w}
// (m < 64-4w), which balances the triangle at 68 K-steps per warp.  PtT is
// overwritten with X^T (XT[c][r] = X[r][c]) once every warp has finished
// reading it; `bar` synchronises the 256 threads.
#pragma once

namespace b2p {

template <class Bar>
__device__ __forceinline__ void xgemm_tri_inplace(float* PtT, int ld, const float* TT, int ldt, Bar bar) {
  const int lane = threadIdx.x & 31, w = (threadIdx.x >> 5) & 7;
  const int cA = 4 * w, cB = 60 - 4 * w;
  const int mA = 4 * w + 4, mB = 64 - 4 * w;
  float accA[4][4], accB[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) accA[i][j] = accB[i][j] = 0.0f;
#pragma unroll 4
  for (int m = 0; m < mA; ++m) {
    const float4 a = *reinterpret_cast<const float4*>(PtT + m * ld + 4 * lane);
    const float4 ba = *reinterpret_cast<const float4*>(TT + m * ldt + cA);
    const float4 bb = *reinterpret_cast<const float4*>(TT + m * ldt + cB);
    const float a4[4] = {a.x, a.y, a.z, a.w};
    const float b4a[4] = {ba.x, ba.y, ba.z, ba.w};
    const float b4b[4] = {bb.x, bb.y, bb.z, bb.w};
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        accA[i][j] = fmaf(a4[i], b4a[j], accA[i][j]);
        accB[i][j] = fmaf(a4[i], b4b[j], accB[i][j]);
      }
  }
#pragma unroll 4
  for (int m = mA; m < mB; ++m) {
    const float4 a = *reinterpret_cast<const float4*>(PtT + m * ld + 4 * lane);
    const float4 bb = *reinterpret_cast<const float4*>(TT + m * ldt + cB);
    const float a4[4] = {a.x, a.y, a.z, a.w};
    const float b4b[4] = {bb.x, bb.y, bb.z, bb.w};
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) accB[i][j] = fmaf(a4[i], b4b[j], accB[i][j]);
  }
  bar();
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    *reinterpret_cast<float4*>(PtT + (cA + j) * ld + 4 * lane) =
        make_float4(accA[0][j], accA[1][j], accA[2][j], accA[3][j]);
    *reinterpret_cast<float4*>(PtT + (cB + j) * ld + 4 * lane) =
        make_float4(accB[0][j], accB[1][j], accB[2][j], accB[3][j]);
  }
  bar();
}

}  // namespace b2p
