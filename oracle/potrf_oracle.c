/*
 * CPU oracle for the batched Cholesky hot path.  TEST INFRASTRUCTURE ONLY:
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg call it as
 * the checker; the library never links or calls it.
 *
 * It restates what the reference computes on this path:
 *   ref_kernel(data) = torch.linalg.cholesky_ex(data, check_errors=False).L
 *     (reference/reference.py:129-130), i.e. LAPACK potrf on CPU: the lower
 *     Cholesky factor by the column-oriented (left-looking) algorithm of
 *     LAPACK's xPOTF2 -- for column j, L[j][j] = sqrt(A[j][j] - sum_k L[j][k]^2)
 *     and L[i][j] = (A[i][j] - sum_k L[i][k] L[j][k]) / L[j][j].  On the first
 *     non-positive pivot LAPACK stops and reports info = j+1.
 *   check_implementation (reference/reference.py:137-188): L1 (max column
 *     sum) norms of triu(L,1), of L L^T - A and of A.
 * plus the Cholesky adjoint used to check the library's backward
 * (Abar = 1/2 (S + S^T), S = L^{-T} Phi(L^T Lbar) L^{-1}), which has no
 * counterpart in the reference.
 *
 * Build: `make -C oracle` (gcc only; output oracle/liboracle_potrf.so).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* FP64 factorization; a and l may alias.  info[b] = 0 or first bad pivot + 1.
 * After a failure the remaining columns are left as NaN (the library's
 * convention; LAPACK leaves them unfactored). */
int oracle_potrf_f64(const double* a, double* l, int64_t batch, int64_t n, int32_t* info) {
  for (int64_t b = 0; b < batch; ++b) {
    const double* A = a + b * n * n;
    double* L = l + b * n * n;
    if (A != L) memcpy(L, A, sizeof(double) * (size_t)(n * n));
    int32_t bad = 0;
    for (int64_t j = 0; j < n; ++j) {
      double d = L[j * n + j];
      for (int64_t k = 0; k < j; ++k) d -= L[j * n + k] * L[j * n + k];
      if (!(d > 0.0) && bad == 0) bad = (int32_t)(j + 1);
      const double ljj = sqrt(d);
      L[j * n + j] = ljj;
      for (int64_t i = j + 1; i < n; ++i) {
        double s = L[i * n + j];
        for (int64_t k = 0; k < j; ++k) s -= L[i * n + k] * L[j * n + k];
        L[i * n + j] = s / ljj;
      }
    }
    for (int64_t i = 0; i < n; ++i)
      for (int64_t j = i + 1; j < n; ++j) L[i * n + j] = 0.0;
    if (bad) {
      const int64_t j0 = bad - 1;
      for (int64_t i = 0; i < n; ++i)
        for (int64_t j = j0; j <= i; ++j) L[i * n + j] = NAN;
    }
    if (info) info[b] = bad;
  }
  return 0;
}

/* Same algorithm in FP32 arithmetic (the reference's dtype). */
int oracle_potrf_f32(const float* a, float* l, int64_t batch, int64_t n, int32_t* info) {
  for (int64_t b = 0; b < batch; ++b) {
    const float* A = a + b * n * n;
    float* L = l + b * n * n;
    if (A != L) memcpy(L, A, sizeof(float) * (size_t)(n * n));
    int32_t bad = 0;
    for (int64_t j = 0; j < n; ++j) {
      float d = L[j * n + j];
      for (int64_t k = 0; k < j; ++k) d -= L[j * n + k] * L[j * n + k];
      if (!(d > 0.0f) && bad == 0) bad = (int32_t)(j + 1);
      const float ljj = sqrtf(d);
      L[j * n + j] = ljj;
      for (int64_t i = j + 1; i < n; ++i) {
        float s = L[i * n + j];
        for (int64_t k = 0; k < j; ++k) s -= L[i * n + k] * L[j * n + k];
        L[i * n + j] = s / ljj;
      }
    }
    for (int64_t i = 0; i < n; ++i)
      for (int64_t j = i + 1; j < n; ++j) L[i * n + j] = 0.0f;
    if (bad) {
      const int64_t j0 = bad - 1;
      for (int64_t i = 0; i < n; ++i)
        for (int64_t j = j0; j <= i; ++j) L[i * n + j] = NAN;
    }
    if (info) info[b] = bad;
  }
  return 0;
}

/* Per matrix, in FP64: out[4*b + 0] = ||A||_1, 1 = ||triu(L,1)||_1,
 * 2 = ||L L^T - A||_1, 3 = ||L L^T - A||_F / ||A||_F.  (L1 = max column sum,
 * as torch.linalg.matrix_norm(ord=1).) */
int oracle_residuals(const float* a, const float* l, int64_t batch, int64_t n, double* out) {
  double* col = (double*)malloc(sizeof(double) * (size_t)n * 3);
  if (!col) return -1;
  for (int64_t b = 0; b < batch; ++b) {
    const float* A = a + b * n * n;
    const float* L = l + b * n * n;
    double* ca = col;
    double* cu = col + n;
    double* cr = col + 2 * n;
    memset(col, 0, sizeof(double) * (size_t)n * 3);
    double fr = 0.0, fa = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      for (int64_t j = 0; j < n; ++j) {
        const double aij = A[i * n + j];
        ca[j] += fabs(aij);
        if (j > i) cu[j] += fabs((double)L[i * n + j]);
        double s = 0.0;
        for (int64_t k = 0; k < n; ++k) s += (double)L[i * n + k] * (double)L[j * n + k];
        const double r = s - aij;
        cr[j] += fabs(r);
        fr += r * r;
        fa += aij * aij;
      }
    }
    double ma = 0.0, mu = 0.0, mr = 0.0;
    for (int64_t j = 0; j < n; ++j) {
      if (ca[j] > ma) ma = ca[j];
      if (cu[j] > mu) mu = cu[j];
      if (cr[j] > mr) mr = cr[j];
    }
    out[4 * b + 0] = ma;
    out[4 * b + 1] = mu;
    out[4 * b + 2] = mr;
    out[4 * b + 3] = fa > 0.0 ? sqrt(fr / fa) : sqrt(fr);
  }
  free(col);
  return 0;
}

/* Cholesky adjoint in FP64: given L and Lbar (lower triangles used),
 * Abar = 1/2 (S + S^T) with S = L^{-T} Phi(L^T Lbar) L^{-1}, where Phi keeps
 * the lower triangle and halves the diagonal. */
int oracle_potrf_backward_f64(const double* l, const double* lbar, double* abar, int64_t batch,
                              int64_t n) {
  double* P = (double*)malloc(sizeof(double) * (size_t)(n * n));
  if (!P) return -1;
  for (int64_t b = 0; b < batch; ++b) {
    const double* L = l + b * n * n;
    const double* G = lbar + b * n * n;
    double* X = abar + b * n * n;
    /* P = Phi(L^T G), G lower. (L^T G)[i][j] = sum_k L[k][i] G[k][j], k >= max(i,j) */
    for (int64_t i = 0; i < n; ++i)
      for (int64_t j = 0; j < n; ++j) {
        double s = 0.0;
        if (j <= i) {
          for (int64_t k = i; k < n; ++k) s += L[k * n + i] * G[k * n + j];
          if (j == i) s *= 0.5;
        }
        P[i * n + j] = s;
      }
    /* Y = L^{-T} P: solve L^T Y = P (upper-triangular back substitution). */
    for (int64_t c = 0; c < n; ++c)
      for (int64_t i = n - 1; i >= 0; --i) {
        double s = P[i * n + c];
        for (int64_t k = i + 1; k < n; ++k) s -= L[k * n + i] * P[k * n + c];
        P[i * n + c] = s / L[i * n + i];
      }
    /* S = Y L^{-1}: solve S L = Y row by row (columns from last to first). */
    for (int64_t r = 0; r < n; ++r)
      for (int64_t j = n - 1; j >= 0; --j) {
        double s = P[r * n + j];
        for (int64_t k = j + 1; k < n; ++k) s -= P[r * n + k] * L[k * n + j];
        P[r * n + j] = s / L[j * n + j];
      }
    for (int64_t i = 0; i < n; ++i)
      for (int64_t j = 0; j < n; ++j) X[i * n + j] = 0.5 * (P[i * n + j] + P[j * n + i]);
  }
  free(P);
  return 0;
}
