// Clebsch-Gordan column solver shared by the gravity and product tables.
#pragma once
#include <cuda_runtime.h>

// ---------------------------------------------------- Clebsch-Gordan ----
// Column (l, m) of clebsch_gordan.m:5-40: the coefficients over
// m1 in [max(-l1, m-l2), min(l1, m+l2)] from the tridiagonal system with the
// last coefficient positive.  The (nnz-1)-square leading block is solved by
// Gaussian elimination with partial pivoting (the LAPACK gtsv recurrence).
// Returns nnz; C must hold 2*min(l1,l2)+1 values.
__device__ __forceinline__ int cg_column(int l1, int l2, int l, int m, double* C, double* dd, double* du, double* dl,
                         double* rb) {
  const int m1lo = max(-l1, m - l2), m1hi = min(l1, m + l2);
  const int nnz = m1hi - m1lo + 1;
  if (nnz <= 1) { C[0] = 1.0; return 1; }
  const double j1 = l1 * (l1 + 1.0), j2 = l2 * (l2 + 1.0), jj = l * (l + 1.0);
  // A(k,k) and A(k-1,k) for k in [0, nnz)
  auto diag = [&](int k) { const double a = m1lo + k, b = m - a; return j1 + j2 + 2 * a * b - jj; };
  auto off = [&](int k) {  // A(k-1, k)
    const double a0 = m1lo + k - 1, a1 = m1lo + k, b0 = m - a0, b1 = m - a1;
    return sqrt(j1 - a0 * a1) * sqrt(j2 - b0 * b1);
  };
  const int n = nnz - 1;
  for (int k = 0; k < n; ++k) { dd[k] = diag(k); rb[k] = 0.0; }
  for (int k = 0; k + 1 < n; ++k) { du[k] = off(k + 1); dl[k] = off(k + 1); }
  rb[n - 1] = -off(n);
  for (int i = 0; i + 1 < n; ++i) {
    if (fabs(dd[i]) >= fabs(dl[i])) {
      const double fct = dl[i] / dd[i];
      dd[i + 1] -= fct * du[i];
      rb[i + 1] -= fct * rb[i];
      dl[i] = 0.0;
    } else {
      const double fct = dd[i] / dl[i];
      dd[i] = dl[i];
      double tmp = dd[i + 1];
      dd[i + 1] = du[i] - fct * tmp;
      if (i + 2 < n) {
        dl[i] = du[i + 1];
        du[i + 1] = -fct * dl[i];
      }
      du[i] = tmp;
      tmp = rb[i];
      rb[i] = rb[i + 1];
      rb[i + 1] = tmp - fct * rb[i + 1];
    }
  }
  rb[n - 1] /= dd[n - 1];
  if (n > 1) rb[n - 2] = (rb[n - 2] - du[n - 2] * rb[n - 1]) / dd[n - 2];
  for (int i = n - 3; i >= 0; --i) rb[i] = (rb[i] - du[i] * rb[i + 1] - dl[i] * rb[i + 2]) / dd[i];
  double ss = 0.0;
  for (int k = 0; k < n; ++k) ss += rb[k] * rb[k];
  const double cn = sqrt(1.0 / (1.0 + ss));
  for (int k = 0; k < n; ++k) C[k] = rb[k] * cn;
  C[n] = cn;
  return nnz;
}

