/*
 * CPU ORACLE — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of NumPP's portable dense linear-solve path, used by
 * tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py as the
 * checker. Nothing in the product (numpp_b200/) links, loads or calls it.
 *
 * Each function names the reference code it restates (paths are inside the
 * CyberdyneCorp/NumPP tree). The arithmetic is the same sequence of IEEE
 * double operations as the reference's templates compiled without FMA
 * contraction (x86-64 baseline, no -mfma), so results are bit-identical to the
 * reference build (checked against oracle/_ref and tests/golden/).
 *
 * Row-major everywhere. Status codes: 1 = ok, 0 = singular (exact zero pivot).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* src/linalg/linalg.cpp:48-71 (lu_decompose<T>): unblocked right-looking LU
 * with partial pivoting. Column-k argmax of |A[i,k]| scanning i = k+1.. with a
 * strict '>' so the first maximum wins; full-row swap; piv is the permutation
 * vector (piv[i] = original row now at position i); permsign flips per swap.
 * Returns 0 as soon as the best pivot is exactly 0.0 (A is then partly
 * factored, as in the reference). */
int oracle_lu_decompose(double* A, int n, int* piv, double* permsign) {
  for (int i = 0; i < n; ++i) piv[i] = i;
  *permsign = 1.0;
  for (int k = 0; k < n; ++k) {
    int pr = k;
    double best = fabs(A[(int64_t)k * n + k]);
    for (int i = k + 1; i < n; ++i) {
      double v = fabs(A[(int64_t)i * n + k]);
      if (v > best) { best = v; pr = i; }
    }
    if (best == 0.0) return 0;
    if (pr != k) {
      for (int j = 0; j < n; ++j) {
        double t = A[(int64_t)k * n + j];
        A[(int64_t)k * n + j] = A[(int64_t)pr * n + j];
        A[(int64_t)pr * n + j] = t;
      }
      int t = piv[k]; piv[k] = piv[pr]; piv[pr] = t;
      *permsign = -*permsign;
    }
    const double akk = A[(int64_t)k * n + k];
    for (int i = k + 1; i < n; ++i) {
      double f = A[(int64_t)i * n + k] / akk;
      A[(int64_t)i * n + k] = f;
      double* ri = A + (int64_t)i * n;
      const double* rk = A + (int64_t)k * n;
      for (int j = k + 1; j < n; ++j) {
        double p = f * rk[j]; /* separate multiply and subtract: no FMA */
        ri[j] = ri[j] - p;
      }
    }
  }
  return 1;
}

/* src/linalg/linalg.cpp:73-90 (lu_solve<T>): X[i,:] = B[piv[i],:], forward
 * substitution with the unit lower factor, back substitution with the upper
 * factor, dividing by the diagonal last. B is n x m row-major, overwritten. */
void oracle_lu_solve(const double* LU, int n, const int* piv, double* B, int m) {
  size_t sz = (size_t)n * (size_t)m;
  double* X = (double*)malloc(sz ? sz * sizeof(double) : 1);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < m; ++j) X[(int64_t)i * m + j] = B[(int64_t)piv[i] * m + j];
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < i; ++k) {
      double l = LU[(int64_t)i * n + k];
      for (int j = 0; j < m; ++j) {
        double p = l * X[(int64_t)k * m + j];
        X[(int64_t)i * m + j] = X[(int64_t)i * m + j] - p;
      }
    }
  for (int i = n - 1; i >= 0; --i) {
    for (int k = i + 1; k < n; ++k) {
      double u = LU[(int64_t)i * n + k];
      for (int j = 0; j < m; ++j) {
        double p = u * X[(int64_t)k * m + j];
        X[(int64_t)i * m + j] = X[(int64_t)i * m + j] - p;
      }
    }
    double d = LU[(int64_t)i * n + i];
    for (int j = 0; j < m; ++j) X[(int64_t)i * m + j] /= d;
  }
  if (sz) memcpy(B, X, sz * sizeof(double));
  free(X);
}

/* src/linalg/linalg.cpp:92-103 (solve_impl): LU of a copy of A, then lu_solve.
 * Returns 0 (the reference throws linalg_error("Singular matrix")). */
int oracle_solve(const double* A, const double* B, double* X, int n, int m) {
  size_t nn = (size_t)n * n;
  double* W = (double*)malloc(nn ? nn * sizeof(double) : 1);
  int* piv = (int*)malloc(n ? n * sizeof(int) : 1);
  double sgn;
  if (nn) memcpy(W, A, nn * sizeof(double));
  int ok = oracle_lu_decompose(W, n, piv, &sgn);
  if (ok) {
    if (n && m) memcpy(X, B, (size_t)n * m * sizeof(double));
    oracle_lu_solve(W, n, piv, X, m);
  }
  free(W); free(piv);
  return ok;
}

/* src/linalg/linalg.cpp:105-115 (inv_impl): LU, then lu_solve against I. */
int oracle_inv(const double* A, double* Ainv, int n) {
  size_t nn = (size_t)n * n;
  double* W = (double*)malloc(nn ? nn * sizeof(double) : 1);
  int* piv = (int*)malloc(n ? n * sizeof(int) : 1);
  double sgn;
  if (nn) memcpy(W, A, nn * sizeof(double));
  int ok = oracle_lu_decompose(W, n, piv, &sgn);
  if (ok) {
    for (size_t i = 0; i < nn; ++i) Ainv[i] = 0.0;
    for (int i = 0; i < n; ++i) Ainv[(int64_t)i * n + i] = 1.0;
    oracle_lu_solve(W, n, piv, Ainv, n);
  }
  free(W); free(piv);
  return ok;
}

/* src/linalg/linalg.cpp:393-407 (det): permsign * prod U[i,i] multiplied in
 * order i = 0..n-1; a singular matrix gives 0.0 (no exception). n = 0 gives 1. */
double oracle_det(const double* A, int n) {
  size_t nn = (size_t)n * n;
  double* W = (double*)malloc(nn ? nn * sizeof(double) : 1);
  int* piv = (int*)malloc(n ? n * sizeof(int) : 1);
  double sgn, d;
  if (nn) memcpy(W, A, nn * sizeof(double));
  if (!oracle_lu_decompose(W, n, piv, &sgn)) d = 0.0;
  else { d = sgn; for (int i = 0; i < n; ++i) d *= W[(int64_t)i * n + i]; }
  free(W); free(piv);
  return d;
}

/* src/linalg/linalg.cpp:408-439 (slogdet): logabsdet = sum log|d_i| and
 * sign *= d_i/|d_i| in order; singular gives (0, -inf). */
void oracle_slogdet(const double* A, int n, double* sign, double* logabsdet) {
  size_t nn = (size_t)n * n;
  double* W = (double*)malloc(nn ? nn * sizeof(double) : 1);
  int* piv = (int*)malloc(n ? n * sizeof(int) : 1);
  double sgn;
  if (nn) memcpy(W, A, nn * sizeof(double));
  if (!oracle_lu_decompose(W, n, piv, &sgn)) {
    *sign = 0.0;
    *logabsdet = -INFINITY;
  } else {
    double logabs = 0.0, s = sgn;
    for (int i = 0; i < n; ++i) {
      double d = W[(int64_t)i * n + i];
      double m = fabs(d);
      logabs += log(m);
      s *= d / m;
    }
    *sign = s;
    *logabsdet = logabs;
  }
  free(W); free(piv);
}

/* src/backend/backend.cpp:55-84 (cpu_matmul): C[m,n] = A[m,k] B[k,n] with the
 * i-p-j loop order, accumulated in p order. */
void oracle_matmul(int64_t m, int64_t n, int64_t k, const double* A, const double* B, double* C) {
  for (int64_t i = 0; i < m; ++i) {
    for (int64_t j = 0; j < n; ++j) C[i * n + j] = 0.0;
    for (int64_t p = 0; p < k; ++p) {
      const double aip = A[i * k + p];
      const double* brow = B + p * n;
      double* crow = C + i * n;
      for (int64_t j = 0; j < n; ++j) {
        double t = aip * brow[j];
        crow[j] = crow[j] + t;
      }
    }
  }
}

/* ---- stacked forms: src/linalg/batched.cpp:51-108 loop the 2-D routine over
 * a contiguous (count, n, n) view. The reference aborts the whole call on the
 * first singular matrix; here each matrix reports its own status in ok[] so a
 * test can check both behaviours. ---- */

void oracle_lu_batched(int64_t count, int n, double* A, int* piv, double* permsign, int* ok) {
  for (int64_t b = 0; b < count; ++b)
    ok[b] = oracle_lu_decompose(A + b * (int64_t)n * n, n, piv + b * n, permsign + b);
}

void oracle_solve_batched(int64_t count, int n, int m, const double* A, const double* B,
                          double* X, int* ok) {
  for (int64_t b = 0; b < count; ++b)
    ok[b] = oracle_solve(A + b * (int64_t)n * n, B + b * (int64_t)n * m,
                         X + b * (int64_t)n * m, n, m);
}

void oracle_inv_batched(int64_t count, int n, const double* A, double* Ainv, int* ok) {
  for (int64_t b = 0; b < count; ++b)
    ok[b] = oracle_inv(A + b * (int64_t)n * n, Ainv + b * (int64_t)n * n, n);
}

void oracle_det_batched(int64_t count, int n, const double* A, double* det) {
  for (int64_t b = 0; b < count; ++b) det[b] = oracle_det(A + b * (int64_t)n * n, n);
}

void oracle_slogdet_batched(int64_t count, int n, const double* A, double* sign, double* logabsdet) {
  for (int64_t b = 0; b < count; ++b)
    oracle_slogdet(A + b * (int64_t)n * n, n, sign + b, logabsdet + b);
}

/* Uneven batch: system i has order n[i] and nrhs[i], its matrix at a_off[i]
 * and its right-hand side / solution at b_off[i] (element offsets). Each system
 * is the 2-D reference call (linalg.cpp:368-385, 393-439, 386-392). inv_off[i]
 * < 0 means no inverse for that system. */
void oracle_solve_grouped(int64_t count, const int* n, const int* nrhs, const int64_t* a_off,
                          const int64_t* b_off, const int64_t* inv_off, const double* A,
                          const double* B, double* X, double* sign, double* logabsdet,
                          double* inv, int* ok) {
  for (int64_t i = 0; i < count; ++i) {
    const double* Ai = A + a_off[i];
    ok[i] = oracle_solve(Ai, B + b_off[i], X + b_off[i], n[i], nrhs[i]);
    if (sign) oracle_slogdet(Ai, n[i], sign + i, logabsdet + i);
    if (inv && inv_off[i] >= 0) oracle_inv(Ai, inv + inv_off[i], n[i]);
  }
}

/* src/linalg/linalg.cpp:117-136 (cholesky_impl<T>, real case): column by
 * column, diag = A[j,j] - sum_p L[j,p]^2 (subtracting in p order), stop when
 * diag <= 0 ("Matrix is not positive definite"); L[j,j] = sqrt(diag); below
 * it L[i,j] = (A[i,j] - sum_p L[i,p] L[j,p]) / L[j,j]. Only the lower triangle
 * of A is read. Returns 1, or 0 when A is not positive definite (L is then
 * partly filled, as far as the reference got). */
int oracle_cholesky(const double* A, double* L, int n) {
  memset(L, 0, sizeof(double) * (size_t)n * n);
  for (int j = 0; j < n; ++j) {
    double sum = A[(int64_t)j * n + j];
    for (int p = 0; p < j; ++p) sum -= L[(int64_t)j * n + p] * L[(int64_t)j * n + p];
    if (sum <= 0.0) return 0;
    const double ljj = sqrt(sum);
    L[(int64_t)j * n + j] = ljj;
    for (int i = j + 1; i < n; ++i) {
      double s = A[(int64_t)i * n + j];
      for (int p = 0; p < j; ++p) s -= L[(int64_t)i * n + p] * L[(int64_t)j * n + p];
      L[(int64_t)i * n + j] = s / ljj;
    }
  }
  return 1;
}

void oracle_cholesky_batched(int64_t count, int n, const double* A, double* L, int* ok) {
  for (int64_t b = 0; b < count; ++b)
    ok[b] = oracle_cholesky(A + b * (int64_t)n * n, L + b * (int64_t)n * n, n);
}

/* src/linalg/linalg.cpp:620-712 (svd_jacobi<T>, real case, economy size) and
 * :755-784 (lstsq). Cyclic one-sided Jacobi on the tall orientation (A, or
 * A^T when m < n): for every column pair in order, the squared norms and the
 * dot product (sums in row order), a sign flip of column j making the dot
 * product positive, then the rotation with zeta = (bb - aa) / (2|c|); at most
 * 60 sweeps, stopping once the largest |c| / sqrt(aa bb) is below 1e-15.
 * Singular values are the column norms, sorted descending (stable here; the
 * reference's std::sort orders equal values arbitrarily). lstsq: tol = (rcond
 * < 0 ? eps * max(m, n) : rcond) * s_max, rank = #{s > tol}, x = V diag(1/s or
 * 0) U^T b with both products accumulated in p order (cpu_matmul). The
 * residuals (m > n and full rank) are sum_i (b - A x)_ij^2 per column j.
 * B is m x k row-major, X n x k. Returns 1 when residuals were formed. */
static void matmul_p(const double* A, const double* B, double* C, int m, int kdim, int n) {
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) C[(int64_t)i * n + j] = 0.0;
  for (int i = 0; i < m; ++i)
    for (int p = 0; p < kdim; ++p) {
      const double a = A[(int64_t)i * kdim + p];
      for (int j = 0; j < n; ++j) C[(int64_t)i * n + j] += a * B[(int64_t)p * n + j];
    }
}

int oracle_lstsq(const double* A, int m, int n, const double* B, int k, double rcond, double* X, double* s,
                 int* rank, double* resid) {
  const int kk = m < n ? m : n, wide = m < n, M = wide ? n : m, N = wide ? m : n;
  double* W = (double*)malloc(sizeof(double) * (size_t)M * N);
  double* V = (double*)calloc((size_t)N * N, sizeof(double));
  for (int i = 0; i < M; ++i)
    for (int j = 0; j < N; ++j) W[(int64_t)i * N + j] = wide ? A[(int64_t)j * n + i] : A[(int64_t)i * n + j];
  for (int i = 0; i < N; ++i) V[(int64_t)i * N + i] = 1.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double maxoff = 0.0;
    for (int i = 0; i < N; ++i)
      for (int j = i + 1; j < N; ++j) {
        double aa = 0, bb = 0, cc = 0;
        for (int r = 0; r < M; ++r) {
          const double xi = W[(int64_t)r * N + i], xj = W[(int64_t)r * N + j];
          aa += fabs(xi) * fabs(xi);
          bb += fabs(xj) * fabs(xj);
          cc += xi * xj;
        }
        if (aa == 0.0 || bb == 0.0) continue;
        const double magc = fabs(cc), off = magc / sqrt(aa * bb);
        if (off > maxoff) maxoff = off;
        if (off < 1e-300) continue;
        const double w = cc / magc;
        for (int r = 0; r < M; ++r) W[(int64_t)r * N + j] = W[(int64_t)r * N + j] * w;
        for (int r = 0; r < N; ++r) V[(int64_t)r * N + j] = V[(int64_t)r * N + j] * w;
        const double zeta = (bb - aa) / (2.0 * magc);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
        for (int r = 0; r < M; ++r) {
          const double xi = W[(int64_t)r * N + i], xj = W[(int64_t)r * N + j];
          W[(int64_t)r * N + i] = cs * xi - sn * xj;
          W[(int64_t)r * N + j] = sn * xi + cs * xj;
        }
        for (int r = 0; r < N; ++r) {
          const double vi = V[(int64_t)r * N + i], vj = V[(int64_t)r * N + j];
          V[(int64_t)r * N + i] = cs * vi - sn * vj;
          V[(int64_t)r * N + j] = sn * vi + cs * vj;
        }
      }
    if (maxoff < 1e-15) break;
  }
  double* sig = (double*)malloc(sizeof(double) * (size_t)N);
  int* ord = (int*)malloc(sizeof(int) * (size_t)N);
  for (int j = 0; j < N; ++j) {
    double s2 = 0;
    for (int r = 0; r < M; ++r) {
      const double aj = fabs(W[(int64_t)r * N + j]);
      s2 += aj * aj;
    }
    sig[j] = sqrt(s2);
    if (sig[j] > 0)
      for (int r = 0; r < M; ++r) W[(int64_t)r * N + j] = W[(int64_t)r * N + j] / sig[j];
    else
      for (int r = 0; r < M; ++r) W[(int64_t)r * N + j] = 0.0;
    ord[j] = j;
  }
  for (int a = 1; a < N; ++a) { /* stable insertion sort, descending */
    const int o = ord[a];
    int b = a - 1;
    while (b >= 0 && sig[ord[b]] < sig[o]) { ord[b + 1] = ord[b]; --b; }
    ord[b + 1] = o;
  }
  double* Us = (double*)malloc(sizeof(double) * (size_t)M * N); /* sorted tall U, M x N */
  double* Vs = (double*)malloc(sizeof(double) * (size_t)N * N); /* sorted V, N x N */
  for (int c = 0; c < N; ++c) {
    s[c] = sig[ord[c]];
    for (int r = 0; r < M; ++r) Us[(int64_t)r * N + c] = W[(int64_t)r * N + ord[c]];
    for (int r = 0; r < N; ++r) Vs[(int64_t)r * N + c] = V[(int64_t)r * N + ord[c]];
  }
  const double smax = kk ? s[0] : 0.0;
  const double eps = 2.220446049250313e-16;
  const double tol = (rcond < 0 ? eps * (m > n ? m : n) : rcond) * smax;
  int rk = 0;
  double* sinv = (double*)malloc(sizeof(double) * (size_t)(kk ? kk : 1));
  for (int i = 0; i < kk; ++i) {
    const int ok = s[i] > tol;
    sinv[i] = ok ? 1.0 / s[i] : 0.0;
    rk += ok;
  }
  *rank = rk;
  /* u (m x kk) and V = conj(vh)^T (n x kk) of the reference's economy svd */
  const double* Um = wide ? Vs : Us;
  const double* Vm = wide ? Us : Vs;
  double* Uh = (double*)malloc(sizeof(double) * (size_t)kk * m);
  for (int c = 0; c < kk; ++c)
    for (int p = 0; p < m; ++p) Uh[(int64_t)c * m + p] = Um[(int64_t)p * kk + c];
  double* T1 = (double*)malloc(sizeof(double) * (size_t)kk * k);
  matmul_p(Uh, B, T1, kk, m, k);
  for (int c = 0; c < kk; ++c)
    for (int j = 0; j < k; ++j) T1[(int64_t)c * k + j] = sinv[c] * T1[(int64_t)c * k + j];
  matmul_p(Vm, T1, X, n, kk, k);
  int has = 0;
  if (m > n && rk == n) {
    double* AX = (double*)malloc(sizeof(double) * (size_t)m * k);
    matmul_p(A, X, AX, m, n, k);
    for (int j = 0; j < k; ++j) {
      double acc = 0.0;
      for (int i = 0; i < m; ++i) {
        const double d = B[(int64_t)i * k + j] - AX[(int64_t)i * k + j];
        acc += fabs(d) * fabs(d);
      }
      resid[j] = acc;
    }
    free(AX);
    has = 1;
  }
  free(W); free(V); free(sig); free(ord); free(Us); free(Vs); free(sinv); free(Uh); free(T1);
  return has;
}
