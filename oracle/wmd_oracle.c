/*
 * TEST INFRASTRUCTURE ONLY — the FP64 CPU oracle for the Sinkhorn WMD solve.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this file (as liboracle.so).  The product library never links it and has no
 * CPU fallback onto it.
 *
 * It restates, in code of its own, the reference's fused solver
 * sinkhorn_wmd_fused.cpp:112-393 (IntelLabs/Optimized-Implementation-of-Word-
 * Movers-Distance), with the same FP64 operation order so that, run with one
 * thread, it reproduces the reference bit for bit:
 *   select          r != 0 in ascending id order          fused:45-63
 *   distance        sqrt(sum_k (a_k - b_k)^2), k ascending fused:35-43
 *   K, K/r          K = exp(-lambda M), K_over_r = (1/r) K fused:210-220
 *   init            u = v_r, x = 0                         fused:188-191
 *   iteration       s = K_w . u, o = c/s, x += K_over_r_w o fused:255-289
 *   u = 1/x                                                fused:313-317
 *   final           x += (K_w * M_w) o                     fused:344-376
 *   reduce          WMD_j = sum_i u_ij x_ij                fused:382-393
 * Differences that do not change results: the target matrix is traversed
 * column by column (one target document at a time, entries in ascending word
 * order), which is the reference's accumulation order when it runs on one
 * OpenMP thread, and which needs no atomics when columns run in parallel.
 *
 * lambda here is the positive regulariser: K = exp(-lambda * M).  The fused
 * reference is called with lamda = -lambda (it computes exp(M * lamda),
 * fused:217); the nonfused reference with lamda = +lambda (it computes
 * exp(-M * lamda), sinkhorn_wmd_nonfused.cpp:172-173).
 *
 * Additions with no reference counterpart (the reference fixes the iteration
 * count, main.py:11-12): a converged mode that iterates each document until its
 * marginal residual  sum_i |u_i (K v)_i - r_i|  falls below a tolerance, and
 * the stable counting-sort builders of CSR (fused:493-506) and CSC layouts.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef uint64_t u64;

/* Compaction of the source histogram: ids with r != 0, ascending (fused:45-63). */
u64 oracle_select(const double* r, u64 V, u64* ids, double* weights) {
  u64 n = 0;
  for (u64 i = 0; i < V; i++) {
    if (r[i] == 0) continue;
    ids[n] = i;
    weights[n] = r[i];
    n++;
  }
  return n;
}

/* Panel build in the fused layout [V][v_r] (fused:197-223).  Writes M, K and
 * K_over_r; any of them may be NULL except K. */
static void build_panel(const double* vecs, u64 V, u64 d, const u64* ids,
                        const double* w, u64 vr, double lambda, double* M,
                        double* K, double* Kr) {
#pragma omp parallel for schedule(static)
  for (long long jj = 0; jj < (long long)V; jj++) {
    u64 j = (u64)jj;
    const double* b = vecs + j * d;
    for (u64 i = 0; i < vr; i++) {
      const double* a = vecs + ids[i] * d;
      double s = 0.0;
      for (u64 k = 0; k < d; k++) {
        const double t = a[k] - b[k];
        s += t * t;
      }
      const double m = sqrt(s);
      /* The fused reference multiplies M by its (negative) lamda argument. */
      const double kv = exp(m * (-lambda));
      if (M) M[j * vr + i] = m;
      K[j * vr + i] = kv;
      if (Kr) Kr[j * vr + i] = (1.0 / w[i]) * kv;
    }
  }
}

/* One document: max_iter x-updates then the K.*M half-step (fused:246-393).
 * u (v_r) and x (v_r) are caller scratch.  Returns the WMD value. */
static double solve_column(const double* K, const double* Kr, const double* M,
                           u64 vr, const u64* rows, const double* vals, u64 n,
                           int max_iter, double* u, double* x) {
  for (u64 i = 0; i < vr; i++) {
    u[i] = (double)vr;
    x[i] = 0.0;
  }
  for (int it = 0; it < max_iter; it++) {
    for (u64 e = 0; e < n; e++) {
      const double* Kw = K + rows[e] * vr;
      double s = 0.0;
      for (u64 k = 0; k < vr; k++) s += Kw[k] * u[k];
      const double o = vals[e] / s;
      const double* Krw = Kr + rows[e] * vr;
      for (u64 i = 0; i < vr; i++) x[i] += Krw[i] * o;
    }
    for (u64 i = 0; i < vr; i++) {
      u[i] = 1.0 / x[i];
      x[i] = 0.0;
    }
  }
  for (u64 e = 0; e < n; e++) {
    const u64 w = rows[e];
    const double* Kw = K + w * vr;
    double s = 0.0;
    for (u64 k = 0; k < vr; k++) s += Kw[k] * u[k];
    const double o = vals[e] / s;
    for (u64 i = 0; i < vr; i++) {
      const u64 idx = i + w * vr;
      x[i] += (K[idx] * M[idx]) * o;
    }
  }
  double acc = 0.0;
  for (u64 i = 0; i < vr; i++) acc += u[i] * x[i];
  return acc;
}

static void set_threads(int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
}

/*
 * Full solve for one source histogram r (dense, length V) against the CSC
 * target matrix (col_ptr[N+1], row_inds[nnz], vals[nnz]).  Returns v_r, or -1
 * on allocation failure.  wmd_out has N entries.
 */
long long oracle_sinkhorn(const double* r, const double* vecs, u64 V, u64 d,
                          u64 N, const u64* col_ptr, const u64* row_inds,
                          const double* vals, double lambda, int max_iter,
                          double* wmd_out, int nthreads) {
  set_threads(nthreads);
  u64* ids = (u64*)malloc((V + 1) * sizeof(u64));
  double* w = (double*)malloc((V + 1) * sizeof(double));
  if (!ids || !w) {
    free(ids);
    free(w);
    return -1;
  }
  const u64 vr = oracle_select(r, V, ids, w);
  double* M = (double*)malloc((V * vr + 1) * sizeof(double));
  double* K = (double*)malloc((V * vr + 1) * sizeof(double));
  double* Kr = (double*)malloc((V * vr + 1) * sizeof(double));
  if (!M || !K || !Kr) {
    free(ids); free(w); free(M); free(K); free(Kr);
    return -1;
  }
  build_panel(vecs, V, d, ids, w, vr, lambda, M, K, Kr);
  int fail = 0;
#pragma omp parallel
  {
    double* u = (double*)malloc((vr + 1) * sizeof(double));
    double* x = (double*)malloc((vr + 1) * sizeof(double));
    if (!u || !x) {
#pragma omp atomic write
      fail = 1;
    } else {
#pragma omp for schedule(dynamic, 16)
      for (long long jj = 0; jj < (long long)N; jj++) {
        const u64 j = (u64)jj;
        const u64 b = col_ptr[j], n = col_ptr[j + 1] - col_ptr[j];
        wmd_out[j] = solve_column(K, Kr, M, vr, row_inds + b, vals + b, n,
                                  max_iter, u, x);
      }
    }
    free(u);
    free(x);
  }
  free(ids); free(w); free(M); free(K); free(Kr);
  return fail ? -1 : (long long)vr;
}

/*
 * Converged FP64 mode (no reference counterpart).  Each document iterates
 * x-updates until the marginal residual
 *     res = sum_i | u_i (K v)_i - r_i |,   v = c ./ (K^T u)
 * measured with the scalings that enter an update, is <= tol, or until
 * max_iter_cap updates have run.  The WMD is then formed with the same final
 * half-step as the fixed-count solve.  iters_out[j] receives the number of
 * x-updates taken, res_out[j] the last residual measured, and, when u_out is
 * not NULL, u_out[j*v_r + i] the final scalings u (after the last update).
 */
long long oracle_sinkhorn_converged(const double* r, const double* vecs, u64 V,
                                    u64 d, u64 N, const u64* col_ptr,
                                    const u64* row_inds, const double* vals,
                                    double lambda, double tol, int max_iter_cap,
                                    double* wmd_out, int* iters_out,
                                    double* res_out, double* u_out,
                                    int nthreads) {
  set_threads(nthreads);
  u64* ids = (u64*)malloc((V + 1) * sizeof(u64));
  double* w = (double*)malloc((V + 1) * sizeof(double));
  if (!ids || !w) {
    free(ids);
    free(w);
    return -1;
  }
  const u64 vr = oracle_select(r, V, ids, w);
  double* M = (double*)malloc((V * vr + 1) * sizeof(double));
  double* K = (double*)malloc((V * vr + 1) * sizeof(double));
  double* Kr = (double*)malloc((V * vr + 1) * sizeof(double));
  if (!M || !K || !Kr) {
    free(ids); free(w); free(M); free(K); free(Kr);
    return -1;
  }
  build_panel(vecs, V, d, ids, w, vr, lambda, M, K, Kr);
  int fail = 0;
#pragma omp parallel
  {
    double* u = (double*)malloc((vr + 1) * sizeof(double));
    double* x = (double*)malloc((vr + 1) * sizeof(double));
    if (!u || !x) {
#pragma omp atomic write
      fail = 1;
    } else {
#pragma omp for schedule(dynamic, 16)
      for (long long jj = 0; jj < (long long)N; jj++) {
        const u64 j = (u64)jj;
        const u64 b = col_ptr[j], n = col_ptr[j + 1] - col_ptr[j];
        const u64* rows = row_inds + b;
        const double* cv = vals + b;
        for (u64 i = 0; i < vr; i++) {
          u[i] = (double)vr;
          x[i] = 0.0;
        }
        int it = 0;
        double res = INFINITY;
        while (it < max_iter_cap) {
          for (u64 e = 0; e < n; e++) {
            const double* Kw = K + rows[e] * vr;
            double s = 0.0;
            for (u64 k = 0; k < vr; k++) s += Kw[k] * u[k];
            const double o = cv[e] / s;
            const double* Krw = Kr + rows[e] * vr;
            for (u64 i = 0; i < vr; i++) x[i] += Krw[i] * o;
          }
          /* (K v)_i = r_i x_i with x = diag(1/r) K v. */
          res = 0.0;
          for (u64 i = 0; i < vr; i++) res += fabs(u[i] * w[i] * x[i] - w[i]);
          for (u64 i = 0; i < vr; i++) {
            u[i] = 1.0 / x[i];
            x[i] = 0.0;
          }
          it++;
          if (res <= tol) break;
        }
        if (u_out)
          for (u64 i = 0; i < vr; i++) u_out[j * vr + i] = u[i];
        for (u64 e = 0; e < n; e++) {
          const u64 wd = rows[e];
          const double* Kw = K + wd * vr;
          double s = 0.0;
          for (u64 k = 0; k < vr; k++) s += Kw[k] * u[k];
          const double o = cv[e] / s;
          for (u64 i = 0; i < vr; i++) {
            const u64 idx = i + wd * vr;
            x[i] += (K[idx] * M[idx]) * o;
          }
        }
        double acc = 0.0;
        for (u64 i = 0; i < vr; i++) acc += u[i] * x[i];
        wmd_out[j] = acc;
        if (iters_out) iters_out[j] = it;
        if (res_out) res_out[j] = res;
      }
    }
    free(u);
    free(x);
  }
  free(ids); free(w); free(M); free(K); free(Kr);
  return fail ? -1 : (long long)vr;
}

/*
 * Stable counting sort of an edge list by its `key` array (0..nkeys-1): the
 * CSR build of fused:493-506 when key = word, the CSC build when key = doc.
 * Entries with equal key keep their input order.  ptr has nkeys+1 entries.
 */
int oracle_counting_sort(u64 nkeys, u64 nnz, const u64* key, const u64* other,
                         const double* w, u64* ptr, u64* other_out,
                         double* w_out) {
  u64* deg = (u64*)calloc(nkeys + 1, sizeof(u64));
  if (!deg) return -1;
  for (u64 e = 0; e < nnz; e++) {
    if (key[e] >= nkeys) {
      free(deg);
      return -2;
    }
    deg[key[e]]++;
  }
  ptr[0] = 0;
  for (u64 k = 1; k <= nkeys; k++) {
    ptr[k] = ptr[k - 1] + deg[k - 1];
    deg[k - 1] = 0;
  }
  for (u64 e = 0; e < nnz; e++) {
    const u64 k = key[e];
    const u64 pos = ptr[k] + deg[k];
    other_out[pos] = other[e];
    w_out[pos] = w[e];
    deg[k]++;
  }
  free(deg);
  return 0;
}

/* Stable CSR (rows = words) -> CSC (columns = docs) transpose.  Within a
 * column the entries come out in ascending row order, with equal rows in
 * their CSR order. */
int oracle_csr_to_csc(u64 nrows, u64 ncols, const u64* row_ptr,
                      const u64* col_inds, const double* vals, u64* col_ptr,
                      u64* row_inds, double* vals_out) {
  const u64 nnz = row_ptr[nrows];
  u64* rows = (u64*)malloc((nnz + 1) * sizeof(u64));
  if (!rows) return -1;
  for (u64 i = 0; i < nrows; i++)
    for (u64 e = row_ptr[i]; e < row_ptr[i + 1]; e++) rows[e] = i;
  const int rc = oracle_counting_sort(ncols, nnz, col_inds, rows, vals,
                                      col_ptr, row_inds, vals_out);
  free(rows);
  return rc;
}
