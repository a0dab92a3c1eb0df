/*
 * CPU oracle for the CSR SpMV / SpMM / SDDMM hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the tests, the smoke
 * check and the CPU-baseline leg of the benchmark call it; the product path
 * (flagsparse_b200) never does.
 *
 * Each function restates the algorithm of flagos-ai/FlagSparse it follows
 * (paths relative to the FlagSparse source tree):
 *
 *  oracle_spmv_f32_acc64  sparse_operations/spmv_csr.py:138-144,702-727,179-205
 *      fp32 values/vector, per-row sum evaluated in fp64, rounded to fp32
 *      (the reference casts fp32 data and x to fp64 for its baseline kernel).
 *  oracle_spmv_dot2[_c]   same operator, evaluated with the Dot2 compensated
 *      dot product (Ogita, Rump, Oishi, SIAM J. Sci. Comput. 26(6), 2005),
 *      i.e. as accurately as in twice double precision; the accuracy yardstick.
 *  oracle_spmm_dot2 / oracle_spmm_f32_acc64
 *      sparse_operations/spmm_csr.py:144-200 (C[row, n] = sum_k a_k B[col_k, n]).
 *  oracle_sddmm_dot2      sparse_operations/sddmm_csr.py:471-483
 *      (out[p] = alpha * <x[row(p)], y[col(p)]> + beta * data[p]).
 *  oracle_transpose       sparse_operations/spmv_csr.py:498-536: stable order by
 *      column (a stable argsort), counts per column, prefix sums.  Written as a
 *      counting sort, which is stable by construction.
 *  oracle_bucketize       sparse_operations/spmv_csr.py:371-417: rows per
 *      row-length bucket in ascending row order (torch.nonzero on each mask).
 *  oracle_spmv_plan       the native SpMV unit plan of this package (segments
 *      and work units), restated sequentially for bit-exact comparison.
 *  oracle_coo_to_csr      sparse_operations/spmv_csr.py:948-984
 *      (coo_to_csr_for_spmv): entries ordered by the key row * n_cols + col
 *      (argsort), row pointers from bincount + cumsum.  Written as two stable
 *      counting sorts (by column, then by row), so repeated (row, col) pairs
 *      keep their input order.
 *
 * Index layout: indptr int64, column indices int32 (the Python wrapper
 * converts other layouts).  OpenMP parallelises over rows where rows are
 * independent; every per-row sum runs in ascending nonzero order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---- error-free transformations (Knuth TwoSum, FMA TwoProduct) ------- */
static inline void two_sum(double a, double b, double* s, double* e) {
  double x = a + b;
  double bb = x - a;
  *e = (a - (x - bb)) + (b - bb);
  *s = x;
}
static inline void two_prod(double a, double b, double* p, double* e) {
  double x = a * b;
  *e = fma(a, b, -x);
  *p = x;
}
typedef struct { double hi, lo; } dd;
static inline void dd_add_prod(dd* acc, double a, double b) {
  double p, pe, s, e;
  two_prod(a, b, &p, &pe);
  two_sum(acc->hi, p, &s, &e);
  acc->hi = s;
  acc->lo += e + pe;
}
static inline double dd_val(dd a) { return a.hi + a.lo; }

static void set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ---- SpMV ------------------------------------------------------------ */
void oracle_spmv_f32_acc64(int64_t m, const int64_t* ptr, const int32_t* idx, const float* val, const float* x,
                           float* y, int nthreads) {
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t r = 0; r < m; ++r) {
    double acc = 0.0;
    for (int64_t k = ptr[r]; k < ptr[r + 1]; ++k) acc += (double)val[k] * (double)x[idx[k]];
    y[r] = (float)acc;
  }
}

void oracle_spmv_dot2(int64_t m, const int64_t* ptr, const int32_t* idx, const double* val, const double* x,
                      double* y, int nthreads) {
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t r = 0; r < m; ++r) {
    dd acc = {0.0, 0.0};
    for (int64_t k = ptr[r]; k < ptr[r + 1]; ++k) dd_add_prod(&acc, val[k], x[idx[k]]);
    y[r] = dd_val(acc);
  }
}

/* complex, interleaved (re, im) */
void oracle_spmv_dot2_c(int64_t m, const int64_t* ptr, const int32_t* idx, const double* val, const double* x,
                        double* y, int nthreads) {
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t r = 0; r < m; ++r) {
    dd re = {0.0, 0.0}, im = {0.0, 0.0};
    for (int64_t k = ptr[r]; k < ptr[r + 1]; ++k) {
      double ar = val[2 * k], ai = val[2 * k + 1];
      double xr = x[2 * (int64_t)idx[k]], xi = x[2 * (int64_t)idx[k] + 1];
      dd_add_prod(&re, ar, xr);
      dd_add_prod(&re, -ai, xi);
      dd_add_prod(&im, ar, xi);
      dd_add_prod(&im, ai, xr);
    }
    y[2 * r] = dd_val(re);
    y[2 * r + 1] = dd_val(im);
  }
}

/* ---- SpMM: B is K x N row-major, C is M x N row-major ---------------- */
void oracle_spmm_dot2(int64_t m, int64_t n, const int64_t* ptr, const int32_t* idx, const double* val,
                      const double* b, double* c, int nthreads) {
  set_threads(nthreads);
#pragma omp parallel
  {
    dd* acc = (dd*)malloc(sizeof(dd) * (size_t)(n > 0 ? n : 1));
#pragma omp for schedule(dynamic, 64)
    for (int64_t r = 0; r < m; ++r) {
      for (int64_t j = 0; j < n; ++j) { acc[j].hi = 0.0; acc[j].lo = 0.0; }
      for (int64_t k = ptr[r]; k < ptr[r + 1]; ++k) {
        const double a = val[k];
        const double* brow = b + (int64_t)idx[k] * n;
        for (int64_t j = 0; j < n; ++j) dd_add_prod(&acc[j], a, brow[j]);
      }
      for (int64_t j = 0; j < n; ++j) c[r * n + j] = dd_val(acc[j]);
    }
    free(acc);
  }
}

void oracle_spmm_f32_acc64(int64_t m, int64_t n, const int64_t* ptr, const int32_t* idx, const float* val,
                           const float* b, float* c, int nthreads) {
  set_threads(nthreads);
#pragma omp parallel
  {
    double* acc = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
#pragma omp for schedule(dynamic, 64)
    for (int64_t r = 0; r < m; ++r) {
      for (int64_t j = 0; j < n; ++j) acc[j] = 0.0;
      for (int64_t k = ptr[r]; k < ptr[r + 1]; ++k) {
        const double a = (double)val[k];
        const float* brow = b + (int64_t)idx[k] * n;
        for (int64_t j = 0; j < n; ++j) acc[j] += a * (double)brow[j];
      }
      for (int64_t j = 0; j < n; ++j) c[r * n + j] = (float)acc[j];
    }
    free(acc);
  }
}

/* ---- SDDMM: x is M x K, y is N x K, both row-major -------------------- */
void oracle_sddmm_dot2(int64_t m, int64_t kdim, const int64_t* ptr, const int32_t* idx, const double* x,
                       const double* y, const double* in, double alpha, double beta, double* out, int nthreads) {
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t r = 0; r < m; ++r) {
    const double* xr = x + r * kdim;
    for (int64_t p = ptr[r]; p < ptr[r + 1]; ++p) {
      const double* yr = y + (int64_t)idx[p] * kdim;
      dd acc = {0.0, 0.0};
      for (int64_t k = 0; k < kdim; ++k) dd_add_prod(&acc, xr[k], yr[k]);
      double v = alpha * dd_val(acc);
      if (in) v += beta * in[p];
      out[p] = v;
    }
  }
}

/* ---- transpose (stable counting sort by column) ---------------------- */
void oracle_transpose(int64_t m, int64_t n, const int64_t* ptr, const int32_t* idx, int64_t* t_ptr, int32_t* t_idx,
                      int64_t* perm) {
  memset(t_ptr, 0, sizeof(int64_t) * (size_t)(n + 1));
  const int64_t nnz = ptr[m];
  for (int64_t k = 0; k < nnz; ++k) t_ptr[idx[k] + 1] += 1;
  for (int64_t c = 0; c < n; ++c) t_ptr[c + 1] += t_ptr[c];
  int64_t* cursor = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
  for (int64_t c = 0; c < n; ++c) cursor[c] = t_ptr[c];
  for (int64_t r = 0; r < m; ++r) {
    for (int64_t k = ptr[r]; k < ptr[r + 1]; ++k) {
      int64_t dst = cursor[idx[k]]++;
      t_idx[dst] = (int32_t)r;
      perm[dst] = k;
    }
  }
  free(cursor);
}

/* ---- COO -> CSR (stable order by (row, col)) ------------------------- */
void oracle_coo_to_csr(int64_t m, int64_t n, int64_t nnz, const int64_t* row, const int64_t* col, int64_t* ptr,
                       int32_t* idx, int64_t* perm) {
  int64_t* tmp = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nnz > 0 ? nnz : 1));
  int64_t* cur = (int64_t*)calloc((size_t)(n + 1), sizeof(int64_t));
  /* pass 1: stable counting sort of the positions by column */
  for (int64_t k = 0; k < nnz; ++k) cur[col[k] + 1] += 1;
  for (int64_t c = 0; c < n; ++c) cur[c + 1] += cur[c];
  for (int64_t k = 0; k < nnz; ++k) tmp[cur[col[k]]++] = k;
  free(cur);
  /* pass 2: stable counting sort of that order by row; ptr = bincount + cumsum */
  memset(ptr, 0, sizeof(int64_t) * (size_t)(m + 1));
  for (int64_t k = 0; k < nnz; ++k) ptr[row[k] + 1] += 1;
  for (int64_t r = 0; r < m; ++r) ptr[r + 1] += ptr[r];
  int64_t* rc = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m > 0 ? m : 1));
  for (int64_t r = 0; r < m; ++r) rc[r] = ptr[r];
  for (int64_t j = 0; j < nnz; ++j) {
    const int64_t k = tmp[j];
    const int64_t dst = rc[row[k]]++;
    perm[dst] = k;
    idx[dst] = (int32_t)col[k];
  }
  free(rc);
  free(tmp);
}

/* ---- stable bucketing ------------------------------------------------- */
void oracle_bucketize(int64_t m, const int64_t* ptr, const int64_t* ub, int nb, int32_t* rows, int64_t* counts) {
  for (int b = 0; b < nb; ++b) counts[b] = 0;
  int64_t off = 0;
  for (int b = 0; b < nb; ++b) {
    int64_t lo = b == 0 ? -1 : ub[b - 1];
    for (int64_t r = 0; r < m; ++r) {
      int64_t len = ptr[r + 1] - ptr[r];
      int in_b = (ub[b] < 0 || len <= ub[b]) && len > lo;
      if (in_b) { rows[off++] = (int32_t)r; counts[b] += 1; }
    }
  }
}

/* ---- SpMV unit plan (segments, units) -------------------------------- */
/* totals[0] = segments, totals[1] = units, totals[2] = scratch slots,
 * totals[3] = row-block units (they precede the long-row chunks); arrays may
 * be NULL (count only).  Unit descriptors (when `units` != NULL) are 6
 * int64 per unit: nnz_begin, nnz_end, row, tag, n_chunks, slot (tag >= 0: row
 * block ending before row `tag`; tag < 0: chunk -(tag+1) of a long row; slot
 * numbers the chunks of rows of >= 2 chunks consecutively, -1 elsewhere). */
/* One sweep over the rows.  With nb >= 0 it writes: row-block units take
 * indices [0, nb) in row order, long-row chunks [nb, nb + long units) in row
 * order.  Returns the counts in out[0..3] = segments, row-block units, slots,
 * long-row chunks. */
static void spmv_plan_sweep(int64_t m, const int64_t* ptr, int64_t cap, int64_t chunk, int64_t nb, int32_t* seg_row0,
                            int32_t* seg_unit0, int64_t* units, int64_t* out) {
  int64_t s = 0, rb = 0, lg = 0, sl = 0;
  int64_t prev_start = -1;
  for (int64_t r = 0; r <= m; ++r) {
    int start = 0;
    if (r < m) {
      int64_t len = ptr[r + 1] - ptr[r];
      int is_long = len > cap;
      if (r == 0 || is_long) {
        start = 1;
      } else {
        int64_t plen = ptr[r] - ptr[r - 1];
        start = plen > cap || ((ptr[r - 1] + r - 1) / cap != (ptr[r] + r) / cap);
      }
    }
    if (r == m || start) {
      /* close the previous segment [prev_start, r) */
      if (prev_start >= 0) {
        int64_t r0 = prev_start;
        int64_t len0 = ptr[r0 + 1] - ptr[r0];
        if (r - r0 == 1 && len0 > cap) {
          int64_t nch = (len0 + chunk - 1) / chunk;
          if (nb >= 0) {
            if (seg_unit0) seg_unit0[s - 1] = (int32_t)(nb + lg);
            for (int64_t k = 0; k < nch && units; ++k) {
              int64_t* d = units + 6 * (nb + lg + k);
              d[0] = ptr[r0] + k * chunk;
              d[1] = ptr[r0] + ((k + 1) * chunk < len0 ? (k + 1) * chunk : len0);
              d[2] = r0;
              d[3] = -(k + 1);
              d[4] = nch;
              d[5] = nch > 1 ? sl + k : -1;
            }
          }
          lg += nch;
          if (nch > 1) sl += nch;
        } else {
          if (nb >= 0) {
            if (seg_unit0) seg_unit0[s - 1] = (int32_t)rb;
            if (units) {
              int64_t* d = units + 6 * rb;
              d[0] = ptr[r0];
              d[1] = ptr[r];
              d[2] = r0;
              d[3] = r;
              d[4] = 1;
              d[5] = -1;
            }
          }
          rb += 1;
        }
      }
      if (r < m) {
        if (nb >= 0 && seg_row0) seg_row0[s] = (int32_t)r;
        s += 1;
        prev_start = r;
      }
    }
  }
  if (nb >= 0) {
    if (seg_row0) seg_row0[s] = (int32_t)m;
    if (seg_unit0) seg_unit0[s] = (int32_t)(rb + lg);
  }
  out[0] = s;
  out[1] = rb;
  out[2] = sl;
  out[3] = lg;
}

void oracle_spmv_plan(int64_t m, const int64_t* ptr, int64_t cap, int64_t chunk, int64_t* totals, int32_t* seg_row0,
                      int32_t* seg_unit0, int64_t* units) {
  int64_t cnt[4];
  spmv_plan_sweep(m, ptr, cap, chunk, -1, NULL, NULL, NULL, cnt);
  if (seg_row0 || seg_unit0 || units) spmv_plan_sweep(m, ptr, cap, chunk, cnt[1], seg_row0, seg_unit0, units, cnt);
  totals[0] = cnt[0];
  totals[1] = cnt[1] + cnt[3];
  totals[2] = cnt[2];
  totals[3] = cnt[1];
}
