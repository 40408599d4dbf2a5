/* CPU restatement of the GLU numeric phase, FP64 -- see glu_oracle.h.
 * TEST INFRASTRUCTURE ONLY (the checker for the CUDA path); compiled with -ffp-contract=off so
 * every multiply-add rounds twice, as the reference's separate multiply and atomicAdd do. */
#include "glu_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>

/* Position of row `r` inside column j, whose sorted rows are sym_r_idx[lo..hi). */
static uint32_t find_row(const uint32_t* ri, uint32_t lo, uint32_t hi, uint32_t r) {
  while (lo < hi) {
    uint32_t mid = lo + (hi - lo) / 2;
    if (ri[mid] < r) lo = mid + 1; else hi = mid;
  }
  return lo;
}

/* numeric.cu:51-89 for one sub-column j of U(c,:): column j receives -L(:,c) * U(c,j). */
static void update_subcolumn(const uint32_t* cp, const uint32_t* ri, double* val, uint32_t c,
                             uint32_t l0, uint32_t l1, uint32_t j) {
  uint32_t k = find_row(ri, cp[j], cp[j + 1], c);
  const double u = val[k];
  ++k;
  for (uint32_t p = l0; p < l1; ++p) {
    const uint32_t r = ri[p];
    while (ri[k] < r) ++k;          /* L(:,c) rows are a subset of column j's rows */
    val[k] += -(val[p] * u);
  }
}

/* Workers of oracle_factor_mt: per parallel pivot column, worker w takes every threads-th
 * sub-column starting at w; two barriers bracket each column. */
typedef struct {
  const uint32_t *cp, *ri, *ci;
  double* val;
  uint32_t c, l0, l1;
  int64_t s0, s1;
  int threads, quit;
  pthread_barrier_t start, done;
} mt_pool;

typedef struct {
  mt_pool* pool;
  int w;
} mt_arg;

static void mt_share(mt_pool* P, int w) {
  for (int64_t s = P->s0 + w; s < P->s1; s += P->threads)
    update_subcolumn(P->cp, P->ri, P->val, P->c, P->l0, P->l1, P->ci[s]);
}

static void* mt_worker(void* arg) {
  mt_arg* a = (mt_arg*)arg;
  mt_pool* P = a->pool;
  for (;;) {
    pthread_barrier_wait(&P->start);
    if (P->quit) break;
    mt_share(P, a->w);
    pthread_barrier_wait(&P->done);
  }
  return NULL;
}

int oracle_factor_mt(uint32_t n, const uint32_t* cp, const uint32_t* ri, const uint32_t* lp,
                     const uint32_t* rp, const uint32_t* ci, const uint32_t* dp, int num_lev,
                     const int* level_ptr, const int* level_idx, double* val, double pert,
                     int threads) {
  int status = 0;
  (void)n;
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  mt_pool P;
  P.cp = cp;
  P.ri = ri;
  P.ci = ci;
  P.val = val;
  P.threads = threads;
  P.quit = 0;
  pthread_t tid[256];
  mt_arg args[256];
  if (threads > 1) {
    pthread_barrier_init(&P.start, NULL, (unsigned)threads);
    pthread_barrier_init(&P.done, NULL, (unsigned)threads);
    for (int w = 1; w < threads; ++w) {
      args[w].pool = &P;
      args[w].w = w;
      pthread_create(&tid[w], NULL, mt_worker, &args[w]);
    }
  }
  for (int lev = 0; lev < num_lev; ++lev) {
    for (int q = level_ptr[lev]; q < level_ptr[lev + 1]; ++q) {
      const uint32_t c = (uint32_t)level_idx[q];
      const uint32_t l0 = lp[c] + 1, l1 = cp[c + 1];
      /* numeric.cu:37-47 (and :139-140 for the perturbed variant) */
      if (pert > 0.0 && l1 > l0 && fabs(val[lp[c]]) < pert) val[lp[c]] = pert;
      const double d = val[lp[c]];
      if (d == 0.0) status = -6;
      for (uint32_t p = l0; p < l1; ++p) val[p] /= d;
      /* numeric.cu:51-89: every sub-column j of U(c,:) receives -L(:,c) * U(c,j).  The
       * sub-columns are distinct targets (the reference gives each its own warp), so they may be
       * updated concurrently: every entry still receives its updates in the same order. */
      const int64_t s0 = (int64_t)dp[c] + 1, s1 = rp[c + 1];
      if (threads > 1 && s1 - s0 >= 8 && (int64_t)(l1 - l0) * (s1 - s0) >= 8192) {
        P.c = c;
        P.l0 = l0;
        P.l1 = l1;
        P.s0 = s0;
        P.s1 = s1;
        pthread_barrier_wait(&P.start);
        mt_share(&P, 0);
        pthread_barrier_wait(&P.done);
      } else {
        for (int64_t s = s0; s < s1; ++s) update_subcolumn(cp, ri, val, c, l0, l1, ci[s]);
      }
    }
  }
  if (threads > 1) {
    P.quit = 1;
    pthread_barrier_wait(&P.start);
    for (int w = 1; w < threads; ++w) pthread_join(tid[w], NULL);
    pthread_barrier_destroy(&P.start);
    pthread_barrier_destroy(&P.done);
  }
  return status;
}

int oracle_factor(uint32_t n, const uint32_t* cp, const uint32_t* ri, const uint32_t* lp,
                  const uint32_t* rp, const uint32_t* ci, const uint32_t* dp, int num_lev,
                  const int* level_ptr, const int* level_idx, double* val, double pert) {
  return oracle_factor_mt(n, cp, ri, lp, rp, ci, dp, num_lev, level_ptr, level_idx, val, pert, 1);
}

double oracle_perturbation(uint32_t n, const uint32_t* cp, const double* val) {
  double norm = 0.0;
  for (uint32_t i = 0; i < n; ++i) {
    double t = 0.0;
    for (uint32_t p = cp[i]; p < cp[i + 1]; ++p) t += fabs(val[p]);
    if (norm < t) norm = t;
  }
  return 3.45e-4 * norm;
}

void oracle_solve(uint32_t n, const uint32_t* cp, const uint32_t* ri, const uint32_t* lp,
                  const double* val, const uint32_t* col_perm, const uint32_t* row_perm_inv,
                  const double* col_scale_perm, const double* row_scale, int mc64_scale,
                  const double* rhs, double* x) {
  double* b = (double*)malloc(sizeof(double) * (n ? n : 1));
  /* symbolic.cc:211-219, with pivot = identity */
  for (uint32_t j = 0; j < n; ++j)
    b[j] = mc64_scale ? rhs[col_perm[j]] * col_scale_perm[j] : rhs[col_perm[j]];
  /* symbolic.cc:221-226: unit L, column oriented */
  for (uint32_t j = 0; j < n; ++j)
    for (uint32_t p = lp[j] + 1; p < cp[j + 1]; ++p) b[ri[p]] -= val[p] * b[j];
  /* symbolic.cc:228-236: U with the diagonal */
  for (int64_t jj = (int64_t)n - 1; jj >= 0; --jj) {
    b[jj] /= val[lp[jj]];
    for (uint32_t p = cp[jj]; p < lp[jj]; ++p) b[ri[p]] -= val[p] * b[jj];
  }
  /* symbolic.cc:238-245 */
  for (uint32_t j = 0; j < n; ++j)
    x[j] = mc64_scale ? b[row_perm_inv[j]] * row_scale[j] : b[row_perm_inv[j]];
  free(b);
}

void oracle_solve_transpose(uint32_t n, const uint32_t* cp, const uint32_t* ri,
                            const uint32_t* lp, const double* val, const uint32_t* col_perm,
                            const uint32_t* row_perm, const double* col_scale_perm,
                            const double* row_scale, int mc64_scale, const double* g,
                            double* lambda) {
  double* w = (double*)malloc(sizeof(double) * (n ? n : 1));
  /* g'[i] = row_scale[row_perm[i]] * g[row_perm[i]]  (transpose of symbolic.cc:238-245) */
  for (uint32_t i = 0; i < n; ++i)
    w[i] = mc64_scale ? row_scale[row_perm[i]] * g[row_perm[i]] : g[row_perm[i]];
  /* U^T z = g': row j of U^T is column j of U (rows < j, then the diagonal) */
  for (uint32_t j = 0; j < n; ++j) {
    double s = w[j];
    for (uint32_t p = cp[j]; p < lp[j]; ++p) s -= val[p] * w[ri[p]];
    w[j] = s / val[lp[j]];
  }
  /* L^T w = z: row j of L^T is column j of L (rows > j), unit diagonal */
  for (int64_t j = (int64_t)n - 1; j >= 0; --j) {
    double s = w[j];
    for (uint32_t p = lp[j] + 1; p < cp[j + 1]; ++p) s -= val[p] * w[ri[p]];
    w[j] = s;
  }
  /* lambda[col_perm[k]] = col_scale_perm[k] * w[k]  (transpose of symbolic.cc:211-219) */
  for (uint32_t k = 0; k < n; ++k)
    lambda[col_perm[k]] = mc64_scale ? col_scale_perm[k] * w[k] : w[k];
  free(w);
}

double oracle_residual(uint32_t n, const int64_t* ap, const int32_t* ai, const double* ax,
                       const double* x, const double* b) {
  double* r = (double*)calloc(n ? n : 1, sizeof(double));
  double* rowsum = (double*)calloc(n ? n : 1, sizeof(double));
  double xn = 0.0, bn = 0.0, an = 0.0, rn = 0.0;
  for (uint32_t j = 0; j < n; ++j) {
    for (int64_t p = ap[j]; p < ap[j + 1]; ++p) {
      r[ai[p]] += ax[p] * x[j];
      rowsum[ai[p]] += fabs(ax[p]);
    }
    if (fabs(x[j]) > xn) xn = fabs(x[j]);
  }
  for (uint32_t i = 0; i < n; ++i) {
    double d = fabs(r[i] - b[i]);
    if (d > rn || d != d) rn = d;
    if (fabs(b[i]) > bn) bn = fabs(b[i]);
    if (rowsum[i] > an) an = rowsum[i];
  }
  free(r);
  free(rowsum);
  return rn / (an * xn + bn);
}

double oracle_flops(uint32_t n, const uint32_t* cp, const uint32_t* lp, const uint32_t* rp,
                    const uint32_t* dp) {
  double f = 0.0;
  for (uint32_t c = 0; c < n; ++c) {
    double nl = (double)(cp[c + 1] - lp[c] - 1);
    double nu = (double)(rp[c + 1] - dp[c] - 1);
    f += nl + 2.0 * nl * nu;
  }
  return f;
}
