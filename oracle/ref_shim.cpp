// C-ABI shim over the reference's own CPU pipeline, compiled together with the reference
// sources into oracle/_ref/libglu_ref.so.  TEST INFRASTRUCTURE ONLY: the parity tests, smoke()
// and bench.py's CPU-baseline leg call it as the checker; the product never links it.
//
// What it exposes, each a thin wrapper around the reference's own code path:
//   ref_open            -> preprocess()                 src/preprocess/preprocess.c:102-158
//                          (NicsLU_Initialize/ReadTriplet/CreateMatrix/Analyze + my_DumpA)
//   ref_symbolic        -> Symbolic_Matrix::fill_in, csr, predictLU, leveling
//                          src/symbolic.cc:11-151 (REAL forced to double by real_double.h)
//   ref_solve           -> Symbolic_Matrix::solve       src/symbolic.cc:200-248
//   ref_nicslu_*        -> NicsLU_Factorize / NicsLU_ReFactorize(_MT) / NicsLU_Solve /
//                          NicsLU_Residual              include/nicslu.h:150-290
// The reference's lu_cmd.cpp:64-111 runs exactly this sequence with LUonDevice in the middle.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unistd.h>
#include <iostream>
#include <streambuf>
#include <vector>

#include "symbolic.h"
#include "preprocess.h"
#include "nicslu.h"

namespace {
struct NullBuf : std::streambuf {
  int overflow(int c) override { return c; }
};
NullBuf g_nullbuf;
std::ostream g_null(&g_nullbuf);

struct RefHandle {
  SNicsLU* nicslu = nullptr;
  double* ax = nullptr;      // preprocessed CSC (my_DumpA output)
  unsigned* ai = nullptr;
  unsigned* ap = nullptr;
  unsigned n = 0, nnz = 0;
  std::vector<int> pivot_identity;   // Symbolic_Matrix::solve reads nicslu->pivot
  Symbolic_Matrix* sym = nullptr;
  bool factorized = false;
};
}  // namespace

extern "C" {

void* ref_open(const char* mtx_path, int quiet) {
  RefHandle* h = new RefHandle();
  h->nicslu = (SNicsLU*)malloc(sizeof(SNicsLU));
  FILE* saved = nullptr;
  fflush(stdout);
  int fd_saved = -1;
  if (quiet) {
    fd_saved = dup(fileno(stdout));
    saved = freopen("/dev/null", "w", stdout);
  }
  int err = preprocess((char*)mtx_path, h->nicslu, &h->ax, &h->ai, &h->ap);
  if (quiet) {
    fflush(stdout);
    dup2(fd_saved, fileno(stdout));
    close(fd_saved);
    (void)saved;
  }
  if (err) {  // preprocess() already freed nicslu and the arrays on failure
    h->nicslu = nullptr;
    h->ax = nullptr; h->ai = nullptr; h->ap = nullptr;
    delete h;
    return nullptr;
  }
  h->n = h->nicslu->n;
  h->nnz = h->nicslu->nnz;
  h->pivot_identity.assign(h->nicslu->pivot, h->nicslu->pivot + h->n);
  return h;
}

int ref_dims(void* hv, unsigned* n, unsigned* nnz) {
  RefHandle* h = (RefHandle*)hv;
  *n = h->n;
  *nnz = h->nnz;
  return 0;
}

int ref_get_preprocessed(void* hv, double* ax, unsigned* ai, unsigned* ap) {
  RefHandle* h = (RefHandle*)hv;
  memcpy(ax, h->ax, sizeof(double) * h->nnz);
  memcpy(ai, h->ai, sizeof(unsigned) * h->nnz);
  memcpy(ap, h->ap, sizeof(unsigned) * (h->n + 1));
  return 0;
}

// Permutations and MC64 scalings that NicsLU_Analyze produced (names as in SNicsLU).
int ref_get_perm(void* hv, unsigned* row_perm, unsigned* row_perm_inv, unsigned* col_perm,
                 unsigned* col_perm_inv, double* row_scale, double* col_scale_perm,
                 unsigned* mc64_scale) {
  RefHandle* h = (RefHandle*)hv;
  SNicsLU* s = h->nicslu;
  memcpy(row_perm, s->row_perm, sizeof(unsigned) * h->n);
  memcpy(row_perm_inv, s->row_perm_inv, sizeof(unsigned) * h->n);
  memcpy(col_perm, s->col_perm, sizeof(unsigned) * h->n);
  memcpy(col_perm_inv, s->col_perm_inv, sizeof(unsigned) * h->n);
  memcpy(row_scale, s->row_scale, sizeof(double) * h->n);
  memcpy(col_scale_perm, s->col_scale_perm, sizeof(double) * h->n);
  *mc64_scale = s->cfgi[1];
  return 0;
}

// Runs the reference symbolic analysis on the preprocessed matrix (lu_cmd.cpp:78-96).
int ref_symbolic(void* hv, unsigned* nnz_lu, int* num_lev) {
  RefHandle* h = (RefHandle*)hv;
  delete h->sym;
  h->sym = new Symbolic_Matrix(h->n, g_null, g_null);
  h->sym->fill_in(h->ai, h->ap);
  h->sym->csr();
  h->sym->predictLU(h->ai, h->ap, h->ax);
  h->sym->leveling();
  *nnz_lu = h->sym->nnz;
  *num_lev = h->sym->num_lev;
  return 0;
}

int ref_sym_get(void* hv, unsigned* sym_c_ptr, unsigned* sym_r_idx, unsigned* l_col_ptr,
                unsigned* csr_r_ptr, unsigned* csr_c_idx, unsigned* csr_diag_ptr,
                int* level_ptr, int* level_idx, double* val) {
  RefHandle* h = (RefHandle*)hv;
  Symbolic_Matrix* m = h->sym;
  if (!m) return -1;
  const unsigned n = m->n, nnz = m->nnz;
  memcpy(sym_c_ptr, m->sym_c_ptr.data(), sizeof(unsigned) * (n + 1));
  memcpy(sym_r_idx, m->sym_r_idx.data(), sizeof(unsigned) * nnz);
  memcpy(l_col_ptr, m->l_col_ptr.data(), sizeof(unsigned) * n);
  memcpy(csr_r_ptr, m->csr_r_ptr.data(), sizeof(unsigned) * (n + 1));
  memcpy(csr_c_idx, m->csr_c_idx.data(), sizeof(unsigned) * nnz);
  memcpy(csr_diag_ptr, m->csr_diag_ptr.data(), sizeof(unsigned) * n);
  memcpy(level_ptr, m->level_ptr.data(), sizeof(int) * (m->num_lev + 1));
  memcpy(level_idx, m->level_idx.data(), sizeof(int) * n);
  memcpy(val, m->val.data(), sizeof(double) * nnz);
  return 0;
}

// Replaces A_sym.val (e.g. with factored values) so ref_solve runs on them.
int ref_sym_set_val(void* hv, const double* val) {
  RefHandle* h = (RefHandle*)hv;
  if (!h->sym) return -1;
  memcpy(h->sym->val.data(), val, sizeof(double) * h->sym->nnz);
  return 0;
}

// Symbolic_Matrix::solve with REAL=double, as lu_cmd.cpp:110-111 calls it.
int ref_solve(void* hv, const double* rhs, double* x) {
  RefHandle* h = (RefHandle*)hv;
  if (!h->sym) return -1;
  int* saved = h->nicslu->pivot;
  h->nicslu->pivot = h->pivot_identity.data();   // preprocess.c:47-51 leaves pivot = identity
  std::vector<REAL> b(rhs, rhs + h->n);
  std::vector<REAL> xv = h->sym->solve(h->nicslu, b);
  h->nicslu->pivot = saved;
  memcpy(x, xv.data(), sizeof(double) * h->n);
  return 0;
}

// ---- NICSLU's own CPU LU: the host-side factorization timed as the CPU baseline ----
int ref_nicslu_factorize(void* hv) {
  RefHandle* h = (RefHandle*)hv;
  int r = NicsLU_Factorize(h->nicslu);
  if (r >= 0) h->factorized = true;
  return r;
}

int ref_nicslu_create_threads(void* hv, unsigned threads) {
  RefHandle* h = (RefHandle*)hv;
  int r = NicsLU_CreateScheduler(h->nicslu);
  if (r < 0) return r;
  return NicsLU_CreateThreads(h->nicslu, threads, 1);
}

// ax_orig: new values in the ORIGINAL (unpermuted, unscaled) CSC order of the file.
int ref_nicslu_refactorize(void* hv, const double* ax_orig, int multithreaded) {
  RefHandle* h = (RefHandle*)hv;
  if (multithreaded) return NicsLU_ReFactorize_MT(h->nicslu, (double*)ax_orig);
  return NicsLU_ReFactorize(h->nicslu, (double*)ax_orig);
}

int ref_nicslu_solve(void* hv, double* rhs_inout) {
  RefHandle* h = (RefHandle*)hv;
  return NicsLU_Solve(h->nicslu, rhs_inout);
}

double ref_nicslu_stat(void* hv, int i) {
  RefHandle* h = (RefHandle*)hv;
  return h->nicslu->stat[i];
}

size_t ref_nicslu_lu_nnz(void* hv) {
  RefHandle* h = (RefHandle*)hv;
  return h->nicslu->lu_nnz;
}

void ref_close(void* hv) {
  RefHandle* h = (RefHandle*)hv;
  if (!h) return;
  delete h->sym;
  if (h->nicslu) {
    NicsLU_Destroy(h->nicslu);
    free(h->nicslu);
  }
  free(h->ax);
  free(h->ai);
  free(h->ap);
  delete h;
}

}  // extern "C"
