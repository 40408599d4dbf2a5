// lu_flow: the reference's lu_cmd flow (src/lu_cmd.cpp:64-111) with its two GPU-side calls,
// LUonDevice (:103) and Symbolic_Matrix::solve (:110-111), swapped for this library's C ABI,
// line for line as the integration guide shows a maintainer doing it.  TEST PROGRAM ONLY: built
// by oracle/Makefile (target `flow`) against the reference's own preprocess + Symbolic_Matrix
// objects in oracle/_ref, run by tests/test_gpu_lu_flow.py; nothing in the product links it.
//
//   lu_flow [-p] matrix.mtx out_prefix
// Runs preprocess -> fill_in -> csr -> predictLU -> leveling (the reference's code), then
//   glu_plan_create / glu_plan_set_solve_maps / glu_batch_create / glu_load_lu_values /
//   glu_refactor / glu_get_lu   (in place of LUonDevice: the factors land in A_sym.val)
//   glu_solve with b = 1        (in place of A_sym.solve(nicslu, b))
// and, as the check, the reference's own A_sym.solve(nicslu, b) on the GPU's factors.  Writes
// out_prefix.val (predictLU's values, LUonDevice's input), out_prefix.lu (the GPU factors),
// out_prefix.x_gpu and out_prefix.x_ref (raw doubles), and prints one summary line.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "glu_b200.h"
#include "nicslu.h"
#include "preprocess.h"
#include "symbolic.h"

namespace {

void check(int st, const char* what) {
  if (st != GLU_OK) {
    std::cerr << "lu_flow: " << what << ": " << glu_status_string(st) << ": " << glu_last_error()
              << "\n";
    exit(2);
  }
}

void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::cerr << "lu_flow: " << what << ": " << cudaGetErrorString(e) << "\n";
    exit(2);
  }
}

void dump(const std::string& path, const double* v, size_t n) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f || fwrite(v, sizeof(double), n, f) != n) {
    std::cerr << "lu_flow: cannot write " << path << "\n";
    exit(2);
  }
  fclose(f);
}

}  // namespace

int main(int argc, char** argv) {
  bool perturb = false;
  int a = 1;
  if (a < argc && !strcmp(argv[a], "-p")) perturb = true, ++a;
  if (argc - a != 2) {
    std::cerr << "usage: lu_flow [-p] matrix.mtx out_prefix\n";
    return 1;
  }
  char* matrix = argv[a];
  const std::string out = argv[a + 1];

  // ---- unchanged: src/lu_cmd.cpp:64-96 ----
  SNicsLU* nicslu = (SNicsLU*)malloc(sizeof(SNicsLU));
  double* ax = nullptr;
  unsigned *ai = nullptr, *ap = nullptr;
  if (preprocess(matrix, nicslu, &ax, &ai, &ap)) return 1;
  const unsigned n = nicslu->n;
  Symbolic_Matrix A_sym(n, std::cout, std::cerr);
  A_sym.fill_in(ai, ap);
  A_sym.csr();
  A_sym.predictLU(ai, ap, ax);
  A_sym.leveling();
  dump(out + ".val", A_sym.val.data(), A_sym.nnz);

  // ---- in place of LUonDevice(A_sym, cout, cerr, PERTURB) ----
  glu_plan_t plan;
  check(glu_plan_create(A_sym.n, A_sym.nnz, A_sym.sym_c_ptr.data(), A_sym.sym_r_idx.data(),
                        A_sym.l_col_ptr.data(), A_sym.csr_r_ptr.data(), A_sym.csr_c_idx.data(),
                        A_sym.csr_diag_ptr.data(), A_sym.num_lev, A_sym.level_ptr.data(),
                        A_sym.level_idx.data(), /*opt=*/nullptr, &plan),
        "glu_plan_create");
  // solve maps from NICSLU's analysis (what Symbolic_Matrix::solve reads, symbolic.cc:203-209)
  check(glu_plan_set_solve_maps(plan, nicslu->col_perm, nicslu->row_perm_inv,
                                nicslu->cfgi[1] ? nicslu->col_scale_perm : nullptr,
                                nicslu->cfgi[1] ? nicslu->row_scale : nullptr),
        "glu_plan_set_solve_maps");
  glu_batch_t batch;
  check(glu_batch_create(plan, 1, &batch), "glu_batch_create");
  double *val_dev, *b_dev, *x_dev;
  check_cuda(cudaMalloc(&val_dev, sizeof(double) * A_sym.nnz), "cudaMalloc");
  check_cuda(cudaMemcpy(val_dev, A_sym.val.data(), sizeof(double) * A_sym.nnz,
                        cudaMemcpyHostToDevice), "copy val");
  check(glu_load_lu_values(batch, 0, 1, val_dev, nullptr), "glu_load_lu_values");
  check(glu_refactor(batch, perturb ? -1.0 : 0.0, nullptr), "glu_refactor");
  check(glu_get_lu(batch, 0, val_dev, nullptr), "glu_get_lu");
  check_cuda(cudaMemcpy(A_sym.val.data(), val_dev, sizeof(double) * A_sym.nnz,
                        cudaMemcpyDeviceToHost), "copy L/U");
  int32_t flags = 0;
  check(glu_batch_status(batch, &flags, nullptr), "glu_batch_status");
  dump(out + ".lu", A_sym.val.data(), A_sym.nnz);

  // ---- in place of A_sym.solve(nicslu, b), b = 1 (lu_cmd.cpp:109-111) ----
  std::vector<double> b(n, 1.0), x(n);
  check_cuda(cudaMalloc(&b_dev, sizeof(double) * n), "cudaMalloc");
  check_cuda(cudaMalloc(&x_dev, sizeof(double) * n), "cudaMalloc");
  check_cuda(cudaMemcpy(b_dev, b.data(), sizeof(double) * n, cudaMemcpyHostToDevice), "copy b");
  check(glu_solve(batch, 1, b_dev, x_dev, /*transpose=*/0, nullptr), "glu_solve");
  check_cuda(cudaMemcpy(x.data(), x_dev, sizeof(double) * n, cudaMemcpyDeviceToHost), "copy x");
  dump(out + ".x_gpu", x.data(), n);

  // ---- the check: the reference's own solve on the factors the GPU produced ----
  std::vector<REAL> xr = A_sym.solve(nicslu, std::vector<REAL>(n, 1.0));
  dump(out + ".x_ref", xr.data(), n);
  double dmax = 0.0, xmax = 0.0;
  for (unsigned i = 0; i < n; ++i) {
    dmax = std::fmax(dmax, std::fabs(x[i] - xr[i]));
    xmax = std::fmax(xmax, std::fabs(xr[i]));
  }
  printf("lu_flow n=%u nnz_lu=%u levels=%d flags=%d max|x_gpu-x_ref|/max|x_ref|=%.3e\n", n,
         A_sym.nnz, A_sym.num_lev, flags, xmax > 0 ? dmax / xmax : dmax);

  cudaFree(val_dev);
  cudaFree(b_dev);
  cudaFree(x_dev);
  glu_batch_destroy(batch);
  glu_plan_destroy(plan);
  NicsLU_Destroy(nicslu);
  free(nicslu);
  free(ax);
  free(ai);
  free(ap);
  return 0;
}
