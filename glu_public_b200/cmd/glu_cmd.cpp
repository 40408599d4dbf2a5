// glu_cmd: the C++ driver of this library, in the shape of the reference's lu_cmd
// (src/lu_cmd.cpp:25-118): read a matrix, run the symbolic analysis, factor it on the GPU,
// solve A x = A * 1 and report the residual and the time of each stage.  Where lu_cmd runs
// NICSLU's MC64 / AMD preprocessing first, this driver factors the matrix as given (rows and
// columns already ordered and scaled by the caller, every diagonal entry structurally present),
// so it uses only the C ABI of include/glu_b200.h and the CUDA runtime.
//
//   glu_cmd [-p] [-r refine_steps] [-s analysis_file] matrix.mtx
//     -p  perturb tiny pivots (pert = 3.45e-4 * ||A||_1, as lu_cmd -p)
//     -r  rounds of iterative refinement after the solve (default 1)
//     -s  keep the symbolic analysis in this file (load it if it matches the matrix)
//     -o  only write the matrix as read (column-sorted 1-based real general, %.17g) to this
//         file and exit: symmetric and skew-symmetric input mirrored, duplicates summed
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "glu_b200.h"

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

void check(int st, const char* what) {
  if (st != GLU_OK) {
    fprintf(stderr, "glu_cmd: %s failed: %s (%d): %s\n", what, glu_status_string(st), st,
            glu_last_error());
    exit(2);
  }
}

void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    fprintf(stderr, "glu_cmd: %s failed: %s\n", what, cudaGetErrorString(e));
    exit(2);
  }
}

// MatrixMarket `coordinate` matrix, square, with field real / integer / pattern (values 1) and
// symmetry general / symmetric (the stored triangle mirrored) / skew-symmetric (mirrored with
// the sign flipped); a file without the banner line is read as real general.  Entries in any
// order; duplicates are summed.  CSC with sorted rows.  Any other banner (array format, complex,
// hermitian, an unknown word) is rejected, so a file is never read as something it is not.
bool read_mtx(const char* path, uint32_t& n, std::vector<uint32_t>& ap, std::vector<uint32_t>& ai,
              std::vector<double>& ax) {
  std::ifstream f(path);
  if (!f) return false;
  std::string line;
  std::string field = "real", symmetry = "general";
  bool first = true;
  while (std::getline(f, line)) {
    std::string tok[5];
    if (first) {
      std::istringstream ss(line);
      for (auto& t : tok) {
        ss >> t;
        for (auto& ch : t) ch = (char)tolower(ch);
      }
    }
    if (first && tok[0] == "%%matrixmarket") {
      // %%MatrixMarket matrix <format> <field> <symmetry>, compared token by token
      if (tok[1] != "matrix" || tok[2] != "coordinate") return false;
      field = tok[3];
      symmetry = tok[4];
      if (field != "real" && field != "integer" && field != "pattern") return false;
      if (symmetry != "general" && symmetry != "symmetric" && symmetry != "skew-symmetric")
        return false;
      first = false;
      continue;
    }
    first = false;
    if (line.empty() || line[0] == '%') continue;
    break;
  }
  const bool mirror = symmetry != "general";
  const double msign = symmetry == "skew-symmetric" ? -1.0 : 1.0;
  const bool pattern = field == "pattern";
  uint64_t m = 0, nn = 0, nnz = 0;
  if (!(std::istringstream(line) >> m >> nn >> nnz) || m != nn || m == 0) return false;
  n = (uint32_t)m;
  std::vector<std::pair<uint64_t, double>> ent;   // key = col * n + row
  ent.reserve(nnz * (mirror ? 2 : 1));
  for (uint64_t e = 0; e < nnz; ++e) {
    uint64_t r, c;
    double v = 1.0;
    if (!(f >> r >> c) || (!pattern && !(f >> v)) || r < 1 || c < 1 || r > m || c > m)
      return false;
    ent.push_back({(c - 1) * m + (r - 1), v});
    if (mirror && r != c) ent.push_back({(r - 1) * m + (c - 1), msign * v});
  }
  std::stable_sort(ent.begin(), ent.end(),
                   [](const auto& a, const auto& b) { return a.first < b.first; });
  ap.assign(n + 1, 0);
  for (size_t e = 0; e < ent.size(); ++e) {
    if (e > 0 && ent[e].first == ent[e - 1].first) {
      ax.back() += ent[e].second;
      continue;
    }
    ai.push_back((uint32_t)(ent[e].first % m));
    ax.push_back(ent[e].second);
    ap[ent[e].first / m + 1]++;
  }
  for (uint32_t j = 0; j < n; ++j) ap[j + 1] += ap[j];
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  bool perturb = false;
  int refine = 1;
  const char* sym_file = nullptr;
  const char* out_file = nullptr;
  const char* path = nullptr;
  for (int i = 1; i < argc; ++i) {
    if (!strcmp(argv[i], "-p")) perturb = true;
    else if (!strcmp(argv[i], "-r") && i + 1 < argc) refine = atoi(argv[++i]);
    else if (!strcmp(argv[i], "-s") && i + 1 < argc) sym_file = argv[++i];
    else if (!strcmp(argv[i], "-o") && i + 1 < argc) out_file = argv[++i];
    else if (!strcmp(argv[i], "-h") || !strcmp(argv[i], "--help")) path = nullptr, argc = 0;
    else path = argv[i];
  }
  if (!path) {
    printf("usage: glu_cmd [-p] [-r refine_steps] [-s analysis_file] [-o out.mtx] matrix.mtx\n");
    return argc == 0 ? 0 : 1;
  }
  uint32_t n = 0;
  std::vector<uint32_t> ap, ai;
  std::vector<double> ax;
  double t0 = now_s();
  if (!read_mtx(path, n, ap, ai, ax)) {
    fprintf(stderr, "glu_cmd: cannot read %s as a square MatrixMarket coordinate matrix\n", path);
    return 1;
  }
  const uint32_t nnz_a = ap[n];
  printf("matrix: n = %u, nnz = %u (read %.3f s)\n", n, nnz_a, now_s() - t0);
  if (out_file) {
    FILE* fo = fopen(out_file, "w");
    if (!fo) {
      fprintf(stderr, "glu_cmd: cannot write %s\n", out_file);
      return 1;
    }
    fprintf(fo, "%%%%MatrixMarket matrix coordinate real general\n%u %u %u\n", n, n, nnz_a);
    for (uint32_t j = 0; j < n; ++j)
      for (uint32_t e = ap[j]; e < ap[j + 1]; ++e)
        fprintf(fo, "%u %u %.17g\n", ai[e] + 1, j + 1, ax[e]);
    fclose(fo);
    return 0;
  }

  // symbolic analysis (Symbolic_Matrix::fill_in + csr + leveling), kept in a file if asked
  t0 = now_s();
  glu_symbolic_t sym = nullptr;
  bool loaded = sym_file && glu_symbolic_load(sym_file, n, ap.data(), ai.data(), &sym) == GLU_OK;
  if (!loaded) {
    check(glu_symbolic_create(n, ap.data(), ai.data(), &sym), "symbolic analysis");
    if (sym_file) check(glu_symbolic_save(sym, sym_file), "saving the analysis");
  }
  uint32_t nnz = 0;
  int32_t num_lev = 0;
  check(glu_symbolic_sizes(sym, &nnz, &num_lev), "symbolic sizes");
  std::vector<uint32_t> cp(n + 1), ri(nnz), lp(n), rp(n + 1), ci(nnz), dp(n);
  std::vector<int32_t> lev_ptr(num_lev + 1), lev_idx(n);
  check(glu_symbolic_get(sym, cp.data(), ri.data(), lp.data(), rp.data(), ci.data(), dp.data(),
                         lev_ptr.data(), lev_idx.data()),
        "symbolic arrays");
  std::vector<int64_t> pos(nnz_a);
  check(glu_symbolic_positions(sym, ap.data(), ai.data(), pos.data()), "entry positions");
  printf("symbolic: nnz(L+U) = %u, levels = %d (%s %.3f s)\n", nnz, num_lev,
         loaded ? "loaded in" : "analysed in", now_s() - t0);

  // plan, one-instance batch, values, refactorization (in place of LUonDevice)
  t0 = now_s();
  glu_plan_t plan = nullptr;
  check(glu_plan_create(n, nnz, cp.data(), ri.data(), lp.data(), rp.data(), ci.data(), dp.data(),
                        num_lev, lev_ptr.data(), lev_idx.data(), nullptr, &plan),
        "plan");
  check(glu_plan_set_ingest(plan, nnz_a, pos.data(), nullptr), "ingest map");
  std::vector<uint32_t> ident(n);
  std::iota(ident.begin(), ident.end(), 0u);
  check(glu_plan_set_solve_maps(plan, ident.data(), ident.data(), nullptr, nullptr), "solve maps");
  std::vector<uint32_t> rows(nnz_a), cols(nnz_a);
  for (uint32_t j = 0; j < n; ++j)
    for (uint32_t e = ap[j]; e < ap[j + 1]; ++e) rows[e] = ai[e], cols[e] = j;
  check(glu_plan_set_original_pattern(plan, nnz_a, rows.data(), cols.data()), "original pattern");
  glu_batch_t batch = nullptr;
  check(glu_batch_create(plan, 1, &batch), "batch");
  double plan_s = now_s() - t0;

  std::vector<double> b(n, 0.0), x(n);
  for (uint32_t j = 0; j < n; ++j)
    for (uint32_t e = ap[j]; e < ap[j + 1]; ++e) b[ai[e]] += ax[e];     // b = A * 1
  double *a_dev = nullptr, *b_dev = nullptr, *x_dev = nullptr, *r_dev = nullptr;
  check_cuda(cudaMalloc(&a_dev, sizeof(double) * nnz_a), "cudaMalloc");
  check_cuda(cudaMalloc(&b_dev, sizeof(double) * n), "cudaMalloc");
  check_cuda(cudaMalloc(&x_dev, sizeof(double) * n), "cudaMalloc");
  check_cuda(cudaMalloc(&r_dev, sizeof(double)), "cudaMalloc");
  check_cuda(cudaMemcpy(a_dev, ax.data(), sizeof(double) * nnz_a, cudaMemcpyHostToDevice),
             "copy A");
  check_cuda(cudaMemcpy(b_dev, b.data(), sizeof(double) * n, cudaMemcpyHostToDevice), "copy b");

  t0 = now_s();
  check(glu_load_values(batch, 0, 1, a_dev, nullptr), "load values");
  check(glu_refactor(batch, perturb ? -1.0 : 0.0, nullptr), "refactorization");
  check_cuda(cudaDeviceSynchronize(), "refactorization");
  const double fact_s = now_s() - t0;
  int32_t flags = 0;
  check(glu_batch_status(batch, &flags, nullptr), "status");

  // solve (in place of Symbolic_Matrix::solve) and refinement on the original matrix
  t0 = now_s();
  check(glu_solve(batch, 1, b_dev, x_dev, 0, nullptr), "solve");
  if (refine > 0)
    check(glu_refine(batch, 1, a_dev, b_dev, x_dev, refine, 0, r_dev, nullptr), "refinement");
  check_cuda(cudaDeviceSynchronize(), "solve");
  const double solve_s = now_s() - t0;
  check_cuda(cudaMemcpy(x.data(), x_dev, sizeof(double) * n, cudaMemcpyDeviceToHost), "copy x");

  // ||A x - b|| / (||A|| ||x|| + ||b||) on the host, max norms
  std::vector<double> r(b), rowsum(n, 0.0);
  for (uint32_t j = 0; j < n; ++j)
    for (uint32_t e = ap[j]; e < ap[j + 1]; ++e) {
      r[ai[e]] -= ax[e] * x[j];
      rowsum[ai[e]] += fabs(ax[e]);
    }
  double rn = 0, an = 0, xn = 0, bn = 0;
  for (uint32_t i = 0; i < n; ++i) {
    rn = std::max(rn, fabs(r[i]));
    an = std::max(an, rowsum[i]);
    xn = std::max(xn, fabs(x[i]));
    bn = std::max(bn, fabs(b[i]));
  }
  printf("plan + batch: %.3f s\n", plan_s);
  printf("numeric factorization: %.3f ms (status flags %d)\n", fact_s * 1e3, flags);
  printf("solve + %d refinement round(s): %.3f ms\n", refine, solve_s * 1e3);
  printf("residual ||Ax-b||/(||A|| ||x|| + ||b||) = %.3e\n", rn / (an * xn + bn));

  cudaFree(a_dev);
  cudaFree(b_dev);
  cudaFree(x_dev);
  cudaFree(r_dev);
  glu_batch_destroy(batch);
  glu_plan_destroy(plan);
  glu_symbolic_destroy(sym);
  return 0;
}
