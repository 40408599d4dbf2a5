// Kernel launch wrappers (host-callable), implemented in kernels.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>

#include "plan.h"

namespace glu {

struct LaunchCounter {
  int64_t n = 0;
};

// A batch of dense column-major matrices: instance b starts at base + b * stride; rows x cols
// (multiples of 64) with leading dimension ld; hasl[k] != 0 if pivot k may be perturbed.
struct DenseView {
  double* base;
  int64_t stride;
  int32_t ld;
  int32_t rows;
  int32_t cols;
  const uint8_t* hasl;
  int32_t nvalid;    // pivots [nvalid, padded count) are identity padding (zero off their diagonal)
};

// One front (see plan_host.h, Front), as the launch code needs it.
struct FrontDev {
  int32_t w, wp, ld, qp;
  int64_t size, g_off, g_cnt, c_off, c_cnt, h_off;
};

// value handling
// clears the value slots of instances [first, first + count); assemble: all but the dense block
// (which the pull then builds column by column), else everything, with identity padding
void launch_prepare_blob(const PlanDev& P, double* vals, int first, int count, bool assemble,
                         cudaStream_t s,
                         LaunchCounter& lc);
void launch_ingest(const PlanDev& P, double* vals, int first, int count, const double* a,
                   cudaStream_t s, LaunchCounter& lc);
void launch_load_lu(const PlanDev& P, double* vals, int first, int count, const double* val,
                    cudaStream_t s, LaunchCounter& lc);
void launch_export_lu(const PlanDev& P, const double* vals, int inst, double* val, cudaStream_t s,
                      LaunchCounter& lc);
void launch_pert(const PlanDev& P, const double* vals, int count, double pert, double* pert_dev,
                 cudaStream_t s, LaunchCounter& lc);

// factorization
// wpc warps per column (1, 2, 4, 8), cpw columns per warp group, `block` threads per CTA (128 or
// 256), `lanes` lanes per column when wpc = 1 (8, 16 or 32); `grow`: a wide level of heavy columns
// that may take more warps per column when the batch leaves the GPU short of `occ` warps per SM;
// levels with several warps per column that are too narrow to fill the GPU split each column's
// updates over several CTAs (needs max_nl, max_pairs)
void launch_sparse_level(const PlanDev& P, double* vals, int count, const double* pert,
                         int32_t* status, int begin, int ncols, int wpc, int max_nl,
                         int max_pairs, int block, int cpw, int lanes, int grow, int occ,
                         cudaStream_t s, LaunchCounter& lc);
// deterministic mode: a level's pivots and scaling (CTA per column), then its updates by one warp
// per target column (targets [t0, t1) of det_tptr) without atomics
void launch_sparse_level_det(const PlanDev& P, double* vals, int count, const double* pert,
                             int32_t* status, int begin, int ncols, int64_t t0, int64_t t1,
                             cudaStream_t s, LaunchCounter& lc);
// deterministic forward solves, one warp per row (which 0: L rows, 1: U rows; rows == nullptr:
// rows begin .. begin + nrows - 1)
void launch_rows_solve(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                       int64_t ylen, const int32_t* rows, int begin, int nrows, int which,
                       cudaStream_t s, LaunchCounter& lc);
// a run of consecutive sparse levels in one cooperative launch (k_sparse_persistent): desc[l] =
// {begin, ncols, mode (0 warp / 1 CTA per column, 3 split), splits}; bar: `groups` barrier
// counters and err: the failure word, both cleared by the launch; every device-side wait gives
// up after budget_ms (instances flagged GLU_INST_TIMEOUT, *err != 0).  persistent_grid: CTAs
// that fit on the device at once with `smem` bytes each (0 if none).
int persistent_grid(size_t smem);
void launch_sparse_persistent(const PlanDev& P, double* vals, int count, const double* pert,
                              int32_t* status, const int4* desc, int nlev, unsigned* bar,
                              int groups, int* err, double budget_ms, int extra, int grid,
                              size_t smem, cudaStream_t s, LaunchCounter& lc);
// dense phase (dense.cu)
int sm_count();
// raises `func`'s dynamic shared-memory limit to `bytes` on the current device (once per kernel
// and device; thread-safe)
void ensure_smem_limit(const void* func, size_t bytes);
void launch_dense_diag(const DenseView& V, int count, const double* pert, int32_t* status, int k,
                       int nb, cudaStream_t s, LaunchCounter& lc);
void launch_dense_trsm(const DenseView& V, int count, int k, int nb, cudaStream_t s,
                       LaunchCounter& lc);
void launch_dense_update(const DenseView& V, int count, int k, int nb, int variant, cudaStream_t s,
                         LaunchCounter& lc);
// LU of the first npiv pivots of the view in groups of `depth` panels of width nb;
// mark(phase, launches_before) after each panel (2), trailing update (3) and in-group update (6)
void launch_dense_factor(const DenseView& V, int count, const double* pert, int32_t* status,
                         int npiv, int nb, int depth, int variant, cudaStream_t s,
                         LaunchCounter& lc, const std::function<void(int, int64_t)>& mark);
// one front for every instance: assemble into F (count * fstride doubles), factor its pivots,
// write back and add its Schur complement
void launch_front(const PlanDev& P, const FrontDev& f, double* vals, int count, double* F,
                  int64_t fstride, const double* pert, int32_t* status, int nb, int depth,
                  int variant, cudaStream_t s, LaunchCounter& lc);
// every front of one level at once (see plan_host.h, FrontLevel), one launch per stage; usable
// when front_level_batched (64-wide panels, fronts * count within a grid dimension)
struct FrontLevel;
bool front_level_batched(const FrontLevel& L, int count, int nb);
void launch_front_level(const PlanDev& P, const FrontLevel& L, double* vals, int count, double* F,
                        int64_t fstride, const double* pert, int32_t* status, cudaStream_t s,
                        LaunchCounter& lc);
// gbuf: count * 2 * ntp * hubs_p doubles, zero outside the gathered entries
void launch_hub_update(const PlanDev& P, double* vals, int count, double* gbuf, int variant,
                       cudaStream_t s, LaunchCounter& lc);
// the dense block can be assembled by the pull (ingest map with per-column rows, block column
// fits in shared memory)
bool dense_assembly(const PlanDev& P);
// asm_flag[b] != 0: instance b's dense block is to be assembled (only read if dense_assembly(P))
// det: the pull entries of a column applied one after another (fixed summation order)
void launch_dense_pull(const PlanDev& P, double* vals, int count, const uint8_t* asm_flag,
                       bool det, cudaStream_t s, LaunchCounter& lc);
// DMMA GEMM C -= A*B, column-major, batched over `count` with element strides
// (M, K, lda, ldb, strides even; A, B 16-byte aligned).  variant: tile shape, see glu_options.
int gemm_variants();
void launch_gemm_sub(int M, int N, int K, const double* A, int lda, const double* B, int ldb,
                     double* C, int ldc, int count, int64_t strideA, int64_t strideB,
                     int64_t strideC, cudaStream_t s, LaunchCounter& lc, int variant);

// solves; y: [count][nrhs][ylen] workspace, ylen = n + (ntp - nt)
void launch_solve_permute_in(const PlanDev& P, int count, int nrhs, const double* B, double* y,
                             int64_t ylen, int transpose, cudaStream_t s, LaunchCounter& lc);
void launch_solve_permute_out(const PlanDev& P, int count, int nrhs, const double* y, double* X,
                              int64_t ylen, int transpose, cudaStream_t s, LaunchCounter& lc);
void launch_sparse_lsolve(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                          int64_t ylen, const int32_t* cols, int begin, int ncols,
                          cudaStream_t s, LaunchCounter& lc);
void launch_sparse_usolve(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                          int64_t ylen, const int32_t* cols, int begin, int ncols,
                          cudaStream_t s, LaunchCounter& lc);
void launch_sparse_utsolve(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                           int64_t ylen, const int32_t* cols, int begin, int ncols,
                           cudaStream_t s, LaunchCounter& lc);
void launch_sparse_ltsolve(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                           int64_t ylen, const int32_t* cols, int begin, int ncols,
                           cudaStream_t s, LaunchCounter& lc);
// fronts fids[0 .. nfronts) of one solve level, every vector (which as in k_front_solve)
// max_w: the widest of the fronts listed in fids (at least their width)
void launch_front_solve(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                        int64_t ylen, const int32_t* fids, int nfronts, int max_w, int which,
                        cudaStream_t s, LaunchCounter& lc);
void launch_border(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                   int64_t ylen, int transpose, cudaStream_t s, LaunchCounter& lc);
void launch_dense_trsv(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                       int64_t ylen, int which, cudaStream_t s, LaunchCounter& lc);
// r = b - op(A) x on the original matrix (R may be null) and per-vector norms; resid (may be
// null) receives ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf) per (instance, rhs)
void launch_residual(const PlanDev& P, int count, int nrhs, const double* a, const double* X,
                     const double* B, double* R, unsigned long long* norms, double* resid,
                     int transpose, cudaStream_t s, LaunchCounter& lc);
void launch_axpy(int64_t n, const double* dx, double* x, cudaStream_t s, LaunchCounter& lc);
void launch_grad(const PlanDev& P, int count, int nrhs, const double* lambda, const double* x,
                 double* ga, cudaStream_t s, LaunchCounter& lc);

}  // namespace glu
