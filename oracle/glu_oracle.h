/* CPU restatement of the GLU numeric phase, FP64.  TEST INFRASTRUCTURE ONLY: it is the checker
 * for the CUDA path (tests/, smoke(), bench.py's CPU-baseline leg); the product never calls it.
 *
 * Arrays are the reference's Symbolic_Matrix members (include/symbolic.h:9-24): filled CSC
 * `sym_c_ptr[n+1]`, `sym_r_idx[nnz]` (rows sorted), `l_col_ptr[n]` (diagonal position), CSR
 * mirror `csr_r_ptr[n+1]`, `csr_c_idx[nnz]`, `csr_diag_ptr[n]`, levels `level_ptr[num_lev+1]`,
 * `level_idx[n]`, values `val[nnz]`.
 *
 * Parity pin: its factor output is checked against the reference's own CPU code run in this
 * container (NICSLU preprocess + symbolic.cc + Symbolic_Matrix::solve, oracle/_ref) through
 * solve residuals, and its solve is checked bit-for-bit against Symbolic_Matrix::solve.
 */
#ifndef GLU_ORACLE_H
#define GLU_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Right-looking level-ordered LU in place (src/numeric.cu:28-89 for the per-column math,
 * src/numeric.cu:423-596 for the level order).  pert > 0 clamps |pivot| < pert to pert for
 * columns whose L part is non-empty (src/numeric.cu:139-140; the clamp sits inside the L loop).
 * Returns 0, or -6 (NICSLU_MATRIX_NUMERIC_SINGULAR) if a zero pivot was met. */
int oracle_factor(uint32_t n, const uint32_t* sym_c_ptr, const uint32_t* sym_r_idx,
                  const uint32_t* l_col_ptr, const uint32_t* csr_r_ptr,
                  const uint32_t* csr_c_idx, const uint32_t* csr_diag_ptr, int num_lev,
                  const int* level_ptr, const int* level_idx, double* val, double pert);

/* oracle_factor with the sub-columns j of each pivot column c updated by `threads` threads
 * (POSIX threads); every entry receives its updates in the same order, so the result is bit-identical
 * to oracle_factor's. */
int oracle_factor_mt(uint32_t n, const uint32_t* sym_c_ptr, const uint32_t* sym_r_idx,
                     const uint32_t* l_col_ptr, const uint32_t* csr_r_ptr,
                     const uint32_t* csr_c_idx, const uint32_t* csr_diag_ptr, int num_lev,
                     const int* level_ptr, const int* level_idx, double* val, double pert,
                     int threads);

/* 3.45e-4 * max column abs sum of val (src/numeric.cu:405-421). */
double oracle_perturbation(uint32_t n, const uint32_t* sym_c_ptr, const double* val);

/* Symbolic_Matrix::solve (src/symbolic.cc:200-248) in FP64, with pivot = identity
 * (src/preprocess/preprocess.c:47-51).  rhs, x: [n]. */
void oracle_solve(uint32_t n, const uint32_t* sym_c_ptr, const uint32_t* sym_r_idx,
                  const uint32_t* l_col_ptr, const double* val, const uint32_t* col_perm,
                  const uint32_t* row_perm_inv, const double* col_scale_perm,
                  const double* row_scale, int mc64_scale, const double* rhs, double* x);

/* Adjoint of oracle_solve: lambda = A^-T g (transposed U then L solve with the permutations and
 * scalings undone).  row_perm is the inverse of row_perm_inv. */
void oracle_solve_transpose(uint32_t n, const uint32_t* sym_c_ptr, const uint32_t* sym_r_idx,
                            const uint32_t* l_col_ptr, const double* val,
                            const uint32_t* col_perm, const uint32_t* row_perm,
                            const double* col_scale_perm, const double* row_scale,
                            int mc64_scale, const double* g, double* lambda);

/* ||A x - b||_inf / (||A||_inf ||x||_inf + ||b||_inf) for a CSC matrix (ap, ai, ax). */
double oracle_residual(uint32_t n, const int64_t* ap, const int32_t* ai, const double* ax,
                       const double* x, const double* b);

/* Algorithmic flop count sum_c (|L(:,c)| + 2 |L(:,c)| |U(c,:)|). */
double oracle_flops(uint32_t n, const uint32_t* sym_c_ptr, const uint32_t* l_col_ptr,
                    const uint32_t* csr_r_ptr, const uint32_t* csr_diag_ptr);

#ifdef __cplusplus
}
#endif
#endif
