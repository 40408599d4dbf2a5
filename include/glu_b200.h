/* glu_b200.h -- C ABI of the B200-native GLU numeric phase (FP64, sm_100a).
 *
 * Drop-in boundary.  The reference calls, after symbolic analysis,
 *     void LUonDevice(Symbolic_Matrix&, ostream&, ostream&, bool PERTURB)   include/numeric.h:6
 * (called from src/lu_cmd.cpp:103) and then the CPU solve
 *     std::vector<REAL> Symbolic_Matrix::solve(SNicsLU*, const std::vector<REAL>&)
 *                                                                          include/symbolic.h:29
 * (called from src/lu_cmd.cpp:111).  A caller replaces those two calls with
 *     glu_plan_create(...)   once per sparsity pattern (takes Symbolic_Matrix's arrays),
 *     glu_batch_create(...)  once per set of value instances,
 *     glu_load_values / glu_refactor / glu_solve / glu_get_lu
 * and keeps everything before them (NICSLU preprocess, Symbolic_Matrix) unchanged.
 *
 * Conventions
 *  - Every entry point returns int: 0 = OK, negative = error.  Codes -1..-16 reuse NICSLU's
 *    meaning (src/nicslu/include/nicslu.h:11-28); codes <= -100 are new.
 *  - Host pointers are plain host memory; "_dev" pointers are device memory on the plan's device.
 *  - Calls that take a `stream` (a cudaStream_t passed as void*, NULL = legacy default stream)
 *    only enqueue work; none of them synchronizes implicitly.
 *  - Handles are not thread-safe; distinct handles may be used from distinct threads/streams.
 *  - Index arrays are 32-bit, as in Symbolic_Matrix; value offsets inside the library are 64-bit.
 */
#ifndef GLU_B200_H
#define GLU_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define GLU_OK                          0
#define GLU_ARGUMENT_ERROR             (-2)   /* NICSLU_ARGUMENT_ERROR */
#define GLU_MEMORY_OVERFLOW            (-3)   /* NICSLU_MEMORY_OVERFLOW (device or host) */
#define GLU_FILE_CANNOT_OPEN           (-4)   /* NICSLU_FILE_CANNOT_OPEN (symbolic save / load) */
#define GLU_MATRIX_STRUCTURAL_SINGULAR (-5)   /* a column has no structural diagonal */
#define GLU_MATRIX_NUMERIC_SINGULAR    (-6)   /* zero pivot met (per-instance status) */
#define GLU_MATRIX_INVALID             (-7)   /* malformed CSC/CSR/level arrays */
#define GLU_MATRIX_ENTRY_DUPLICATED    (-8)   /* NICSLU_MATRIX_ENTRY_DUPLICATED */
#define GLU_NUMERIC_OVERFLOW           (-16)  /* NaN/Inf pivot (per-instance status) */
#define GLU_CUDA_ERROR                 (-100) /* a CUDA runtime call failed */
#define GLU_TIMEOUT                    (-101) /* a bounded device-side wait expired */
#define GLU_BUDGET_EXCEEDED            (-102) /* request exceeds the device memory budget */
#define GLU_NOT_READY                  (-103) /* call order violated (e.g. solve before refactor) */

/* per-instance status flags (bitwise OR), read with glu_batch_status */
#define GLU_INST_ZERO_PIVOT   1
#define GLU_INST_NAN_PIVOT    2
#define GLU_INST_PERTURBED    4
#define GLU_INST_TIMEOUT      8

typedef struct glu_symbolic_s* glu_symbolic_t;
typedef struct glu_plan_s* glu_plan_t;
typedef struct glu_batch_s* glu_batch_t;
typedef struct glu_group_s* glu_group_t;

/* Tuning knobs of a plan.  Zero-initialise and call glu_options_default, or pass NULL. */
typedef struct glu_options {
  double dense_threshold;     /* min density of the trailing block handled densely (default 0.9) */
  int32_t dense_min;          /* min order of a dense trailing block (default 128) */
  int32_t panel;              /* dense panel width nb: 64 or 128 (default 64) */
  int32_t sparse_warps_per_col; /* warps that share one column in the sparse level kernels:
                                   1, 2, 4 or 8 (8 = the whole CTA of 256 threads); 0 = by level:
                                   1 on wide levels, 8 on narrow ones (default 0) */
  int32_t sparse_cols_per_warp; /* columns one warp group takes in turn within a level launch
                                   (1, 2 or 4; default 1): fewer, longer-lived CTAs on levels of
                                   many small columns */
  int32_t gemm_variant;       /* DMMA GEMM variant 0..13: m8n8k4 tiles 0: 64x64 2-stage,
                                 1: 64x64, 2: 128x64, 3: 64x128, 4: 128x128 (3-stage);
                                 m16n8k8 tiles (2-stage) 5: 64x64, 6: 128x64, 7: 128x128,
                                 10: 64x128, and with C prefetched 8: 64x64, 9: 128x64;
                                 k-steps of 16 instead of 32: m8n8k4 64x64 11: 3-stage,
                                 12: 2-stage, m16n8k8 64x64 13: 3-stage (default 12) */
  int32_t deterministic;      /* 1: bit-identical results from run to run.  By default the
                                 sparse levels, the sparse-to-dense pull, the fronts and the
                                 forward solve add into shared targets with FP64 atomics, so
                                 sums may round differently from run to run; in this mode every
                                 target is owned by one warp or CTA that adds its contributions
                                 in a fixed order (each level's update pairs grouped by target
                                 column, row-wise forward solves), fronts and the cooperative
                                 level launch are off (default 0) */
  int32_t device;             /* CUDA device ordinal (default: current device) */
  double hub_min_frac;        /* sparse column joins the hub GEMM if |L21(:,c)||U12(c,:)| >=
                                 hub_min_frac * ntp^2 (default 0.02) */
  int32_t hub_max;            /* at most this many hub columns (default 256) */
  int32_t front_min_w;        /* supernodal runs of at least this many sparse columns become
                                 dense fronts (default 16; 0 disables fronts) */
  double front_min_flops;     /* ... if their update costs at least this many flops (1e6) */
  int32_t update_depth;       /* dense panels per trailing update: each group of this many panels
                                 is factored left-looking inside the group, then the rest of the
                                 block takes one update with K = update_depth * panel, so it is
                                 read and written once per group (1, 2, 4 or 8; default 8) */
  int32_t sparse_persistent;  /* runs of at least this many consecutive narrow sparse levels
                                 (at most two columns of the batch per SM) without
                                 fronts are factored by ONE cooperative launch that walks the
                                 levels with device-side barriers instead of one launch per
                                 level (0 = never; default 2) */
  double level_wait_ms;       /* bound of every device-side wait of that launch: a barrier not
                                 reached within it marks the instances GLU_INST_TIMEOUT and the
                                 launch returns (default 1000) */
  int32_t wide_level_cols;    /* a level of at least this many columns is "wide" (default 592 =
                                 4 x 148 SMs); with sparse_warps_per_col = 0 wide levels get one
                                 warp per column, narrow levels a CTA per column ... */
  int32_t narrow_col_work;    /* ... if their mean update work per column (|L| * |U| products)
                                 exceeds this (default 256) */
  int32_t sparse_block;       /* threads per CTA of the sparse level kernels: 128 or 256
                                 (default 256) */
  int32_t front_batch;        /* 1: all fronts of a level are assembled, factored and written back
                                 together, one launch per stage (default); 0: one launch chain per
                                 front, on up to four streams */
  int32_t sparse_col_lanes;   /* lanes that share one column on levels with a warp per column:
                                 32, 16 or 8 (several short columns per warp); 0 = by level,
                                 the count that wastes the fewest lane-steps over the level's
                                 columns (default 32) */
  int32_t level_warps_per_sm; /* warps per SM the sparse level launches aim for (0..64): a wide
                                 level of heavy columns takes 2, 4 or 8 warps per column while
                                 its columns of the batch number fewer than half of that many
                                 warps, and a narrow level's columns are split over CTAs up to
                                 that many warps (0: one warp per column on wide levels, splits
                                 up to two CTAs per SM; default 64) */
} glu_options;

void glu_options_default(glu_options* opt);
const char* glu_status_string(int status);
const char* glu_last_error(void);      /* thread-local detail for the last failing call */

/* ---- fast symbolic analysis (host, row f2) ----
 * Same output, bit for bit, as Symbolic_Matrix::fill_in + csr + leveling
 * (src/symbolic.cc:11-151) on the preprocessed CSC (ap[n+1], ai[nnz], rows in any order),
 * computed with a pruned depth-first reach instead of repeated set unions. */
int glu_symbolic_create(uint32_t n, const uint32_t* ap, const uint32_t* ai, glu_symbolic_t* out);
int glu_symbolic_sizes(glu_symbolic_t s, uint32_t* nnz, int32_t* num_lev);
int glu_symbolic_order(glu_symbolic_t s, uint32_t* n);
int glu_symbolic_get(glu_symbolic_t s, uint32_t* sym_c_ptr, uint32_t* sym_r_idx,
                     uint32_t* l_col_ptr, uint32_t* csr_r_ptr, uint32_t* csr_c_idx,
                     uint32_t* csr_diag_ptr, int32_t* level_ptr, int32_t* level_idx);
/* Position of every entry of A(ap, ai) in the filled pattern (what Symbolic_Matrix::predictLU
 * searches for with std::find, src/symbolic.cc:82-103).  pos[nnz_a]; duplicates map to -1
 * except the first, as predictLU keeps the first match. */
int glu_symbolic_positions(glu_symbolic_t s, const uint32_t* ap, const uint32_t* ai,
                           int64_t* pos);
void glu_symbolic_destroy(glu_symbolic_t s);
/* Serialisation of an analysis, so that a later run (or another process) skips it: the file
 * holds the filled CSC, the CSR mirror, the level sets and a 64-bit digest of the pattern
 * (ap, ai) the analysis was made from, plus a checksum of the whole.  The reference has no
 * counterpart (its analysis is recomputed by every run of lu_cmd).  glu_symbolic_load checks
 * the file (format, sizes, checksum, index ranges) and, when ap and ai are given, that they are
 * the pattern it was made from (same n, same entries in the same order): GLU_FILE_CANNOT_OPEN
 * if the file cannot be read or written, GLU_MATRIX_INVALID if it is damaged or belongs to
 * another pattern. */
int glu_symbolic_save(glu_symbolic_t s, const char* path);
int glu_symbolic_load(const char* path, uint32_t n, const uint32_t* ap, const uint32_t* ai,
                      glu_symbolic_t* out);

/* ---- plan: one sparsity pattern, resident on the device ----
 * Replaces the H2D copies and level bookkeeping of LUonDevice (src/numeric.cu:339-421).  The
 * arrays are Symbolic_Matrix's members (include/symbolic.h:9-24); they are copied, the caller
 * keeps ownership.  Builds the position maps, the sparse/dense split and the level schedule. */
int glu_plan_create(uint32_t n, uint32_t nnz, const uint32_t* sym_c_ptr,
                    const uint32_t* sym_r_idx, const uint32_t* l_col_ptr,
                    const uint32_t* csr_r_ptr, const uint32_t* csr_c_idx,
                    const uint32_t* csr_diag_ptr, int32_t num_lev, const int32_t* level_ptr,
                    const int32_t* level_idx, const glu_options* opt, glu_plan_t* out);

/* Value-ingest map (replaces predictLU + my_DumpA + _I_NicsLU_MC64Scale for new values,
 * src/symbolic.cc:82-103, src/preprocess/preprocess.c:8-100,
 * src/nicslu/source/nicslu_mc64scale.c:58-83): original entry e of the user's matrix goes to
 * filled-pattern position lu_pos[e] (or is dropped if -1) multiplied by scale[e].  scale may be
 * NULL (all ones). */
int glu_plan_set_ingest(glu_plan_t p, uint64_t nnz_a, const int64_t* lu_pos, const double* scale);

/* Builds the ingest map from the user's ORIGINAL CSC (ap[n+1], ai[nnz_a]) and NICSLU's analysis
 * arrays: entry (r, c) lands in filled column row_perm_inv[c], row col_perm_inv[r], scaled by
 * row_scale[c] * col_scale_perm[col_perm_inv[r]] (the product _I_NicsLU_MC64Scale forms,
 * src/nicslu/source/nicslu_mc64scale.c:38-46).  Scales may be NULL (mc64 scaling off). */
int glu_plan_ingest_from_nicslu(glu_plan_t p, uint32_t n, const uint32_t* ap, const uint32_t* ai,
                                const uint32_t* row_perm_inv, const uint32_t* col_perm_inv,
                                const double* row_scale, const double* col_scale_perm);

/* Row/column permutation and MC64 scaling of the solve (src/symbolic.cc:200-248 with
 * pivot = identity): b'[k] = rhs[col_perm[k]] * col_scale_perm[k];  x[j] = y[row_perm_inv[j]] *
 * row_scale[j].  Scales may be NULL (mc64 scaling off, cfgi[1] = 0). */
int glu_plan_set_solve_maps(glu_plan_t p, const uint32_t* col_perm, const uint32_t* row_perm_inv,
                            const double* col_scale_perm, const double* row_scale);

/* Plan statistics: i = 0 n, 1 nnz_lu, 2 tail start t, 3 dense order nt, 4 sparse levels,
 * 5 flops per refactor (sum_c |L(:,c)| + 2|L(:,c)||U(c,:)|), 6 bytes of device plan data,
 * 7 value slots per instance, 8 sparse update map entries, 9 dense panel width,
 * 10 padded dense order ntp, 11 flops of the padded dense LU, 12 L-solve levels,
 * 13 U-solve levels, 14 sparse value slots S, 15 hub columns, 16 sparse-to-dense updates,
 * 17 of them in the hub GEMM, 18 pull entries, 19 fronts, 20 updates done inside fronts,
 * 21 largest front buffer (doubles per instance), 22 sparse-phase levels (single columns and
 * fronts), 23 dense panels per trailing update, 24 DMMA GEMM variant, 25 extra chunks of pull
 * entries of heavy dense columns (applied by their own CTAs when the batch is a few matrices),
 * 26 widest front (columns). */
int glu_plan_stat(glu_plan_t p, int i, double* value);
int glu_plan_destroy(glu_plan_t p);

/* ---- batch: `count` value instances of one plan, factored in place on the device ---- */
int glu_batch_create(glu_plan_t p, int32_t count, glu_batch_t* out);
/* Same, but the caller provides the value storage (count * glu_batch_slots_per_instance doubles,
 * 256-byte aligned device memory) -- used to stay inside a memory budget. */
int glu_batch_slots_per_instance(glu_plan_t p, uint64_t* slots);
int glu_batch_create_external(glu_plan_t p, int32_t count, double* storage_dev, glu_batch_t* out);
int glu_batch_destroy(glu_batch_t b);

/* Loads values for instances [first, first+count): a_dev holds count rows of nnz_a doubles in
 * the user's original entry order (ingest map applied on the device).  The dense trailing block is
 * not cleared here: glu_refactor assembles it column by column from the loaded entries, so until
 * then glu_get_lu does not show it. */
int glu_load_values(glu_batch_t b, int32_t first, int32_t count, const double* a_dev, void* stream);
/* Loads already-preprocessed filled-pattern values (Symbolic_Matrix::val layout, nnz doubles per
 * instance, fill positions zero) -- the exact input LUonDevice takes. */
int glu_load_lu_values(glu_batch_t b, int32_t first, int32_t count, const double* val_dev,
                       void* stream);

/* Numeric refactorization of every instance (the work of LUonDevice, src/numeric.cu:423-596).
 * pert > 0 enables static-pivot perturbation: |pivot| < pert becomes pert for columns with a
 * non-empty L part (src/numeric.cu:139-140).  pert < 0 means "compute 3.45e-4 * ||A||_1 per
 * instance" as src/numeric.cu:405-421 does. */
int glu_refactor(glu_batch_t b, double pert, void* stream);

/* glu_refactor with CUDA events recorded around every launch; synchronizes the stream and
 * returns the device time (ms) and launch count of each phase (arrays of 7): 0 pivot-perturbation
 * setup, 1 sparse levels (single columns), 2 dense panels (diagonal block + L21/U12), 3 dense
 * trailing updates (DMMA), 4 sparse-to-dense contributions (pull + hub GEMM), 5 fronts,
 * 6 updates of a panel by the earlier panels of its group (thin DMMA products). */
int glu_refactor_timed(glu_batch_t b, double pert, void* stream, double* phase_ms,
                       int64_t* phase_launches);

/* Autotuner: the plan options that minimise the device time of one refactorization of
 * instances [0, count) of a_dev (original entry order, through the plan's ingest map), by
 * coordinate descent from *best (the starting options: pass glu_options_default's, or a
 * previous result) over the dense-block density threshold, DMMA GEMM variant, panel width,
 * panels per trailing update, hub threshold, warps per column, columns per warp, the wide-level
 * threshold, the sparse block size and the cooperative level launch, each candidate timed with
 * glu_refactor_timed (best of `repeats`).  The reference hard-codes its launch thresholds and
 * block sizes instead (src/numeric.cu:423-545).
 * Builds and frees a plan and a batch per candidate (device memory for `count` instances) and
 * synchronizes the stream; candidates that do not fit in device memory are skipped.  *best and
 * *best_ms (may be NULL) receive the result; the plan itself is unchanged -- create the tuned
 * plan with glu_plan_create(..., best, ...). */
int glu_autotune(glu_plan_t p, int32_t count, const double* a_dev, int32_t repeats,
                 glu_options* best, double* best_ms, void* stream);

/* Per-instance status flags (GLU_INST_*), copied to host (synchronizes the stream). */
int glu_batch_status(glu_batch_t b, int32_t* flags, void* stream);

/* Solves A_i X_i = B_i for every instance i with nrhs right-hand sides (Symbolic_Matrix::solve
 * semantics).  B_dev, X_dev: [count][nrhs][n] doubles (column-major per instance).
 * transpose != 0 solves A_i^T X_i = B_i (the adjoint).  X may alias B. */
int glu_solve(glu_batch_t b, int32_t nrhs, const double* B_dev, double* X_dev, int transpose,
              void* stream);

/* Pattern of the user's ORIGINAL matrix: entry e is A(rows[e], cols[e]) in the user's indexing,
 * in the order of the value arrays given to glu_load_values.  Needed by glu_residual,
 * glu_refine and glu_grad_a. */
int glu_plan_set_original_pattern(glu_plan_t p, uint64_t nnz_a, const uint32_t* rows,
                                  const uint32_t* cols);

/* Relative residual ||b - op(A) x||_inf / (||A||_inf ||x||_inf + ||b||_inf) of every
 * (instance, rhs) on the original matrix (a_dev: [count][nnz_a] values), written to
 * resid_dev[count * nrhs].  op(A) = A^T when transpose != 0.  Generalises the reference's
 * residual check (NicsLU_Residual, src/nicslu/source/nicslu_residual.c:9). */
int glu_residual(glu_batch_t b, int32_t nrhs, const double* a_dev, const double* B_dev,
                 const double* X_dev, int transpose, double* resid_dev, void* stream);

/* Allocation-free variant of glu_residual.  No counterpart in the reference.
 * For callers that may not allocate device memory between solves -- a simulator loop whose
 * device memory is all owned by its own pool, or a section where a cudaMalloc (which can
 * synchronize the device) is not allowed.  Its scratch is a fixed 2 MiB array in the library's
 * static device memory, held by every GPU that loads the library until the process exits.
 * Limit: count * nrhs <= GLU_NOALLOC_MAX_VECTORS (larger calls return GLU_BUDGET_EXCEEDED).
 * The first call on a device looks up the array's device address (set-up work): make it before
 * any stream capture.  The address is kept for the life of the process, so cudaDeviceReset
 * while the library is loaded is not supported.  All calls share the array: calls that overlap
 * on the GPU race. */
#define GLU_NOALLOC_MAX_VECTORS 65536
int glu_residual_noalloc(glu_batch_t b, int32_t nrhs, const double* a_dev, const double* B_dev,
                         const double* X_dev, int transpose, double* resid_dev, void* stream);

/* `steps` rounds of iterative refinement of X (r = B - op(A) X; solve op(A) D = r; X += D), the
 * GPU counterpart of NicsLU_Refine (src/nicslu/source/nicslu_refine.c:10-90), for systems that
 * static pivoting leaves marginally accurate.  resid_dev (may be NULL) receives the final
 * relative residuals.  A fixed step count keeps the call capturable in a CUDA graph. */
int glu_refine(glu_batch_t b, int32_t nrhs, const double* a_dev, const double* B_dev,
               double* X_dev, int32_t steps, int transpose, double* resid_dev, void* stream);

/* Gradient over A's nonzeros: gA[i][e] = -sum_k lambda[i][k][rows[e]] * x[i][k][cols[e]] on the
 * original pattern (glu_plan_set_original_pattern); lambda, x: [count][nrhs][n]. */
int glu_grad_a(glu_batch_t b, int32_t nrhs, const double* lambda_dev, const double* x_dev,
               double* ga_dev, void* stream);

/* Copies the factored values of instance i back in Symbolic_Matrix::val layout (L strictly
 * below l_col_ptr, U with diagonal), i.e. what LUonDevice leaves in A_sym.val. */
int glu_get_lu(glu_batch_t b, int32_t instance, double* val_dev, void* stream);

/* CUDA graph of load_values + refactor + solve (+ refine_steps rounds of refinement) for the
 * whole batch: capture once, replay with new contents of a_dev / B_dev. */
int glu_graph_capture(glu_batch_t b, const double* a_dev, int32_t nrhs, const double* B_dev,
                      double* X_dev, double pert, int32_t refine_steps, void* stream);
int glu_graph_launch(glu_batch_t b, void* stream);

/* Several batches of different patterns and uneven sizes in ONE CUDA graph: each batch's
 * load_values + refactor (+ solve + refine_steps rounds of refinement when nrhs[i] > 0) runs on
 * its own branch, so the whole group is one launch.  Arrays are indexed by batch; all batches
 * on one device.  Workspaces are allocated before the capture. */
int glu_group_capture(int32_t nbatch, const glu_batch_t* batches, const double* const* a_dev,
                      const int32_t* nrhs, const double* const* B_dev, double* const* X_dev,
                      double pert, int32_t refine_steps, void* stream, glu_group_t* out);
int glu_group_launch(glu_group_t g, void* stream);
int glu_group_launch_count(glu_group_t g, int64_t* launches);
int glu_group_destroy(glu_group_t g);

/* Test hook of the bounded device-side waits: glu_refactor with every barrier of the
 * cooperative level launches made unreachable (one arrival more than the CTAs that exist) and
 * the wait bound set to wait_ms.  Synchronizes the stream; returns GLU_TIMEOUT when a wait gave
 * up (the instances then carry GLU_INST_TIMEOUT and their factors are incomplete), GLU_OK if the
 * plan has no such launch.  No counterpart in the reference. */
int glu_debug_refactor_unreachable_barrier(glu_batch_t b, double wait_ms, void* stream);

/* Number of kernel launches the last glu_refactor / glu_solve enqueued (for accounting). */
int glu_batch_launch_count(glu_batch_t b, int64_t* launches);

/* Test hook: the dense trailing-update kernel (FP64 DMMA) on caller buffers, C -= A * B,
 * column-major, `count` problems with element strides sA, sB, sC.  M, K, lda, ldb, sA, sB even;
 * A and B 16-byte aligned.  No counterpart in the reference. */
int glu_debug_gemm_sub(int32_t M, int32_t N, int32_t K, const double* A, int32_t lda,
                       const double* B, int32_t ldb, double* C, int32_t ldc, int32_t count,
                       int64_t sA, int64_t sB, int64_t sC, int32_t variant, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GLU_B200_H */
