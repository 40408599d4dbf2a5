// C ABI of libglu_b200 (declared in include/glu_b200.h): plan / batch handles, device memory,
// launch sequencing and CUDA-graph capture.
//
// Launch structure of one refactorization (replaces the host loop of LUonDevice,
// src/numeric.cu:423-596, which launches 1..3*width kernels per level and synchronizes the
// device after every level): one kernel per sparse level, then two kernels per dense panel,
// all enqueued on the caller's stream with no host synchronization, so the whole sequence can
// be captured once in a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "glu_b200.h"
#include "internal.h"
#include "kernels.cuh"
#include "plan.h"
#include "plan_host.h"

namespace glu {

static thread_local char g_err[512] = "";

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

namespace {

// Makes the plan's device current for one entry point (and restores the caller's afterwards).
// It also clears the thread's last-error slot, so the launch checks of this call report its own
// failures, not an error some earlier runtime call of the caller left behind (errors that make
// the context unusable are reported again by every later call anyway).
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
    cudaGetLastError();
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

int cuda_status(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(GLU_CUDA_ERROR, "%s: %s", what, cudaGetErrorString(e));
  return GLU_OK;
}

}  // namespace
}  // namespace glu

struct glu_plan_s {
  int device = 0;
  glu::HostPlan hp;
  glu::PlanDev P{};
  std::vector<void*> allocs;
  size_t dev_bytes = 0;
  bool has_ingest = false, has_solve = false, has_grad = false;
  int32_t* d_lcols = nullptr;
  int32_t* d_ucols = nullptr;
  glu_options opt{};
  // host copies the autotuner needs to build the same plan with other options
  std::vector<int32_t> lev_ptr, lev_idx;
  std::vector<int64_t> ing_pos;
  std::vector<double> ing_scale;

  template <class T>
  int upload(const std::vector<T>& v, const T** out) {
    *out = nullptr;
    if (v.empty()) return GLU_OK;
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(T) * v.size()) != cudaSuccess) {
      cudaGetLastError();
      return glu::set_error(GLU_MEMORY_OVERFLOW, "cudaMalloc of %zu bytes failed",
                            sizeof(T) * v.size());
    }
    allocs.push_back(p);
    dev_bytes += sizeof(T) * v.size();
    if (cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return glu::cuda_status("plan upload");
    *out = static_cast<const T*>(p);
    return GLU_OK;
  }
  template <class T>
  void release(const T* p) {
    if (!p) return;
    auto it = std::find(allocs.begin(), allocs.end(), (void*)p);
    if (it != allocs.end()) {
      cudaFree(*it);
      allocs.erase(it);
    }
  }
};

struct glu_batch_s {
  glu_plan_s* plan = nullptr;
  int count = 0;
  double* vals = nullptr;
  bool own_vals = false;
  double* pert = nullptr;
  int32_t* status = nullptr;
  double* y = nullptr;
  double* gbuf = nullptr;       // hub panels G_L | G_U per instance (zero outside gathered slots)
  double* fbuf = nullptr;       // front buffers, front_area doubles per instance
  static constexpr int kFrontStreams = 4;
  cudaStream_t fstream[kFrontStreams] = {};   // concurrent fronts of one level
  cudaEvent_t ffork = nullptr, fjoin[kFrontStreams] = {};
  double* rbuf = nullptr;       // refinement residual / correction [count][nrhs][n]
  unsigned long long* norms = nullptr;  // [count * nrhs][4]
  int64_t r_vectors = 0;
  int64_t ylen = 0;
  int64_t y_vectors = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t own_stream = nullptr;
  int64_t launches = 0;
  bool loaded = false, factored = false;
  uint8_t* asm_flag = nullptr;  // [count] the last load left the instance's dense block for the
                                // pull to assemble (original-order ingest) instead of clearing it
  // runs of consecutive front-free sparse levels [l0, l1) of hp.slevels factored by one
  // cooperative launch each (k_sparse_persistent); their level descriptors in pdesc
  struct PRun {
    int l0, l1;
    int64_t desc_off;
    int grid;
    size_t smem;
  };
  std::vector<PRun> pruns;
  int4* pdesc = nullptr;
  unsigned* pbar = nullptr;     // pgroups barrier counters, then the failure word
  int pgroups = 0;
  int pextra = 0;               // test hook: arrivals added to every barrier target
  double pwait_ms = 1000.0;
};

namespace {

using glu::set_error;

int check_plan(glu_plan_t p) {
  if (!p) return set_error(GLU_ARGUMENT_ERROR, "null plan");
  return GLU_OK;
}

int ensure_workspace(glu_batch_t b, int64_t vectors, cudaStream_t s) {
  if (b->y_vectors >= vectors) return GLU_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &cs);
  if (cs != cudaStreamCaptureStatusNone)
    return set_error(GLU_NOT_READY, "solve workspace must be allocated before stream capture "
                     "(run one solve with the same nrhs first)");
  if (b->y) cudaFree(b->y);
  b->y = nullptr;
  b->y_vectors = 0;
  if (cudaMalloc(&b->y, sizeof(double) * b->ylen * vectors) != cudaSuccess) {
    cudaGetLastError();
    return set_error(GLU_MEMORY_OVERFLOW, "solve workspace allocation failed");
  }
  b->y_vectors = vectors;
  return GLU_OK;
}

// Optional per-phase timing: CUDA events recorded between launches on the launching stream.
struct PhaseTimer {
  std::vector<cudaEvent_t> ev;
  std::vector<int> phase;       // phase of the interval that ends at ev[i]
  cudaStream_t s = nullptr;
  void mark(int ph) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, s);
    ev.push_back(e);
    phase.push_back(ph);
  }
  ~PhaseTimer() {
    for (auto e : ev) cudaEventDestroy(e);
  }
};

int do_refactor(glu_batch_t b, double pert, cudaStream_t s, PhaseTimer* tm = nullptr,
                int64_t* phase_launches = nullptr) {
  glu_plan_s* pl = b->plan;
  const glu::PlanDev& P = pl->P;
  glu::LaunchCounter lc;
  auto mark = [&](int ph, int64_t before) {
    if (tm) tm->mark(ph);
    if (phase_launches) phase_launches[ph] += lc.n - before;
  };
  if (tm) tm->mark(-1);
  int64_t c0 = lc.n;
  cudaMemsetAsync(b->status, 0, sizeof(int32_t) * b->count, s);
  glu::launch_pert(P, b->vals, b->count, pert, b->pert, s, lc);
  mark(0, c0);
  const int gv = pl->hp.gemm_variant;
  const int nb = pl->hp.panel;
  size_t next_run = 0;
  for (size_t li = 0; li < pl->hp.slevels.size(); ++li) {
    if (next_run < b->pruns.size() && b->pruns[next_run].l0 == (int)li) {
      // a run of front-free levels: one cooperative launch with device-side level barriers
      const glu_batch_s::PRun& R = b->pruns[next_run++];
      c0 = lc.n;
      glu::launch_sparse_persistent(P, b->vals, b->count, b->pert, b->status,
                                    b->pdesc + R.desc_off, R.l1 - R.l0, b->pbar, b->pgroups,
                                    reinterpret_cast<int*>(b->pbar + b->pgroups), b->pwait_ms,
                                    b->pextra, R.grid, R.smem, s, lc);
      mark(1, c0);
      li = R.l1 - 1;
      continue;
    }
    const auto& L = pl->hp.slevels[li];
    const glu::FrontLevel& FL = pl->hp.flevels[li];
    if (L.f1 > L.f0 && pl->opt.front_batch &&
        glu::front_level_batched(FL, b->count, pl->hp.panel)) {
      // the level's single columns, then all of its fronts together, one launch per stage
      c0 = lc.n;
      if (L.ncols > 0)
        glu::launch_sparse_level(P, b->vals, b->count, b->pert, b->status, L.begin, L.ncols,
                                 L.wpc, L.max_nl, L.max_pairs, pl->hp.sparse_block,
                                 pl->hp.cols_per_warp, L.lanes, L.grow, pl->hp.level_warps, s,
                                 lc);
      mark(1, c0);
      c0 = lc.n;
      glu::launch_front_level(P, FL, b->vals, b->count, b->fbuf, pl->hp.front_area, b->pert,
                              b->status, s, lc);
      mark(5, c0);
      continue;
    }
    // a level's fronts on up to kFrontStreams streams, concurrently with each other and with the
    // level's single columns (all units of a level are independent); one stream when timing
    const int nf = L.f1 - L.f0;
    const int ns = (!tm && nf > 0 && b->ffork)
                       ? std::min(nf + (L.ncols > 0 ? 1 : 0), glu_batch_s::kFrontStreams)
                       : 1;
    if (ns > 1) {
      cudaEventRecord(b->ffork, s);
      for (int i = 0; i < ns; ++i) cudaStreamWaitEvent(b->fstream[i], b->ffork, 0);
    }
    c0 = lc.n;
    if (L.ncols > 0 && pl->hp.deterministic)
      glu::launch_sparse_level_det(P, b->vals, b->count, b->pert, b->status, L.begin, L.ncols,
                                   L.t0, L.t1, s, lc);
    else if (L.ncols > 0)
      glu::launch_sparse_level(P, b->vals, b->count, b->pert, b->status, L.begin, L.ncols, L.wpc,
                               L.max_nl, L.max_pairs, pl->hp.sparse_block, pl->hp.cols_per_warp,
                               L.lanes, L.grow, pl->hp.level_warps, s, lc);
    mark(1, c0);
    c0 = lc.n;
    for (int32_t fi = L.f0; fi < L.f1; ++fi) {
      const glu::Front& f = pl->hp.fronts[fi];
      const glu::FrontDev fd{f.w, f.wp, f.ld, f.qp, f.size, f.g_off, f.g_cnt, f.c_off, f.c_cnt,
                             f.h_off};
      cudaStream_t fs = ns > 1 ? b->fstream[(fi - L.f0) % ns] : s;
      glu::launch_front(P, fd, b->vals, b->count, b->fbuf + f.foff, pl->hp.front_area, b->pert,
                        b->status, nb, pl->hp.update_depth, gv, fs, lc);
    }
    if (ns > 1) {
      for (int i = 0; i < ns; ++i) {
        cudaEventRecord(b->fjoin[i], b->fstream[i]);
        cudaStreamWaitEvent(s, b->fjoin[i], 0);
      }
    }
    mark(5, c0);
  }
  c0 = lc.n;
  glu::launch_dense_pull(P, b->vals, b->count, b->asm_flag, pl->hp.deterministic, s, lc);
  glu::launch_hub_update(P, b->vals, b->count, b->gbuf, gv, s, lc);
  mark(4, c0);
  const glu::DenseView DV{b->vals + P.dbase, P.blob, (int32_t)P.ntp, (int32_t)P.ntp,
                          (int32_t)P.ntp, P.dhasl, (int32_t)P.nt};
  glu::launch_dense_factor(DV, b->count, b->pert, b->status, (int)P.ntp, nb,
                           pl->hp.update_depth, gv, s, lc, mark);
  b->launches = lc.n;
  b->factored = true;
  return glu::cuda_status("refactor launch");
}

int ensure_refine_workspace(glu_batch_t b, int64_t vectors, cudaStream_t s) {
  if (b->r_vectors >= vectors) return GLU_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &cs);
  if (cs != cudaStreamCaptureStatusNone)
    return set_error(GLU_NOT_READY, "refinement workspace must be allocated before stream "
                     "capture (run one residual/refine call with the same nrhs first)");
  if (b->rbuf) cudaFree(b->rbuf);
  if (b->norms) cudaFree(b->norms);
  b->rbuf = nullptr;
  b->norms = nullptr;
  b->r_vectors = 0;
  if (cudaMalloc(&b->rbuf, sizeof(double) * b->plan->hp.n * vectors) != cudaSuccess ||
      cudaMalloc(&b->norms, sizeof(unsigned long long) * 4 * vectors) != cudaSuccess) {
    cudaGetLastError();
    return set_error(GLU_MEMORY_OVERFLOW, "refinement workspace allocation failed");
  }
  b->r_vectors = vectors;
  return GLU_OK;
}

int do_solve(glu_batch_t b, int nrhs, const double* B, double* X, int transpose, cudaStream_t s);

// `steps` rounds of iterative refinement on the ORIGINAL matrix: r = b - op(A) x, solve
// op(A) d = r with the factors, x += d.  resid (may be null): final relative residuals.
int do_refine(glu_batch_t b, int nrhs, const double* a, const double* B, double* X, int steps,
              int transpose, double* resid, cudaStream_t s, int64_t* launches) {
  const glu::PlanDev& P = b->plan->P;
  int st = ensure_refine_workspace(b, (int64_t)b->count * nrhs, s);
  if (st) return st;
  glu::LaunchCounter lc;
  for (int it = 0; it < steps; ++it) {
    glu::launch_residual(P, b->count, nrhs, a, X, B, b->rbuf, b->norms, nullptr, transpose, s, lc);
    if ((st = do_solve(b, nrhs, b->rbuf, b->rbuf, transpose, s))) return st;
    lc.n += b->launches;
    glu::launch_axpy((int64_t)b->count * nrhs * P.n, b->rbuf, X, s, lc);
  }
  if (resid)
    glu::launch_residual(P, b->count, nrhs, a, X, B, nullptr, b->norms, resid, transpose, s, lc);
  if (launches) *launches = lc.n;
  return glu::cuda_status("refine");
}

int do_solve(glu_batch_t b, int nrhs, const double* B, double* X, int transpose, cudaStream_t s) {
  glu_plan_s* pl = b->plan;
  const glu::PlanDev& P = pl->P;
  const glu::HostPlan& hp = pl->hp;
  int st = ensure_workspace(b, (int64_t)b->count * nrhs, s);
  if (st) return st;
  glu::LaunchCounter lc;
  double* y = b->y;
  const int64_t yl = b->ylen;
  const int cnt = b->count;
  glu::launch_solve_permute_in(P, cnt, nrhs, B, y, yl, transpose, s, lc);
  const int nl = (int)hp.lptr.size() - 1, nu = (int)hp.uptr.size() - 1;
  // one solve level: its single columns, then its fronts (independent of each other)
  auto lvl = [&](bool L, int l, int which) {
    const std::vector<int32_t>& ptr = L ? hp.lptr : hp.uptr;
    const std::vector<int32_t>& fptr = L ? hp.lfr_ptr : hp.ufr_ptr;
    const int ncols = ptr[l + 1] - ptr[l];
    if (ncols > 0) {
      const int32_t* cols = L ? pl->d_lcols : pl->d_ucols;
      if (which == 0) glu::launch_sparse_lsolve(P, b->vals, cnt, nrhs, y, yl, cols, ptr[l], ncols, s, lc);
      if (which == 1) glu::launch_sparse_usolve(P, b->vals, cnt, nrhs, y, yl, cols, ptr[l], ncols, s, lc);
      if (which == 2) glu::launch_sparse_utsolve(P, b->vals, cnt, nrhs, y, yl, cols, ptr[l], ncols, s, lc);
      if (which == 3) glu::launch_sparse_ltsolve(P, b->vals, cnt, nrhs, y, yl, cols, ptr[l], ncols, s, lc);
    }
    const int nf = fptr[l + 1] - fptr[l];
    if (nf > 0) {
      const std::vector<int32_t>& fl = L ? hp.lfr : hp.ufr;
      int max_w = 0;
      for (int k = fptr[l]; k < fptr[l + 1]; ++k) max_w = std::max(max_w, hp.fw[fl[k]]);
      glu::launch_front_solve(P, b->vals, cnt, nrhs, y, yl, (L ? P.lfr : P.ufr) + fptr[l], nf,
                              max_w, which, s, lc);
    }
  };
  if (!transpose && hp.deterministic) {
    // row-wise (pull) solves: every entry of y is written by one warp, sums in a fixed order
    for (int l = 0; l < nl; ++l)
      glu::launch_rows_solve(P, b->vals, cnt, nrhs, y, yl, pl->d_lcols, hp.lptr[l],
                             hp.lptr[l + 1] - hp.lptr[l], 0, s, lc);
    if (P.nt > 0)    // rows of the dense block take their L21 part (columns < t)
      glu::launch_rows_solve(P, b->vals, cnt, nrhs, y, yl, nullptr, (int)P.t, (int)P.nt, 0, s, lc);
    glu::launch_dense_trsv(P, b->vals, cnt, nrhs, y, yl, 0, s, lc);
    glu::launch_dense_trsv(P, b->vals, cnt, nrhs, y, yl, 1, s, lc);
    for (int l = 0; l < nu; ++l)    // U rows, the border U(r < t, j >= t) included
      glu::launch_rows_solve(P, b->vals, cnt, nrhs, y, yl, pl->d_ucols, hp.uptr[l],
                             hp.uptr[l + 1] - hp.uptr[l], 1, s, lc);
  } else if (!transpose) {
    for (int l = 0; l < nl; ++l) lvl(true, l, 0);
    glu::launch_dense_trsv(P, b->vals, cnt, nrhs, y, yl, 0, s, lc);
    glu::launch_dense_trsv(P, b->vals, cnt, nrhs, y, yl, 1, s, lc);
    glu::launch_border(P, b->vals, cnt, nrhs, y, yl, 0, s, lc);
    for (int l = 0; l < nu; ++l) lvl(false, l, 1);
  } else {
    for (int l = nu - 1; l >= 0; --l) lvl(false, l, 2);
    glu::launch_border(P, b->vals, cnt, nrhs, y, yl, 1, s, lc);
    glu::launch_dense_trsv(P, b->vals, cnt, nrhs, y, yl, 2, s, lc);
    glu::launch_dense_trsv(P, b->vals, cnt, nrhs, y, yl, 3, s, lc);
    for (int l = nl - 1; l >= 0; --l) lvl(true, l, 3);
  }
  glu::launch_solve_permute_out(P, cnt, nrhs, y, X, yl, transpose, s, lc);
  b->launches = lc.n;
  return glu::cuda_status("solve launch");
}

}  // namespace

namespace glu {
// Read-only view of a batch for glu_residual_noalloc (noalloc.cu).
int batch_residual_view(glu_batch_t b, const PlanDev** P, int* count, int* device,
                        int* has_pattern) {
  if (!b) return set_error(GLU_ARGUMENT_ERROR, "null batch");
  *P = &b->plan->P;
  *count = b->count;
  *device = b->plan->device;
  *has_pattern = b->plan->has_grad ? 1 : 0;
  return GLU_OK;
}
}  // namespace glu

extern "C" {

void glu_options_default(glu_options* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->dense_threshold = 0.9;
  o->dense_min = 128;
  o->panel = 64;
  o->device = -1;
  o->hub_min_frac = 0.02;
  o->hub_max = 256;
  o->front_min_w = 16;
  o->front_min_flops = 1e6;
  o->gemm_variant = 12;
  o->update_depth = 8;
  o->sparse_persistent = 2;
  o->level_wait_ms = 1000.0;
  o->sparse_cols_per_warp = 1;
  o->wide_level_cols = 4 * 148;
  o->narrow_col_work = 256;
  o->sparse_block = 256;
  o->front_batch = 1;
  o->sparse_col_lanes = 32;
  o->level_warps_per_sm = 64;
}

const char* glu_status_string(int st) {
  switch (st) {
    case GLU_OK: return "ok";
    case GLU_ARGUMENT_ERROR: return "argument error";
    case GLU_MEMORY_OVERFLOW: return "memory overflow";
    case GLU_MATRIX_STRUCTURAL_SINGULAR: return "structurally singular matrix";
    case GLU_MATRIX_NUMERIC_SINGULAR: return "numerically singular matrix";
    case GLU_MATRIX_INVALID: return "invalid matrix";
    case GLU_MATRIX_ENTRY_DUPLICATED: return "duplicated matrix entry";
    case GLU_NUMERIC_OVERFLOW: return "numeric overflow";
    case GLU_CUDA_ERROR: return "CUDA error";
    case GLU_TIMEOUT: return "device wait timed out";
    case GLU_BUDGET_EXCEEDED: return "memory budget exceeded";
    case GLU_NOT_READY: return "call order violated";
    default: return "unknown status";
  }
}

const char* glu_last_error(void) { return glu::g_err; }

int glu_plan_create(uint32_t n, uint32_t nnz, const uint32_t* sym_c_ptr,
                    const uint32_t* sym_r_idx, const uint32_t* l_col_ptr,
                    const uint32_t* csr_r_ptr, const uint32_t* csr_c_idx,
                    const uint32_t* csr_diag_ptr, int32_t num_lev, const int32_t* level_ptr,
                    const int32_t* level_idx, const glu_options* opt, glu_plan_t* out) {
  if (!out || !sym_c_ptr || !sym_r_idx || !l_col_ptr || !csr_r_ptr || !csr_c_idx ||
      !csr_diag_ptr || !level_ptr || !level_idx)
    return set_error(GLU_ARGUMENT_ERROR, "null argument");
  *out = nullptr;
  glu_options o;
  if (opt) o = *opt; else glu_options_default(&o);
  if (o.dense_threshold <= 0.0) o.dense_threshold = 0.9;
  if (o.gemm_variant < 0 || o.gemm_variant >= glu::gemm_variants())
    return set_error(GLU_ARGUMENT_ERROR, "gemm_variant out of range");
  if (o.update_depth != 1 && o.update_depth != 2 && o.update_depth != 4 && o.update_depth != 8)
    return set_error(GLU_ARGUMENT_ERROR, "update_depth must be 1, 2, 4 or 8");
  if (o.sparse_persistent < 0) return set_error(GLU_ARGUMENT_ERROR, "sparse_persistent < 0");
  if (!(o.level_wait_ms > 0.0)) o.level_wait_ms = 1000.0;
  if (o.sparse_warps_per_col != 0 && o.sparse_warps_per_col != 1 && o.sparse_warps_per_col != 2 &&
      o.sparse_warps_per_col != 4 && o.sparse_warps_per_col != 8)
    return set_error(GLU_ARGUMENT_ERROR, "sparse_warps_per_col must be 0, 1, 2, 4 or 8");
  if (o.sparse_cols_per_warp == 0) o.sparse_cols_per_warp = 1;
  if (o.sparse_cols_per_warp != 1 && o.sparse_cols_per_warp != 2 && o.sparse_cols_per_warp != 4)
    return set_error(GLU_ARGUMENT_ERROR, "sparse_cols_per_warp must be 1, 2 or 4");
  if (o.sparse_block == 0) o.sparse_block = 256;
  if (o.sparse_block != 128 && o.sparse_block != 256)
    return set_error(GLU_ARGUMENT_ERROR, "sparse_block must be 128 or 256");
  if (o.sparse_col_lanes != 0 && o.sparse_col_lanes != 8 && o.sparse_col_lanes != 16 &&
      o.sparse_col_lanes != 32)
    return set_error(GLU_ARGUMENT_ERROR, "sparse_col_lanes must be 0, 8, 16 or 32");
  if (o.level_warps_per_sm < 0 || o.level_warps_per_sm > 64)
    return set_error(GLU_ARGUMENT_ERROR, "level_warps_per_sm must be in [0, 64]");
  glu_plan_s* p = new (std::nothrow) glu_plan_s();
  if (!p) return set_error(GLU_MEMORY_OVERFLOW, "host allocation failed");
  p->opt = o;
  int st;
  try {
    st = glu::build_host_plan(n, nnz, sym_c_ptr, sym_r_idx, l_col_ptr, csr_r_ptr, csr_c_idx,
                              csr_diag_ptr, num_lev, level_ptr, level_idx, o, p->hp);
  } catch (const std::bad_alloc&) {
    st = set_error(GLU_MEMORY_OVERFLOW, "host allocation failed while building the plan");
  }
  if (st != GLU_OK) {
    delete p;
    return st;
  }
  if (o.device >= 0) {
    p->device = o.device;
  } else if (cudaGetDevice(&p->device) != cudaSuccess) {
    cudaGetLastError();
    delete p;
    return set_error(GLU_CUDA_ERROR, "no CUDA device");
  }
  glu::DeviceGuard g(p->device);
  glu::HostPlan& hp = p->hp;
  glu::PlanDev& P = p->P;
  p->lev_ptr.assign(level_ptr, level_ptr + num_lev + 1);
  p->lev_idx.assign(level_idx, level_idx + n);
  P.n = hp.n;
  P.nnz = hp.nnz;
  P.t = hp.t;
  P.nt = hp.nt;
  P.ntp = hp.ntp;
  P.S = hp.S;
  P.dbase = hp.dbase;
  P.blob = hp.blob;
  P.hubs_p = hp.hubs_p;
  P.ngl = (int64_t)hp.gl_src.size();
  P.ngu = (int64_t)hp.gu_src.size();
  P.npull = hp.pull_ptr.empty() ? 0 : hp.pull_ptr.back();
  P.npullx = (int64_t)hp.pull_xcol.size();
  P.nbordck = (int64_t)hp.bord_ckcol.size();
  std::vector<uint8_t> dh = hp.dhasl;
  if ((st = p->upload(hp.cp, &P.cp)) || (st = p->upload(hp.ri, &P.ri)) ||
      (st = p->upload(hp.lp, &P.lp)) || (st = p->upload(hp.lsplit, &P.lsplit)) ||
      (st = p->upload(hp.pair_ptr, &P.pair_ptr)) || (st = p->upload(hp.pair_j, &P.pair_j)) ||
      (st = p->upload(hp.pair_uslot, &P.pair_uslot)) ||
      (st = p->upload(hp.pair_moff, &P.pair_moff)) || (st = p->upload(hp.tmap, &P.tmap)) ||
      (st = p->upload(hp.scols, &P.scols)) || (st = p->upload(dh, &P.dhasl)) ||
      (st = p->upload(hp.pos2slot, &P.pos2slot)) ||
      (st = p->upload(hp.bord_ptr, &P.bord_ptr)) || (st = p->upload(hp.bord_row, &P.bord_row)) ||
      (st = p->upload(hp.bord_slot, &P.bord_slot)) ||
      (st = p->upload(hp.bord_ckcol, &P.bord_ckcol)) || (st = p->upload(hp.bord_ck0, &P.bord_ck0)) || (st = p->upload(hp.gl_src, &P.gl_src)) ||
      (st = p->upload(hp.gl_dst, &P.gl_dst)) || (st = p->upload(hp.gu_src, &P.gu_src)) ||
      (st = p->upload(hp.gu_dst, &P.gu_dst)) || (st = p->upload(hp.pull_ptr, &P.pull_ptr)) ||
      (st = p->upload(hp.pull_lb, &P.pull_lb)) || (st = p->upload(hp.pull_le, &P.pull_le)) ||
      (st = p->upload(hp.pull_uslot, &P.pull_uslot)) ||
      (st = p->upload(hp.pull_mend, &P.pull_mend)) ||
      (st = p->upload(hp.pull_xcol, &P.pull_xcol)) || (st = p->upload(hp.pull_xe, &P.pull_xe)) ||
      (st = p->upload(hp.fg_slot, &P.fg_slot)) || (st = p->upload(hp.fg_idx, &P.fg_idx)) ||
      (st = p->upload(hp.fc_slot, &P.fc_slot)) || (st = p->upload(hp.fc_idx, &P.fc_idx)) ||
      (st = p->upload(hp.fhasl, &P.fhasl))) {
    glu_plan_destroy(p);
    return st;
  }
  if (hp.deterministic &&
      ((st = p->upload(hp.det_q, &P.det_q)) || (st = p->upload(hp.det_c, &P.det_c)) ||
       (st = p->upload(hp.det_tptr, &P.det_tptr)) || (st = p->upload(hp.rp, &P.rp)) ||
       (st = p->upload(hp.ci, &P.ci)) || (st = p->upload(hp.dp, &P.dp)) ||
       (st = p->upload(hp.csr_slot, &P.csr_slot)))) {
    glu_plan_destroy(p);
    return st;
  }
  const int32_t* lc = nullptr;
  const int32_t* uc = nullptr;
  if ((st = p->upload(hp.fgeom, &P.fgeom)) || (st = p->upload(hp.fg_aidx, &P.fg_aidx)) ||
      (st = p->upload(hp.fc_aidx, &P.fc_aidx))) {
    glu_plan_destroy(p);
    return st;
  }
  if ((st = p->upload(hp.lcols, &lc)) || (st = p->upload(hp.ucols, &uc)) ||
      (st = p->upload(hp.fs0, &P.fs0)) || (st = p->upload(hp.fw, &P.fw)) ||
      (st = p->upload(hp.lfr, &P.lfr)) || (st = p->upload(hp.ufr, &P.ufr))) {
    glu_plan_destroy(p);
    return st;
  }
  P.fw_max = 0;
  for (int32_t w : hp.fw) P.fw_max = std::max(P.fw_max, w);
  p->d_lcols = const_cast<int32_t*>(lc);
  p->d_ucols = const_cast<int32_t*>(uc);
  *out = p;
  return GLU_OK;
}

int glu_plan_set_ingest(glu_plan_t p, uint64_t nnz_a, const int64_t* lu_pos, const double* scale) {
  if (int st = check_plan(p)) return st;
  if (!lu_pos && nnz_a) return set_error(GLU_ARGUMENT_ERROR, "null lu_pos");
  std::vector<int64_t> slot(nnz_a);
  for (uint64_t e = 0; e < nnz_a; ++e) {
    const int64_t q = lu_pos[e];
    if (q >= (int64_t)p->hp.nnz) return set_error(GLU_ARGUMENT_ERROR, "lu_pos out of range");
    slot[e] = q < 0 ? -1 : p->hp.pos2slot[q];
  }
  glu::DeviceGuard g(p->device);
  p->release(p->P.ing_slot);
  p->release(p->P.ing_scale);
  p->P.ing_slot = nullptr;
  p->P.ing_scale = nullptr;
  int st = p->upload(slot, &p->P.ing_slot);
  if (st) return st;
  if (scale) {
    std::vector<double> sc(scale, scale + nnz_a);
    if ((st = p->upload(sc, &p->P.ing_scale))) return st;
  }
  // per dense column, the rows the ingest writes and the rows fronts add their Schur
  // complements to (duplicates removed); the latter are also cleared by every load
  p->release(p->P.asm_ptr);
  p->release(p->P.asm_row);
  p->release(p->P.asm_zero);
  p->P.asm_ptr = nullptr;
  p->P.asm_row = nullptr;
  p->P.asm_zero = nullptr;
  p->P.nasm_zero = 0;
  const int64_t ntp = p->P.ntp, dbase = p->P.dbase;
  if (ntp > 0) {
    std::vector<std::pair<int32_t, int32_t>> cr;     // (column, row)
    for (uint64_t e = 0; e < nnz_a; ++e) {
      if (slot[e] < dbase) continue;
      const int64_t d = slot[e] - dbase;
      cr.emplace_back((int32_t)(d / ntp), (int32_t)(d % ntp));
    }
    std::vector<int32_t> zero;
    for (int32_t s : p->hp.fc_slot) {
      if (s < dbase) continue;
      const int64_t d = s - dbase;
      cr.emplace_back((int32_t)(d / ntp), (int32_t)(d % ntp));
      zero.push_back(s);
    }
    std::sort(zero.begin(), zero.end());
    zero.erase(std::unique(zero.begin(), zero.end()), zero.end());
    if (!zero.empty()) {
      if ((st = p->upload(zero, &p->P.asm_zero))) return st;
      p->P.nasm_zero = (int64_t)zero.size();
    }
    std::sort(cr.begin(), cr.end());
    cr.erase(std::unique(cr.begin(), cr.end()), cr.end());
    std::vector<int32_t> ptr(ntp + 1, 0), row(cr.size());
    for (size_t i = 0; i < cr.size(); ++i) {
      ptr[cr[i].first + 1]++;
      row[i] = cr[i].second;
    }
    for (int64_t j = 0; j < ntp; ++j) ptr[j + 1] += ptr[j];
    if ((st = p->upload(ptr, &p->P.asm_ptr))) return st;
    if (!row.empty() && (st = p->upload(row, &p->P.asm_row))) return st;
  }
  p->ing_pos.assign(lu_pos, lu_pos + nnz_a);
  if (scale) p->ing_scale.assign(scale, scale + nnz_a);
  else p->ing_scale.clear();
  p->P.nnz_a = (int64_t)nnz_a;
  p->has_ingest = true;
  return GLU_OK;
}

int glu_plan_ingest_from_nicslu(glu_plan_t p, uint32_t n, const uint32_t* ap, const uint32_t* ai,
                                const uint32_t* row_perm_inv, const uint32_t* col_perm_inv,
                                const double* row_scale, const double* col_scale_perm) {
  if (int st = check_plan(p)) return st;
  if (!ap || !ai || !row_perm_inv || !col_perm_inv)
    return set_error(GLU_ARGUMENT_ERROR, "null argument");
  if (n != p->hp.n) return set_error(GLU_ARGUMENT_ERROR, "order mismatch");
  const uint64_t nnz_a = ap[n];
  std::vector<int64_t> pos(nnz_a);
  std::vector<double> scale;
  if (row_scale && col_scale_perm) scale.resize(nnz_a);
  const glu::HostPlan& hp = p->hp;
  std::vector<uint8_t> seen(hp.nnz, 0);
  for (uint32_t c = 0; c < n; ++c) {
    const uint32_t i = row_perm_inv[c];
    if (i >= n) return set_error(GLU_ARGUMENT_ERROR, "row_perm_inv out of range");
    for (uint32_t e = ap[c]; e < ap[c + 1]; ++e) {
      if (ai[e] >= n) return set_error(GLU_ARGUMENT_ERROR, "row index out of range");
      const uint32_t k = col_perm_inv[ai[e]];
      if (k >= n) return set_error(GLU_ARGUMENT_ERROR, "col_perm_inv out of range");
      const uint32_t* b = hp.ri.data() + hp.cp[i];
      const uint32_t* en = hp.ri.data() + hp.cp[i + 1];
      const uint32_t* f = std::lower_bound(b, en, k);
      if (f == en || *f != k)
        return set_error(GLU_MATRIX_INVALID, "entry (%u,%u) is not in the filled pattern", k, i);
      const int64_t q = f - hp.ri.data();
      if (seen[q]) return set_error(GLU_MATRIX_ENTRY_DUPLICATED, "duplicate entry (%u,%u)", ai[e], c);
      seen[q] = 1;
      pos[e] = q;
      // _I_NicsLU_MC64Scale: ax[j] *= row_scale[i] * col_scale_perm[ai[j]]
      if (!scale.empty()) scale[e] = row_scale[c] * col_scale_perm[k];
    }
  }
  return glu_plan_set_ingest(p, nnz_a, pos.data(), scale.empty() ? nullptr : scale.data());
}

int glu_plan_set_solve_maps(glu_plan_t p, const uint32_t* col_perm, const uint32_t* row_perm_inv,
                            const double* col_scale_perm, const double* row_scale) {
  if (int st = check_plan(p)) return st;
  if (!col_perm || !row_perm_inv) return set_error(GLU_ARGUMENT_ERROR, "null permutation");
  const uint32_t n = p->hp.n;
  std::vector<uint32_t> cpv(col_perm, col_perm + n), rpi(row_perm_inv, row_perm_inv + n);
  std::vector<uint32_t> rperm(n, UINT32_MAX);
  std::vector<uint8_t> chk(n, 0);
  for (uint32_t j = 0; j < n; ++j) {
    if (rpi[j] >= n || rperm[rpi[j]] != UINT32_MAX)
      return set_error(GLU_ARGUMENT_ERROR, "row_perm_inv is not a permutation");
    rperm[rpi[j]] = j;
    if (cpv[j] >= n || chk[cpv[j]]) return set_error(GLU_ARGUMENT_ERROR, "col_perm is not a permutation");
    chk[cpv[j]] = 1;
  }
  glu::DeviceGuard g(p->device);
  glu::PlanDev& P = p->P;
  p->release(P.col_perm);
  p->release(P.row_perm_inv);
  p->release(P.row_perm);
  p->release(P.col_scale_perm);
  p->release(P.row_scale);
  P.col_perm = P.row_perm_inv = P.row_perm = nullptr;
  P.col_scale_perm = P.row_scale = nullptr;
  int st;
  if ((st = p->upload(cpv, &P.col_perm)) || (st = p->upload(rpi, &P.row_perm_inv)) ||
      (st = p->upload(rperm, &P.row_perm)))
    return st;
  if (col_scale_perm && row_scale) {
    std::vector<double> a(col_scale_perm, col_scale_perm + n), b(row_scale, row_scale + n);
    if ((st = p->upload(a, &P.col_scale_perm)) || (st = p->upload(b, &P.row_scale))) return st;
  }
  p->has_solve = true;
  return GLU_OK;
}

int glu_plan_set_original_pattern(glu_plan_t p, uint64_t nnz_a, const uint32_t* rows,
                                  const uint32_t* cols) {
  if (int st = check_plan(p)) return st;
  if (nnz_a && (!rows || !cols)) return set_error(GLU_ARGUMENT_ERROR, "null pattern");
  const uint32_t n = p->hp.n;
  for (uint64_t e = 0; e < nnz_a; ++e)
    if (rows[e] >= n || cols[e] >= n)
      return set_error(GLU_ARGUMENT_ERROR, "pattern index out of range");
  // row-major and column-major orders of the entries (residual of A x and of A^T x)
  std::vector<int64_t> rptr(n + 1, 0), cptr(n + 1, 0), re(nnz_a), ce(nnz_a);
  for (uint64_t e = 0; e < nnz_a; ++e) {
    rptr[rows[e] + 1]++;
    cptr[cols[e] + 1]++;
  }
  for (uint32_t i = 0; i < n; ++i) {
    rptr[i + 1] += rptr[i];
    cptr[i + 1] += cptr[i];
  }
  {
    std::vector<int64_t> fr(rptr.begin(), rptr.end() - 1), fc(cptr.begin(), cptr.end() - 1);
    for (uint64_t e = 0; e < nnz_a; ++e) {
      re[fr[rows[e]]++] = (int64_t)e;
      ce[fc[cols[e]]++] = (int64_t)e;
    }
  }
  glu::DeviceGuard g(p->device);
  glu::PlanDev& P = p->P;
  p->release(P.g_row);
  p->release(P.g_col);
  p->release(P.o_row_ptr);
  p->release(P.o_row_e);
  p->release(P.o_col_ptr);
  p->release(P.o_col_e);
  P.g_row = P.g_col = nullptr;
  P.o_row_ptr = P.o_row_e = P.o_col_ptr = P.o_col_e = nullptr;
  std::vector<uint32_t> r(rows, rows + nnz_a), c(cols, cols + nnz_a);
  int st;
  if ((st = p->upload(r, &P.g_row)) || (st = p->upload(c, &P.g_col)) ||
      (st = p->upload(rptr, &P.o_row_ptr)) || (st = p->upload(re, &P.o_row_e)) ||
      (st = p->upload(cptr, &P.o_col_ptr)) || (st = p->upload(ce, &P.o_col_e)))
    return st;
  P.nnz_g = (int64_t)nnz_a;
  p->has_grad = true;
  return GLU_OK;
}

int glu_plan_stat(glu_plan_t p, int i, double* v) {
  if (int st = check_plan(p)) return st;
  if (!v) return set_error(GLU_ARGUMENT_ERROR, "null output");
  const glu::HostPlan& hp = p->hp;
  switch (i) {
    case 0: *v = hp.n; break;
    case 1: *v = hp.nnz; break;
    case 2: *v = hp.t; break;
    case 3: *v = hp.nt; break;
    case 4: *v = (double)hp.slevels.size(); break;
    case 5: *v = hp.flops; break;
    case 6: *v = (double)p->dev_bytes; break;
    case 7: *v = (double)hp.blob; break;
    case 8: *v = (double)hp.tmap.size(); break;
    case 9: *v = hp.panel; break;
    case 10: *v = hp.ntp; break;
    case 11: *v = hp.flops_dense; break;
    case 12: *v = (double)(hp.lptr.size() - 1); break;
    case 13: *v = (double)(hp.uptr.size() - 1); break;
    case 14: *v = (double)hp.S; break;
    case 15: *v = (double)hp.hubs.size(); break;
    case 16: *v = hp.dense_updates; break;
    case 17: *v = hp.hub_updates; break;
    case 18: *v = (double)(hp.pull_ptr.empty() ? 0 : hp.pull_ptr.back()); break;
    case 19: *v = (double)hp.fronts.size(); break;
    case 20: *v = hp.front_updates; break;
    case 21: *v = (double)hp.front_max; break;
    case 22: *v = (double)hp.slevels.size(); break;
    case 23: *v = (double)hp.update_depth; break;
    case 24: *v = (double)hp.gemm_variant; break;
    case 25: *v = (double)hp.pull_xcol.size(); break;
    case 26: *v = (double)p->P.fw_max; break;
    default: return set_error(GLU_ARGUMENT_ERROR, "unknown statistic %d", i);
  }
  return GLU_OK;
}

int glu_plan_destroy(glu_plan_t p) {
  if (!p) return GLU_OK;
  {
    glu::DeviceGuard g(p->device);
    for (void* a : p->allocs) cudaFree(a);
  }
  delete p;
  return GLU_OK;
}

int glu_batch_slots_per_instance(glu_plan_t p, uint64_t* slots) {
  if (int st = check_plan(p)) return st;
  if (!slots) return set_error(GLU_ARGUMENT_ERROR, "null output");
  *slots = (uint64_t)p->hp.blob;
  return GLU_OK;
}

// Runs of at least opt.sparse_persistent consecutive narrow sparse levels without fronts, and the
// per-level work descriptors of their cooperative launches: {begin, ncols, mode, splits} with
// mode 0 (warp per column) or 1 (CTA per column) as the plan chose, or 3 when a level's columns
// are fewer than the CTAs an instance gets and carry many pairs (each column's pairs are then
// split over several CTAs, as launch_sparse_level does for one launch per level).
static int build_persistent(glu_batch_s* b) {
  const glu::HostPlan& hp = b->plan->hp;
  const glu_options& o = b->plan->opt;
  b->pwait_ms = o.level_wait_ms;
  if (o.sparse_persistent <= 0 || hp.deterministic) return GLU_OK;
  const int nl = (int)hp.slevels.size();
  const int grid0 = glu::persistent_grid(0);
  if (grid0 <= 0) return GLU_OK;                 // the kernel cannot run here: per-level launches
  // narrow levels only: at most two columns of the whole batch per SM.  A wider level's own
  // launch costs little next to its work, and it keeps the per-level kernel's occupancy (the
  // cooperative kernel holds four CTAs per SM, the per-level one six) and dynamic block
  // scheduling: on the mesh, cooperative runs over levels of up to 19,000 columns were slower
  // than one launch per level (sparse phase 28.0 vs 22.8 ms)
  const int64_t narrow = 2 * (int64_t)glu::sm_count();
  auto plain = [&](int k) {
    return hp.slevels[k].f1 == hp.slevels[k].f0 && hp.slevels[k].ncols > 0 &&
           (int64_t)hp.slevels[k].ncols * b->count <= narrow;
  };
  std::vector<std::pair<int, int>> runs;
  for (int l = 0; l < nl;) {
    if (!plain(l)) {
      ++l;
      continue;
    }
    int e = l;
    while (e < nl && plain(e)) ++e;
    if (e - l >= std::max(1, o.sparse_persistent)) runs.emplace_back(l, e);
    l = e;
  }
  if (runs.empty()) return GLU_OK;
  constexpr int kSplitMaxL = 6144;               // L(:,c) staged in 48 KB of shared memory
  std::vector<int4> desc;
  int max_groups = 1;
  for (auto [l0, l1] : runs) {
    auto describe = [&](int grid, size_t* smem) {
      const int G = std::min(b->count, grid);
      const int cpg = grid / G;
      std::vector<int4> d;
      *smem = 0;
      for (int l = l0; l < l1; ++l) {
        const glu::LevelLaunch& L = hp.slevels[l];
        int mode = L.mode, splits = 1;
        if (L.mode == 1 && L.ncols < cpg && L.max_pairs > 16 && L.max_nl <= kSplitMaxL) {
          splits = std::min((cpg + L.ncols - 1) / L.ncols, (L.max_pairs + 7) / 8);
          if (splits > 1) {
            mode = 3;
            *smem = std::max(*smem, sizeof(double) * (size_t)std::max(L.max_nl, 1));
          }
        }
        d.push_back(make_int4(L.begin, L.ncols, mode, splits));
      }
      return d;
    };
    // no more CTAs than the run's widest level can use (a warp per column, or a CTA per column
    // with its pairs split up to 16 ways), so a tail of one-column levels meets at barriers of
    // a few CTAs instead of the whole GPU
    int64_t need = 1;
    for (int l = l0; l < l1; ++l) {
      const glu::LevelLaunch& L = hp.slevels[l];
      need = std::max<int64_t>(need, L.mode == 0 ? (L.ncols + 7) / 8
                                                 : (int64_t)L.ncols *
                                                       std::min(16, (L.max_pairs + 7) / 8 + 1));
    }
    const int g0 = (int)std::min<int64_t>(grid0, std::max<int64_t>(1, need) * b->count);
    size_t smem = 0;
    std::vector<int4> d = describe(g0, &smem);
    int grid = g0;
    if (smem > 0) {
      grid = std::min(g0, glu::persistent_grid(smem));
      if (grid <= 0) continue;                   // leave this run to per-level launches
      size_t smem2 = 0;
      d = describe(grid, &smem2);
      smem = std::max(smem, smem2);
    }
    glu_batch_s::PRun R{l0, l1, (int64_t)desc.size(), grid, smem};
    desc.insert(desc.end(), d.begin(), d.end());
    b->pruns.push_back(R);
    max_groups = std::max(max_groups, std::min(b->count, grid));
  }
  if (b->pruns.empty()) return GLU_OK;
  b->pgroups = max_groups;
  if (cudaMalloc(&b->pdesc, sizeof(int4) * desc.size()) != cudaSuccess ||
      cudaMalloc(&b->pbar, sizeof(unsigned) * (max_groups + 1)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(GLU_MEMORY_OVERFLOW, "cudaMalloc of the level-run descriptors failed");
  }
  if (cudaMemcpy(b->pdesc, desc.data(), sizeof(int4) * desc.size(), cudaMemcpyHostToDevice) !=
      cudaSuccess)
    return glu::cuda_status("level-run descriptors");
  return GLU_OK;
}

static int batch_create(glu_plan_t p, int32_t count, double* storage, glu_batch_t* out) {
  if (int st = check_plan(p)) return st;
  if (!out || count <= 0 || count > 65535)
    return set_error(GLU_ARGUMENT_ERROR, "count must be in [1, 65535]");
  *out = nullptr;
  glu::DeviceGuard g(p->device);
  glu_batch_s* b = new (std::nothrow) glu_batch_s();
  if (!b) return set_error(GLU_MEMORY_OVERFLOW, "host allocation failed");
  b->plan = p;
  b->count = count;
  b->ylen = (int64_t)p->hp.n + (int64_t)(p->hp.ntp - p->hp.nt);
  const size_t bytes = sizeof(double) * (size_t)p->hp.blob * count;
  if (storage) {
    if (reinterpret_cast<uintptr_t>(storage) % 256)
      return delete b, set_error(GLU_ARGUMENT_ERROR, "storage must be 256-byte aligned");
    b->vals = storage;
  } else {
    if (cudaMalloc(&b->vals, bytes) != cudaSuccess) {
      cudaGetLastError();
      delete b;
      return set_error(GLU_MEMORY_OVERFLOW, "cudaMalloc of %zu bytes for %d instances failed",
                       bytes, count);
    }
    b->own_vals = true;
  }
  if (p->hp.front_area > 0) {
    const size_t fbytes = sizeof(double) * (size_t)p->hp.front_area * count;
    if (cudaMalloc(&b->fbuf, fbytes) != cudaSuccess) {
      cudaGetLastError();
      glu_batch_destroy(b);
      return set_error(GLU_MEMORY_OVERFLOW, "cudaMalloc of %zu bytes (front buffers) failed", fbytes);
    }
  }
  if (p->P.hubs_p > 0) {
    const size_t gbytes = sizeof(double) * 2 * (size_t)p->P.ntp * p->P.hubs_p * count;
    if (cudaMalloc(&b->gbuf, gbytes) != cudaSuccess) {
      cudaGetLastError();
      glu_batch_destroy(b);
      return set_error(GLU_MEMORY_OVERFLOW, "cudaMalloc of %zu bytes (hub panels) failed", gbytes);
    }
    cudaMemset(b->gbuf, 0, gbytes);
  }
  if (cudaMalloc(&b->pert, sizeof(double) * count) != cudaSuccess ||
      cudaMalloc(&b->status, sizeof(int32_t) * count) != cudaSuccess ||
      cudaMalloc(&b->asm_flag, count) != cudaSuccess) {
    cudaGetLastError();
    glu_batch_destroy(b);
    return set_error(GLU_MEMORY_OVERFLOW, "cudaMalloc failed");
  }
  cudaMemset(b->status, 0, sizeof(int32_t) * count);
  cudaMemset(b->asm_flag, 0, count);
  if (int st = build_persistent(b)) {
    glu_batch_destroy(b);
    return st;
  }
  if (!p->hp.fronts.empty()) {
    bool ok = cudaEventCreateWithFlags(&b->ffork, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; ok && i < glu_batch_s::kFrontStreams; ++i)
      ok = cudaStreamCreateWithFlags(&b->fstream[i], cudaStreamNonBlocking) == cudaSuccess &&
           cudaEventCreateWithFlags(&b->fjoin[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      glu_batch_destroy(b);
      return set_error(GLU_MEMORY_OVERFLOW, "front streams / events");
    }
  }
  *out = b;
  return glu::cuda_status("batch create");
}

int glu_batch_create(glu_plan_t p, int32_t count, glu_batch_t* out) {
  return batch_create(p, count, nullptr, out);
}

int glu_batch_create_external(glu_plan_t p, int32_t count, double* storage_dev, glu_batch_t* out) {
  if (!storage_dev) return set_error(GLU_ARGUMENT_ERROR, "null storage");
  return batch_create(p, count, storage_dev, out);
}

int glu_batch_destroy(glu_batch_t b) {
  if (!b) return GLU_OK;
  glu::DeviceGuard g(b->plan->device);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->own_stream) cudaStreamDestroy(b->own_stream);
  for (int i = 0; i < glu_batch_s::kFrontStreams; ++i) {
    if (b->fstream[i]) cudaStreamDestroy(b->fstream[i]);
    if (b->fjoin[i]) cudaEventDestroy(b->fjoin[i]);
  }
  if (b->ffork) cudaEventDestroy(b->ffork);
  if (b->own_vals && b->vals) cudaFree(b->vals);
  if (b->pert) cudaFree(b->pert);
  if (b->status) cudaFree(b->status);
  if (b->asm_flag) cudaFree(b->asm_flag);
  if (b->y) cudaFree(b->y);
  if (b->gbuf) cudaFree(b->gbuf);
  if (b->fbuf) cudaFree(b->fbuf);
  if (b->rbuf) cudaFree(b->rbuf);
  if (b->norms) cudaFree(b->norms);
  if (b->pdesc) cudaFree(b->pdesc);
  if (b->pbar) cudaFree(b->pbar);
  delete b;
  return GLU_OK;
}

int glu_load_values(glu_batch_t b, int32_t first, int32_t count, const double* a_dev,
                    void* stream) {
  if (!b) return set_error(GLU_ARGUMENT_ERROR, "null batch");
  if (!b->plan->has_ingest) return set_error(GLU_NOT_READY, "no ingest map (glu_plan_set_ingest)");
  if (first < 0 || count <= 0 || first + count > b->count || !a_dev)
    return set_error(GLU_ARGUMENT_ERROR, "instance range");
  glu::DeviceGuard g(b->plan->device);
  cudaStream_t s = (cudaStream_t)stream;
  glu::LaunchCounter lc;
  const bool asm_ok = glu::dense_assembly(b->plan->P);
  glu::launch_prepare_blob(b->plan->P, b->vals, first, count, asm_ok, s, lc);
  glu::launch_ingest(b->plan->P, b->vals, first, count, a_dev, s, lc);
  cudaMemsetAsync(b->asm_flag + first, asm_ok ? 1 : 0, count, s);
  b->loaded = true;
  b->factored = false;
  return glu::cuda_status("load values");
}

int glu_load_lu_values(glu_batch_t b, int32_t first, int32_t count, const double* val_dev,
                       void* stream) {
  if (!b) return set_error(GLU_ARGUMENT_ERROR, "null batch");
  if (first < 0 || count <= 0 || first + count > b->count || !val_dev)
    return set_error(GLU_ARGUMENT_ERROR, "instance range");
  glu::DeviceGuard g(b->plan->device);
  cudaStream_t s = (cudaStream_t)stream;
  glu::LaunchCounter lc;
  glu::launch_prepare_blob(b->plan->P, b->vals, first, count, false, s, lc);
  glu::launch_load_lu(b->plan->P, b->vals, first, count, val_dev, s, lc);
  cudaMemsetAsync(b->asm_flag + first, 0, count, s);
  b->loaded = true;
  b->factored = false;
  return glu::cuda_status("load LU values");
}

int glu_refactor(glu_batch_t b, double pert, void* stream) {
  if (!b) return set_error(GLU_ARGUMENT_ERROR, "null batch");
  if (!b->loaded) return set_error(GLU_NOT_READY, "no values loaded");
  glu::DeviceGuard g(b->plan->device);
  return do_refactor(b, pert, (cudaStream_t)stream);
}

int glu_refactor_timed(glu_batch_t b, double pert, void* stream, double* phase_ms,
                       int64_t* phase_launches) {
  if (!b || !phase_ms || !phase_launches) return set_error(GLU_ARGUMENT_ERROR, "null argument");
  if (!b->loaded) return set_error(GLU_NOT_READY, "no values loaded");
  glu::DeviceGuard g(b->plan->device);
  cudaStream_t s = (cudaStream_t)stream;
  for (int i = 0; i < 7; ++i) {
    phase_ms[i] = 0.0;
    phase_launches[i] = 0;
  }
  PhaseTimer tm;
  tm.s = s;
  int st = do_refactor(b, pert, s, &tm, phase_launches);
  if (st) return st;
  if (cudaStreamSynchronize(s) != cudaSuccess) return glu::cuda_status("refactor");
  for (size_t i = 1; i < tm.ev.size(); ++i) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, tm.ev[i - 1], tm.ev[i]);
    if (tm.phase[i] >= 0 && tm.phase[i] < 7) phase_ms[tm.phase[i]] += ms;
  }
  return glu::cuda_status("refactor timed");
}

int glu_debug_refactor_unreachable_barrier(glu_batch_t b, double wait_ms, void* stream) {
  if (!b || !(wait_ms > 0.0)) return set_error(GLU_ARGUMENT_ERROR, "bad argument");
  if (!b->loaded) return set_error(GLU_NOT_READY, "no values loaded");
  glu::DeviceGuard g(b->plan->device);
  cudaStream_t s = (cudaStream_t)stream;
  const double saved = b->pwait_ms;
  b->pextra = 1;
  b->pwait_ms = wait_ms;
  int st = do_refactor(b, 0.0, s);
  b->pextra = 0;
  b->pwait_ms = saved;
  if (st) return st;
  if (cudaStreamSynchronize(s) != cudaSuccess) return glu::cuda_status("refactor");
  if (b->pruns.empty()) return GLU_OK;
  std::vector<int32_t> flags(b->count);
  if (cudaMemcpy(flags.data(), b->status, sizeof(int32_t) * b->count, cudaMemcpyDeviceToHost) !=
      cudaSuccess)
    return glu::cuda_status("status");
  for (int32_t f : flags)
    if (f & GLU_INST_TIMEOUT)
      return set_error(GLU_TIMEOUT, "a device-side level barrier gave up after %.3f ms", wait_ms);
  return GLU_OK;
}

int glu_autotune(glu_plan_t p, int32_t count, const double* a_dev, int32_t repeats,
                 glu_options* best, double* best_ms, void* stream) {
  if (int st = check_plan(p)) return st;
  if (!best || count <= 0 || !a_dev) return set_error(GLU_ARGUMENT_ERROR, "bad argument");
  if (!p->has_ingest) return set_error(GLU_NOT_READY, "no ingest map (glu_plan_set_ingest)");
  if (repeats < 1) repeats = 1;
  glu::DeviceGuard g(p->device);
  cudaStream_t s = (cudaStream_t)stream;
  const glu::HostPlan& hp = p->hp;
  // device time of one refactorization of the sample with options o (best of `repeats`)
  auto time_options = [&](const glu_options& o, double* ms_out) -> int {
    glu_plan_t c = nullptr;
    glu_batch_t b = nullptr;
    int st = glu_plan_create(hp.n, hp.nnz, hp.cp.data(), hp.ri.data(), hp.lp.data(),
                             hp.rp.data(), hp.ci.data(), hp.dp.data(),
                             (int32_t)p->lev_ptr.size() - 1, p->lev_ptr.data(),
                             p->lev_idx.data(), &o, &c);
    if (!st)
      st = glu_plan_set_ingest(c, p->ing_pos.size(), p->ing_pos.data(),
                               p->ing_scale.empty() ? nullptr : p->ing_scale.data());
    if (!st) st = glu_batch_create(c, count, &b);
    double bestt = 1e300;
    for (int r = 0; !st && r < repeats; ++r) {
      double ms[7];
      int64_t nl[7];
      st = glu_load_values(b, 0, count, a_dev, s);
      if (!st) st = glu_refactor_timed(b, 0.0, s, ms, nl);
      double t = 0.0;
      for (double x : ms) t += x;
      if (!st) bestt = std::min(bestt, t);
    }
    glu_batch_destroy(b);
    glu_plan_destroy(c);
    *ms_out = bestt;
    return st;
  };
  glu_options cur = *best;
  double cur_ms = 0.0;
  if (int st = time_options(cur, &cur_ms)) return st;
  // coordinate descent over the knobs, as the Python autotuner does
  const int32_t variants[] = {12, 11, 13, 0, 6, 5};
  const int32_t panels[] = {64, 128};
  const int32_t depths[] = {8, 4, 2, 1};
  const double hubs[] = {0.02, 0.005, 0.08};
  const int32_t wpcs[] = {0, 1, 2, 4, 8};
  const int32_t cpws[] = {1, 2, 4};
  const int32_t wides[] = {4 * 148, 148, 16 * 148};
  const int32_t blocks[] = {256, 128};
  const int32_t persist[] = {2, 0};
  const int32_t lanes[] = {32, 0, 16, 8};
  const int32_t occs[] = {64, 0, 24, 48};
  const double dths[] = {0.9, 0.8, 0.95, 0.99};
  auto try_knob = [&](auto setter, auto& values) -> int {
    for (auto v : values) {
      glu_options o = cur;
      setter(o, v);
      if (memcmp(&o, &cur, sizeof(o)) == 0) continue;
      double ms = 0.0;
      const int st = time_options(o, &ms);
      if (st == GLU_MEMORY_OVERFLOW) continue;      // this candidate does not fit: skip it
      if (st) return st;
      if (ms < cur_ms) cur = o, cur_ms = ms;
    }
    return GLU_OK;
  };
  // the dense/sparse split first: it changes which columns the other knobs act on
  int st = try_knob([](glu_options& o, double v) { o.dense_threshold = v; }, dths);
  if (!st) st = try_knob([](glu_options& o, int32_t v) { o.gemm_variant = v; }, variants);
  if (!st) st = try_knob([](glu_options& o, int32_t v) { o.panel = v; }, panels);
  if (!st) st = try_knob([](glu_options& o, int32_t v) { o.update_depth = v; }, depths);
  if (!st) st = try_knob([](glu_options& o, double v) { o.hub_min_frac = v; }, hubs);
  if (!st) st = try_knob([](glu_options& o, int32_t v) { o.sparse_warps_per_col = v; }, wpcs);
  if (!st) st = try_knob([](glu_options& o, int32_t v) { o.sparse_cols_per_warp = v; }, cpws);
  if (!st) st = try_knob([](glu_options& o, int32_t v) { o.wide_level_cols = v; }, wides);
  if (!st) st = try_knob([](glu_options& o, int32_t v) { o.sparse_block = v; }, blocks);
  if (!st) st = try_knob([](glu_options& o, int32_t v) { o.sparse_persistent = v; }, persist);
  if (!st) st = try_knob([](glu_options& o, int32_t v) { o.sparse_col_lanes = v; }, lanes);
  if (!st) st = try_knob([](glu_options& o, int32_t v) { o.level_warps_per_sm = v; }, occs);
  if (st) return st;
  *best = cur;
  if (best_ms) *best_ms = cur_ms;
  return GLU_OK;
}

int glu_batch_status(glu_batch_t b, int32_t* flags, void* stream) {
  if (!b || !flags) return set_error(GLU_ARGUMENT_ERROR, "null argument");
  glu::DeviceGuard g(b->plan->device);
  cudaStream_t s = (cudaStream_t)stream;
  cudaMemcpyAsync(flags, b->status, sizeof(int32_t) * b->count, cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  return glu::cuda_status("status");
}

int glu_solve(glu_batch_t b, int32_t nrhs, const double* B_dev, double* X_dev, int transpose,
              void* stream) {
  if (!b || !B_dev || !X_dev || nrhs <= 0) return set_error(GLU_ARGUMENT_ERROR, "bad argument");
  if ((int64_t)nrhs * b->count > 65535)
    return set_error(GLU_ARGUMENT_ERROR, "count * nrhs must be <= 65535");
  if (!b->plan->has_solve) return set_error(GLU_NOT_READY, "no solve maps (glu_plan_set_solve_maps)");
  if (!b->factored) return set_error(GLU_NOT_READY, "solve before refactor");
  glu::DeviceGuard g(b->plan->device);
  return do_solve(b, nrhs, B_dev, X_dev, transpose, (cudaStream_t)stream);
}

int glu_residual(glu_batch_t b, int32_t nrhs, const double* a_dev, const double* B_dev,
                 const double* X_dev, int transpose, double* resid_dev, void* stream) {
  if (!b || !a_dev || !B_dev || !X_dev || !resid_dev || nrhs <= 0)
    return set_error(GLU_ARGUMENT_ERROR, "bad argument");
  if (!b->plan->has_grad) return set_error(GLU_NOT_READY, "no original pattern");
  if ((int64_t)nrhs * b->count > 65535)
    return set_error(GLU_ARGUMENT_ERROR, "count * nrhs must be <= 65535");
  glu::DeviceGuard g(b->plan->device);
  cudaStream_t s = (cudaStream_t)stream;
  int st = ensure_refine_workspace(b, (int64_t)b->count * nrhs, s);
  if (st) return st;
  glu::LaunchCounter lc;
  glu::launch_residual(b->plan->P, b->count, nrhs, a_dev, X_dev, B_dev, nullptr, b->norms,
                       resid_dev, transpose, s, lc);
  return glu::cuda_status("residual");
}

int glu_refine(glu_batch_t b, int32_t nrhs, const double* a_dev, const double* B_dev,
               double* X_dev, int32_t steps, int transpose, double* resid_dev, void* stream) {
  if (!b || !a_dev || !B_dev || !X_dev || nrhs <= 0 || steps < 0)
    return set_error(GLU_ARGUMENT_ERROR, "bad argument");
  if (!b->plan->has_grad || !b->plan->has_solve)
    return set_error(GLU_NOT_READY, "refinement needs the original pattern and solve maps");
  if (!b->factored) return set_error(GLU_NOT_READY, "refine before refactor");
  if ((int64_t)nrhs * b->count > 65535)
    return set_error(GLU_ARGUMENT_ERROR, "count * nrhs must be <= 65535");
  glu::DeviceGuard g(b->plan->device);
  int64_t nl = 0;
  int st = do_refine(b, nrhs, a_dev, B_dev, X_dev, steps, transpose, resid_dev,
                     (cudaStream_t)stream, &nl);
  b->launches = nl;
  return st;
}

int glu_grad_a(glu_batch_t b, int32_t nrhs, const double* lambda_dev, const double* x_dev,
               double* ga_dev, void* stream) {
  if (!b || !lambda_dev || !x_dev || !ga_dev || nrhs <= 0)
    return set_error(GLU_ARGUMENT_ERROR, "bad argument");
  if (!b->plan->has_grad) return set_error(GLU_NOT_READY, "no gradient pattern");
  glu::DeviceGuard g(b->plan->device);
  glu::LaunchCounter lc;
  glu::launch_grad(b->plan->P, b->count, nrhs, lambda_dev, x_dev, ga_dev, (cudaStream_t)stream, lc);
  b->launches = lc.n;
  return glu::cuda_status("grad");
}

int glu_get_lu(glu_batch_t b, int32_t instance, double* val_dev, void* stream) {
  if (!b || !val_dev || instance < 0 || instance >= b->count)
    return set_error(GLU_ARGUMENT_ERROR, "bad argument");
  glu::DeviceGuard g(b->plan->device);
  glu::LaunchCounter lc;
  glu::launch_export_lu(b->plan->P, b->vals, instance, val_dev, (cudaStream_t)stream, lc);
  return glu::cuda_status("export LU");
}

int glu_graph_capture(glu_batch_t b, const double* a_dev, int32_t nrhs, const double* B_dev,
                      double* X_dev, double pert, int32_t refine_steps, void* stream) {
  if (!b || !a_dev) return set_error(GLU_ARGUMENT_ERROR, "bad argument");
  if (!b->plan->has_ingest) return set_error(GLU_NOT_READY, "no ingest map");
  if (nrhs > 0 && (!B_dev || !X_dev || !b->plan->has_solve))
    return set_error(GLU_NOT_READY, "solve inputs / maps missing");
  glu::DeviceGuard g(b->plan->device);
  cudaStream_t s = (cudaStream_t)stream;
  if (!s) {
    if (!b->own_stream && cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking))
      return glu::cuda_status("stream create");
    s = b->own_stream;
  }
  if (refine_steps > 0 && (nrhs <= 0 || !b->plan->has_grad))
    return set_error(GLU_NOT_READY, "refinement needs right-hand sides and the original pattern");
  if (nrhs > 0) {
    int st = ensure_workspace(b, (int64_t)b->count * nrhs, s);
    if (st) return st;
    if (refine_steps > 0 && (st = ensure_refine_workspace(b, (int64_t)b->count * nrhs, s)))
      return st;
  }
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return glu::cuda_status("begin capture");
  glu::LaunchCounter lc;
  const bool asm_ok = glu::dense_assembly(b->plan->P);
  glu::launch_prepare_blob(b->plan->P, b->vals, 0, b->count, asm_ok, s, lc);
  glu::launch_ingest(b->plan->P, b->vals, 0, b->count, a_dev, s, lc);
  cudaMemsetAsync(b->asm_flag, asm_ok ? 1 : 0, b->count, s);
  b->loaded = true;
  int st = do_refactor(b, pert, s);
  int64_t total = lc.n + b->launches;
  if (st == GLU_OK && nrhs > 0) {
    st = do_solve(b, nrhs, B_dev, X_dev, 0, s);
    total += b->launches;
  }
  if (st == GLU_OK && refine_steps > 0) {
    int64_t nl = 0;
    st = do_refine(b, nrhs, a_dev, B_dev, X_dev, refine_steps, 0, nullptr, s, &nl);
    total += nl;
  }
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &graph);
  if (st != GLU_OK) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  if (e != cudaSuccess) return set_error(GLU_CUDA_ERROR, "end capture: %s", cudaGetErrorString(e));
  b->graph = graph;
  if (cudaGraphInstantiate(&b->exec, graph, 0) != cudaSuccess)
    return glu::cuda_status("graph instantiate");
  b->launches = total;
  return GLU_OK;
}

int glu_graph_launch(glu_batch_t b, void* stream) {
  if (!b || !b->exec) return set_error(GLU_NOT_READY, "no captured graph");
  glu::DeviceGuard g(b->plan->device);
  // NULL launches on the legacy default stream, like every other entry point
  if (cudaGraphLaunch(b->exec, (cudaStream_t)stream) != cudaSuccess)
    return glu::cuda_status("graph launch");
  b->factored = true;
  return GLU_OK;
}

}  // extern "C"

struct glu_group_s {
  int device = 0;
  std::vector<glu_batch_t> batches;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> events;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t launches = 0;
};

extern "C" {

int glu_group_destroy(glu_group_t g) {
  if (!g) return GLU_OK;
  glu::DeviceGuard dg(g->device);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  for (auto e : g->events) cudaEventDestroy(e);
  for (auto st : g->streams) cudaStreamDestroy(st);
  delete g;
  return GLU_OK;
}

int glu_group_capture(int32_t nbatch, const glu_batch_t* batches, const double* const* a_dev,
                      const int32_t* nrhs, const double* const* B_dev, double* const* X_dev,
                      double pert, int32_t refine_steps, void* stream, glu_group_t* out) {
  if (!out || nbatch <= 0 || !batches || !a_dev || !nrhs)
    return set_error(GLU_ARGUMENT_ERROR, "bad argument");
  *out = nullptr;
  const int dev = batches[0] ? batches[0]->plan->device : -1;
  for (int i = 0; i < nbatch; ++i) {
    glu_batch_t b = batches[i];
    if (!b || !a_dev[i]) return set_error(GLU_ARGUMENT_ERROR, "batch %d: null argument", i);
    if (b->plan->device != dev) return set_error(GLU_ARGUMENT_ERROR, "batches on different devices");
    if (!b->plan->has_ingest) return set_error(GLU_NOT_READY, "batch %d: no ingest map", i);
    if (nrhs[i] > 0 && (!B_dev || !X_dev || !B_dev[i] || !X_dev[i] || !b->plan->has_solve))
      return set_error(GLU_NOT_READY, "batch %d: solve inputs / maps missing", i);
    if (refine_steps > 0 && nrhs[i] > 0 && !b->plan->has_grad)
      return set_error(GLU_NOT_READY, "batch %d: refinement needs the original pattern", i);
    if ((int64_t)nrhs[i] * b->count > 65535)
      return set_error(GLU_ARGUMENT_ERROR, "batch %d: count * nrhs must be <= 65535", i);
  }
  glu::DeviceGuard dg(dev);
  glu_group_s* g = new (std::nothrow) glu_group_s();
  if (!g) return set_error(GLU_MEMORY_OVERFLOW, "host allocation failed");
  g->device = dev;
  g->batches.assign(batches, batches + nbatch);
  cudaStream_t s = (cudaStream_t)stream;
  int st = GLU_OK;
  // everything that allocates happens before the capture
  for (int i = 0; i < nbatch && st == GLU_OK; ++i) {
    if (nrhs[i] > 0) st = ensure_workspace(batches[i], (int64_t)batches[i]->count * nrhs[i], s);
    if (st == GLU_OK && nrhs[i] > 0 && refine_steps > 0)
      st = ensure_refine_workspace(batches[i], (int64_t)batches[i]->count * nrhs[i], s);
  }
  for (int i = 0; i < nbatch + 1 && st == GLU_OK; ++i) {
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      st = glu::cuda_status("event create");
      break;
    }
    g->events.push_back(e);
    if (i < nbatch) {
      cudaStream_t bs;
      if (cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking) != cudaSuccess) {
        st = glu::cuda_status("stream create");
        break;
      }
      g->streams.push_back(bs);
    }
  }
  if (st != GLU_OK) {
    glu_group_destroy(g);
    return st;
  }
  if (!s) {
    // capture needs a non-default origin stream
    cudaStream_t os;
    if (cudaStreamCreateWithFlags(&os, cudaStreamNonBlocking) != cudaSuccess) {
      glu_group_destroy(g);
      return glu::cuda_status("stream create");
    }
    g->streams.push_back(os);
    s = os;
  }
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    glu_group_destroy(g);
    return glu::cuda_status("begin capture");
  }
  cudaEvent_t fork = g->events[nbatch];
  cudaEventRecord(fork, s);
  int64_t total = 0;
  for (int i = 0; i < nbatch && st == GLU_OK; ++i) {
    glu_batch_t b = batches[i];
    cudaStream_t bs = g->streams[i];
    cudaStreamWaitEvent(bs, fork, 0);            // the branch joins the capture here
    glu::LaunchCounter lc;
    const bool asm_ok = glu::dense_assembly(b->plan->P);
    glu::launch_prepare_blob(b->plan->P, b->vals, 0, b->count, asm_ok, bs, lc);
    glu::launch_ingest(b->plan->P, b->vals, 0, b->count, a_dev[i], bs, lc);
    cudaMemsetAsync(b->asm_flag, asm_ok ? 1 : 0, b->count, bs);
    b->loaded = true;
    st = do_refactor(b, pert, bs);
    total += lc.n + b->launches;
    if (st == GLU_OK && nrhs[i] > 0) {
      st = do_solve(b, nrhs[i], B_dev[i], X_dev[i], 0, bs);
      total += b->launches;
    }
    if (st == GLU_OK && nrhs[i] > 0 && refine_steps > 0) {
      int64_t nl = 0;
      st = do_refine(b, nrhs[i], a_dev[i], B_dev[i], X_dev[i], refine_steps, 0, nullptr, bs, &nl);
      total += nl;
    }
    cudaEventRecord(g->events[i], bs);
    cudaStreamWaitEvent(s, g->events[i], 0);     // join back into the origin stream
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &graph);
  if (st != GLU_OK || e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    glu_group_destroy(g);
    return st != GLU_OK ? st : set_error(GLU_CUDA_ERROR, "end capture: %s", cudaGetErrorString(e));
  }
  g->graph = graph;
  if (cudaGraphInstantiate(&g->exec, graph, 0) != cudaSuccess) {
    glu_group_destroy(g);
    return glu::cuda_status("graph instantiate");
  }
  g->launches = total;
  *out = g;
  return GLU_OK;
}

int glu_group_launch(glu_group_t g, void* stream) {
  if (!g || !g->exec) return set_error(GLU_NOT_READY, "no captured group");
  glu::DeviceGuard dg(g->device);
  if (cudaGraphLaunch(g->exec, (cudaStream_t)stream) != cudaSuccess)
    return glu::cuda_status("group launch");
  for (auto b : g->batches) b->factored = true;
  return GLU_OK;
}

int glu_group_launch_count(glu_group_t g, int64_t* launches) {
  if (!g || !launches) return set_error(GLU_ARGUMENT_ERROR, "null argument");
  *launches = g->launches;
  return GLU_OK;
}

int glu_batch_launch_count(glu_batch_t b, int64_t* launches) {
  if (!b || !launches) return set_error(GLU_ARGUMENT_ERROR, "null argument");
  *launches = b->launches;
  return GLU_OK;
}

// Test hook: the trailing-update DMMA GEMM on caller buffers, C -= A * B (column-major).
int glu_debug_gemm_sub(int32_t M, int32_t N, int32_t K, const double* A, int32_t lda,
                       const double* B, int32_t ldb, double* C, int32_t ldc, int32_t count,
                       int64_t sA, int64_t sB, int64_t sC, int32_t variant, void* stream) {
  if (variant < 0 || variant >= glu::gemm_variants())
    return set_error(GLU_ARGUMENT_ERROR, "gemm variant");
  if (!A || !B || !C || M < 0 || N < 0 || K < 0 || (lda & 1) || (ldb & 1) || (M & 1) || (K & 1) ||
      lda < M || ldb < K || ldc < M || count <= 0 || count > 65535 ||
      (reinterpret_cast<uintptr_t>(A) & 15) || (reinterpret_cast<uintptr_t>(B) & 15) ||
      (sA & 1) || (sB & 1))
    return set_error(GLU_ARGUMENT_ERROR, "gemm arguments (even sizes/strides, 16-byte aligned)");
  glu::LaunchCounter lc;
  glu::launch_gemm_sub(M, N, K, A, lda, B, ldb, C, ldc, count, sA, sB, sC, (cudaStream_t)stream,
                       lc, variant);
  return glu::cuda_status("gemm");
}

}  // extern "C"
