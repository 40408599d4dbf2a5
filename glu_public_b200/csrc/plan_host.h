// Host-side plan construction (pure C++; no CUDA).
#pragma once

#include <cstdint>
#include <vector>

#include "glu_b200.h"
#include "plan.h"

namespace glu {

// One level of the sparse phase: single columns scols[begin, begin+ncols) (one launch of the
// sparse level kernel) and fronts [f0, f1) (dense supernodal blocks, see Front).
struct LevelLaunch {
  int32_t begin;
  int32_t ncols;
  int32_t mode;      // 0 = one warp per column, 1 = several warps per column (see wpc)
  int32_t level;
  int32_t f0 = 0, f1 = 0;
  int32_t max_nl = 0;      // longest L part of the level's columns
  int32_t max_pairs = 0;   // most update pairs (c, j) of one column
  int32_t wpc = 1;         // warps sharing one column (1, 2, 4, 8)
  int32_t lanes = 32;      // lanes sharing one column when wpc = 1 (8, 16, 32)
  int32_t grow = 0;        // wide level of heavy columns: more warps per column while the
                           // level's columns of the batch leave the GPU short of warps
  int64_t t0 = 0, t1 = 0;  // deterministic mode: the level's target columns in det_tptr
};

// A front: a run of consecutive sparse columns S = [s0, s0+w) with identical structure below
// (rows R) and to the right (columns J) -- a fundamental supernode.  It is factored as a dense
// (wp+mp) x (wp+qp) block: [A(S,S) A(S,J); A(R,S) 0], padded to 64-multiples (identity on the
// padded pivots); after its w pivots the block's lower-right part holds -L(R,S) U(S,J), which is
// added to the targets.
struct Front {
  int32_t s0, w, wp, m, mp, q, qp, ld;
  int64_t size;                // ld * (wp + qp) doubles
  int64_t g_off, g_cnt;        // gather / write-back entries in fg_slot / fg_idx
  int64_t c_off, c_cnt;        // Schur-complement entries in fc_slot / fc_idx
  int64_t h_off;               // wp entries in fhasl
  int32_t level;
  int64_t foff = 0;            // offset of its buffer in an instance's front area
};

// The fronts of one level handled together, one launch per stage for all of them: fronts
// [f0, f0 + nf) (consecutive in HostPlan::fronts), their gather / write-back entries [g0, g1) and
// Schur-complement entries [c0, c1) (consecutive too), their buffers within the first `area`
// doubles of an instance's front area, and per 64-pivot step i (pivot k = 64 i) over the fronts
// that still have a pivot there: the largest trailing-update extents mmax / nmax and the most
// L21 + U12 tiles of 128 (tiles4) and of 32 (tiles1) rows or columns.
struct FrontLevel {
  int32_t f0 = 0, nf = 0;
  int64_t g0 = 0, g1 = 0, c0 = 0, c1 = 0, area = 0;
  std::vector<int32_t> mmax, nmax, tiles4, tiles1;
};

struct HostPlan {
  uint32_t n = 0, nnz = 0, t = 0, nt = 0, ntp = 0;
  int64_t S = 0, dbase = 0, blob = 0;
  int32_t panel = 64;
  int32_t gemm_variant = 0;
  int32_t update_depth = 1;
  int32_t sparse_block = 256;                // threads per CTA of the sparse level kernels
  int32_t level_warps = 64;                  // warps per SM the sparse level launches aim for
  int32_t cols_per_warp = 1;                 // columns a warp group takes in turn
  std::vector<uint32_t> cp, ri, lp, rp, ci, dp;
  std::vector<uint32_t> lsplit;
  std::vector<int64_t> pair_ptr;
  std::vector<int32_t> pair_j, pair_uslot;
  std::vector<int64_t> pair_moff;
  std::vector<int32_t> tmap;
  std::vector<int32_t> scols;
  std::vector<LevelLaunch> slevels;
  std::vector<Front> fronts;
  std::vector<int32_t> fg_slot, fg_idx, fc_slot, fc_idx;
  std::vector<uint8_t> fhasl;
  int64_t front_max = 0;                     // largest front buffer (doubles per instance)
  std::vector<FrontLevel> flevels;           // per entry of slevels (nf = 0: no fronts)
  std::vector<FrontGeom> fgeom;              // per front
  std::vector<int32_t> fg_aidx, fc_aidx;     // map indices within an instance's front area
  int64_t front_area = 0;                    // buffers of one level's fronts side by side
  double front_updates = 0;
  std::vector<int32_t> hubs;                 // sparse columns whose D contribution is a GEMM
  int32_t hubs_p = 0;
  std::vector<int32_t> gl_src, gl_dst, gu_src, gu_dst;
  std::vector<int64_t> pull_ptr;
  std::vector<int32_t> pull_uslot;
  std::vector<uint32_t> pull_lb, pull_le;
  std::vector<int64_t> pull_mend;            // [nt] end of the entries a column's own CTA pulls
  std::vector<int32_t> pull_xcol;            // [nx] column of each extra chunk of pull entries
  std::vector<int64_t> pull_xe;              // [2 nx] the chunk's entry range
  double dense_updates = 0, hub_updates = 0;
  std::vector<uint8_t> dhasl;
  std::vector<int64_t> pos2slot;
  std::vector<int32_t> lcols, lptr, ucols, uptr;
  // fronts in the solve schedules: level l runs fronts lfr[lfr_ptr[l] .. lfr_ptr[l+1])
  std::vector<int32_t> lfr, lfr_ptr, ufr, ufr_ptr;
  std::vector<int32_t> fs0, fw;               // first column and width of every front
  std::vector<int64_t> bord_ptr;
  std::vector<int32_t> bord_row, bord_slot;
  std::vector<int32_t> bord_ckcol;            // chunks of <= 1024 border entries: tail column
  std::vector<int64_t> bord_ck0;              //   and first entry
  double flops = 0.0;
  double flops_dense = 0.0;   // flops of the padded dense LU (what the dense kernels execute)
  // deterministic mode (no FP64 atomics, every sum in a fixed order): per level, the update
  // pairs (c, j) of its columns grouped by target column j, sources in the level's column order
  // within a target -- target k of the whole list owns pairs det_q[det_tptr[k] ..
  // det_tptr[k + 1]) (source columns det_c); and the slot of every CSR entry (row-wise solves)
  bool deterministic = false;
  std::vector<int64_t> det_q, det_tptr;
  std::vector<int32_t> det_c, csr_slot;
};

// Validates the Symbolic_Matrix arrays and builds the plan.  Returns a GLU_* status.
int build_host_plan(uint32_t n, uint32_t nnz, const uint32_t* cp, const uint32_t* ri,
                    const uint32_t* lp, const uint32_t* rp, const uint32_t* ci,
                    const uint32_t* dp, int32_t num_lev, const int32_t* level_ptr,
                    const int32_t* level_idx, const glu_options& opt, HostPlan& hp);

}  // namespace glu
