// Host-side plan construction (pure C++; no CUDA).
#pragma once

#include <cstdint>
#include <vector>

#include "glu_b200.h"

namespace glu {

// One launch of the sparse level kernel: columns scols[begin, begin+ncols) form one level.
struct LevelLaunch {
  int32_t begin;
  int32_t ncols;
  int32_t mode;      // 0 = warp per column, 1 = CTA per column
  int32_t level;
};

struct HostPlan {
  uint32_t n = 0, nnz = 0, t = 0, nt = 0, ntp = 0;
  int64_t S = 0, dbase = 0, blob = 0;
  int32_t panel = 64;
  int32_t gemm_variant = 0;
  std::vector<uint32_t> cp, ri, lp, rp, ci, dp;
  std::vector<uint32_t> lsplit;
  std::vector<int64_t> pair_ptr;
  std::vector<int32_t> pair_j, pair_uslot;
  std::vector<int64_t> pair_moff;
  std::vector<int32_t> tmap;
  std::vector<int32_t> scols;
  std::vector<LevelLaunch> slevels;
  std::vector<int32_t> hubs;                 // sparse columns whose D contribution is a GEMM
  int32_t hubs_p = 0;
  std::vector<int32_t> gl_src, gl_dst, gu_src, gu_dst;
  std::vector<int64_t> pull_ptr;
  std::vector<int32_t> pull_c, pull_uslot;
  double dense_updates = 0, hub_updates = 0;
  std::vector<uint8_t> dhasl;
  std::vector<int64_t> pos2slot;
  std::vector<int32_t> lcols, lptr, ucols, uptr;
  std::vector<int64_t> bord_ptr;
  std::vector<int32_t> bord_row, bord_slot;
  double flops = 0.0;
  double flops_dense = 0.0;   // flops of the padded dense LU (what the dense kernels execute)
};

// Validates the Symbolic_Matrix arrays and builds the plan.  Returns a GLU_* status.
int build_host_plan(uint32_t n, uint32_t nnz, const uint32_t* cp, const uint32_t* ri,
                    const uint32_t* lp, const uint32_t* rp, const uint32_t* ci,
                    const uint32_t* dp, int32_t num_lev, const int32_t* level_ptr,
                    const int32_t* level_idx, const glu_options& opt, HostPlan& hp);

}  // namespace glu
