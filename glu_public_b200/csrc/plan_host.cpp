// Host-side plan construction: validation, sparse/dense split, slot layout, position maps and
// level schedules.  See plan.h for the value layout.
//
// What it replaces in the reference: LUonDevice's per-level mode selection
// (src/numeric.cu:423-596, thresholds 896/448/16) and the per-update search of the kernels
// (src/numeric.cu:57-89 scans the whole sub-column j for every (c, j) pair).  Here every (c, j)
// pair gets a precomputed run of target slots (the "position map"), and the trailing block that
// fill has made dense is split off for the dense kernels.
#include "plan_host.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <tuple>

#include "internal.h"
#include "plan.h"

namespace glu {

namespace {

int validate(uint32_t n, uint32_t nnz, const uint32_t* cp, const uint32_t* ri, const uint32_t* lp,
             const uint32_t* rp, const uint32_t* ci, const uint32_t* dp, int32_t num_lev,
             const int32_t* level_ptr, const int32_t* level_idx) {
  if (n == 0) return set_error(GLU_MATRIX_INVALID, "n == 0");
  if (cp[0] != 0 || cp[n] != nnz) return set_error(GLU_MATRIX_INVALID, "sym_c_ptr ends");
  for (uint32_t j = 0; j < n; ++j) {
    if (cp[j + 1] <= cp[j]) return set_error(GLU_MATRIX_INVALID, "empty column %u", j);
    for (uint32_t p = cp[j]; p < cp[j + 1]; ++p) {
      if (ri[p] >= n) return set_error(GLU_MATRIX_INVALID, "row out of range, col %u", j);
      if (p > cp[j] && ri[p] <= ri[p - 1])
        return set_error(GLU_MATRIX_INVALID, "rows not strictly increasing in column %u", j);
    }
    if (lp[j] < cp[j] || lp[j] >= cp[j + 1] || ri[lp[j]] != j)
      return set_error(GLU_MATRIX_STRUCTURAL_SINGULAR, "l_col_ptr[%u] is not the diagonal", j);
  }
  // the CSR mirror must be the transpose of the CSC pattern (src/symbolic.cc:55-79)
  std::vector<uint32_t> rp2, ci2, dp2;
  std::vector<uint32_t> vcp(cp, cp + n + 1), vri(ri, ri + nnz);
  symbolic_csr(n, vcp, vri, rp2, ci2, dp2);
  if (memcmp(rp2.data(), rp, 4 * (size_t)(n + 1)) || memcmp(ci2.data(), ci, 4 * (size_t)nnz) ||
      memcmp(dp2.data(), dp, 4 * (size_t)n))
    return set_error(GLU_MATRIX_INVALID, "CSR mirror does not match the CSC pattern");
  if (num_lev <= 0 || level_ptr[0] != 0 || level_ptr[num_lev] != (int32_t)n)
    return set_error(GLU_MATRIX_INVALID, "level_ptr ends");
  std::vector<int32_t> lev_of(n, -1);
  for (int32_t l = 0; l < num_lev; ++l) {
    if (level_ptr[l + 1] < level_ptr[l]) return set_error(GLU_MATRIX_INVALID, "level_ptr order");
    for (int32_t q = level_ptr[l]; q < level_ptr[l + 1]; ++q) {
      const int32_t c = level_idx[q];
      if (c < 0 || (uint32_t)c >= n || lev_of[c] >= 0)
        return set_error(GLU_MATRIX_INVALID, "level_idx is not a permutation");
      lev_of[c] = l;
    }
  }
  // every dependency of a column must sit in an earlier level (src/symbolic.cc:106-151)
  for (uint32_t i = 0; i < n; ++i) {
    for (uint32_t p = cp[i]; p < lp[i]; ++p) {
      const uint32_t k = ri[p];
      if (lp[k] + 1 != cp[k + 1] && lev_of[k] >= lev_of[i])
        return set_error(GLU_MATRIX_INVALID, "level order violates U dependency %u->%u", k, i);
    }
    for (uint32_t q = rp[i]; q < dp[i]; ++q)
      if (lev_of[ci[q]] >= lev_of[i])
        return set_error(GLU_MATRIX_INVALID, "level order violates L dependency %u->%u", ci[q], i);
  }
  return GLU_OK;
}

// Smallest t such that the trailing block [t, n)^2 has density >= thr and order >= min_order;
// n if none.  count[t] = number of entries with min(row, col) >= t.
uint32_t choose_split(uint32_t n, const uint32_t* cp, const uint32_t* ri, double thr,
                      int32_t min_order) {
  std::vector<uint64_t> cnt(n + 1, 0);
  for (uint32_t j = 0; j < n; ++j)
    for (uint32_t p = cp[j]; p < cp[j + 1]; ++p) cnt[std::min(j, ri[p])]++;
  for (int64_t t = (int64_t)n - 1; t >= 0; --t) cnt[t] += cnt[t + 1];
  if (min_order <= 0 || thr > 1.0) return n;
  for (uint32_t t = 0; t + (uint32_t)min_order <= n; ++t) {
    const double m = (double)(n - t);
    if ((double)cnt[t] >= thr * m * m) return t;
  }
  return n;
}

// Lanes that share one column on a level with a warp per column.  A group of g lanes walks a
// column's scaling and each of its update pairs in ceil(|L(:,c)| / g) steps of g lanes, so the
// level costs sum_c (pairs_c + 1) * ceil(|L(:,c)| / g) * g lane-steps; `fixed` (8, 16, 32) wins
// unless it is 0, then the smallest cost does, 32 unless a narrower group saves a quarter.
int32_t column_lanes(int32_t fixed, const uint32_t* cp, const uint32_t* lp,
                     const std::vector<int64_t>& pair_ptr, const int32_t* cols, int32_t ncols) {
  if (fixed == 8 || fixed == 16 || fixed == 32) return fixed;
  int64_t cost[3] = {0, 0, 0};                 // g = 8, 16, 32
  for (int32_t i = 0; i < ncols; ++i) {
    const int32_t c = cols[i];
    const int64_t nl = (int64_t)(cp[c + 1] - lp[c] - 1);
    const int64_t steps = pair_ptr[c + 1] - pair_ptr[c] + 1;
    for (int k = 0; k < 3; ++k) {
      const int64_t g = 8 << k;
      cost[k] += steps * ((nl + g - 1) / g) * g;
    }
  }
  int32_t best = 32;
  int64_t bc = cost[2];
  for (int k = 1; k >= 0; --k)
    if (4 * cost[k] <= 3 * bc) {
      best = 8 << k;
      bc = cost[k];
    }
  return best;
}

}  // namespace

int build_host_plan(uint32_t n, uint32_t nnz, const uint32_t* cp, const uint32_t* ri,
                    const uint32_t* lp, const uint32_t* rp, const uint32_t* ci,
                    const uint32_t* dp, int32_t num_lev, const int32_t* level_ptr,
                    const int32_t* level_idx, const glu_options& opt, HostPlan& hp) {
  int st = validate(n, nnz, cp, ri, lp, rp, ci, dp, num_lev, level_ptr, level_idx);
  if (st != GLU_OK) return st;
  hp.n = n;
  hp.nnz = nnz;
  hp.cp.assign(cp, cp + n + 1);
  hp.ri.assign(ri, ri + nnz);
  hp.lp.assign(lp, lp + n);
  hp.rp.assign(rp, rp + n + 1);
  hp.ci.assign(ci, ci + nnz);
  hp.dp.assign(dp, dp + n);
  hp.panel = opt.panel == 128 ? 128 : 64;
  hp.gemm_variant = opt.gemm_variant;
  hp.update_depth = opt.update_depth;
  hp.deterministic = opt.deterministic != 0;
  hp.sparse_block = opt.sparse_block == 128 ? 128 : 256;
  hp.level_warps = std::max(0, std::min(opt.level_warps_per_sm, 64));
  hp.cols_per_warp = opt.sparse_cols_per_warp == 2 || opt.sparse_cols_per_warp == 4
                         ? opt.sparse_cols_per_warp : 1;

  // ---- sparse / dense split ----
  const uint32_t t = choose_split(n, cp, ri, opt.dense_threshold, opt.dense_min);
  hp.t = t;
  hp.nt = n - t;
  // the dense block is padded (identity) to a whole number of panels, so every panel step and
  // every 64-row block of the dense kernels lies inside it
  const uint32_t align = (uint32_t)std::max(kDenseAlign, hp.panel);
  hp.ntp = hp.nt ? (uint32_t)(((hp.nt + align - 1) / align) * align) : 0;

  // ---- slots ----
  hp.pos2slot.assign(nnz, 0);
  int64_t s = 0;
  for (uint32_t j = 0; j < n; ++j)
    for (uint32_t p = cp[j]; p < cp[j + 1]; ++p)
      if (!(j >= t && ri[p] >= t)) hp.pos2slot[p] = s++;
  hp.S = s;
  hp.dbase = (s + 31) / 32 * 32;
  const int64_t dsize = (int64_t)hp.ntp * hp.ntp;
  hp.blob = (hp.dbase + dsize + 31) / 32 * 32;
  for (uint32_t j = t; j < n; ++j)
    for (uint32_t p = cp[j]; p < cp[j + 1]; ++p)
      if (ri[p] >= t)
        hp.pos2slot[p] = hp.dbase + (int64_t)(ri[p] - t) + (int64_t)(j - t) * hp.ntp;
  if (hp.blob >= ((int64_t)1 << 31))
    return set_error(GLU_BUDGET_EXCEEDED, "one instance needs %lld value slots (> 2^31)",
                     (long long)hp.blob);

  // ---- flops ----
  double f = 0.0;
  for (uint32_t c = 0; c < n; ++c) {
    const double nl = (double)(cp[c + 1] - lp[c] - 1), nu = (double)(rp[c + 1] - dp[c] - 1);
    f += nl + 2.0 * nl * nu;
  }
  hp.flops = f;
  {
    const double m = (double)hp.ntp;
    hp.flops_dense = m > 0 ? (2.0 / 3.0) * m * m * m : 0.0;
  }

  // ---- sparse columns: L split, (c, j) pairs and target-slot runs ----
  hp.lsplit.assign(t, 0);
  hp.pair_ptr.assign((size_t)t + 1, 0);
  for (uint32_t c = 0; c < t; ++c) {
    uint32_t k = lp[c] + 1;
    while (k < cp[c + 1] && ri[k] < t) ++k;
    hp.lsplit[c] = k - (lp[c] + 1);
    hp.pair_ptr[c + 1] = hp.pair_ptr[c] + (rp[c + 1] - dp[c] - 1);
  }
  const int64_t npairs = hp.pair_ptr[t];

  // ---- fronts: fundamental supernodes among the sparse columns ----
  std::vector<int32_t> front_of(t, -1);
  // fronts add their Schur complements to shared targets with atomics: none in deterministic mode
  if (opt.front_min_w > 0 && !hp.deterministic) {
    auto nLc = [&](uint32_t c) { return cp[c + 1] - lp[c] - 1; };
    auto nUc = [&](uint32_t c) { return rp[c + 1] - dp[c] - 1; };
    // column c continues the supernode of c - 1
    auto continues = [&](uint32_t c) {
      if (nLc(c - 1) != nLc(c) + 1 || nUc(c - 1) != nUc(c) + 1) return false;
      if (ri[lp[c - 1] + 1] != c || ci[dp[c - 1] + 1] != c) return false;
      if (memcmp(ri + lp[c - 1] + 2, ri + lp[c] + 1, 4 * (size_t)nLc(c))) return false;
      if (memcmp(ci + dp[c - 1] + 2, ci + dp[c] + 1, 4 * (size_t)nUc(c))) return false;
      return true;
    };
    const int64_t cap = (int64_t)1 << 27;      // doubles per instance (1 GiB)
    uint32_t s0 = 0;
    for (uint32_t c = 1; c <= t; ++c) {
      if (c < t && continues(c)) continue;
      const uint32_t s1 = c, w = s1 - s0;
      const uint32_t m = nLc(s1 - 1), q = nUc(s1 - 1);
      const double work = 2.0 * w * (double)m * q;
      Front f{};
      f.s0 = (int32_t)s0;
      f.w = (int32_t)w;
      // pivots padded to a whole number of panels (the dense steps work panel by panel)
      f.wp = (int32_t)((w + hp.panel - 1) / hp.panel * hp.panel);
      f.m = (int32_t)m;
      f.mp = (int32_t)((m + 63) / 64 * 64);
      f.q = (int32_t)q;
      f.qp = (int32_t)((q + 63) / 64 * 64);
      f.ld = f.wp + f.mp;
      f.size = (int64_t)f.ld * (f.wp + f.qp);
      if ((int32_t)w >= opt.front_min_w && work >= opt.front_min_flops && f.size <= cap) {
        for (uint32_t x = s0; x < s1; ++x) front_of[x] = (int32_t)hp.fronts.size();
        hp.fronts.push_back(f);
      }
      s0 = c;
    }
  }

  hp.pair_j.resize(npairs);
  hp.pair_uslot.resize(npairs);
  hp.pair_moff.resize(npairs);
  hp.tmap.clear();
  for (uint32_t c = 0; c < t; ++c) {
    const uint32_t l0 = lp[c] + 1, l1 = cp[c + 1];
    int64_t pi = hp.pair_ptr[c];
    if (front_of[c] >= 0) {              // a front applies this column's updates itself
      for (uint32_t q = dp[c] + 1; q < rp[c + 1]; ++q, ++pi) {
        hp.pair_j[pi] = (int32_t)ci[q];
        hp.pair_uslot[pi] = 0;
        hp.pair_moff[pi] = (int64_t)hp.tmap.size();
      }
      continue;
    }
    for (uint32_t q = dp[c] + 1; q < rp[c + 1]; ++q, ++pi) {
      const uint32_t j = ci[q];
      const uint32_t* b = ri + cp[j];
      const uint32_t* e = ri + cp[j + 1];
      const uint32_t* fpos = std::lower_bound(b, e, c);
      uint32_t k = (uint32_t)(fpos - ri);       // position of U(c, j) in column j
      hp.pair_j[pi] = (int32_t)j;
      hp.pair_uslot[pi] = (int32_t)hp.pos2slot[k];
      hp.pair_moff[pi] = (int64_t)hp.tmap.size();
      const uint32_t nmap = (j < t) ? (l1 - l0) : hp.lsplit[c];
      ++k;
      for (uint32_t p = l0; p < l0 + nmap; ++p) {
        const uint32_t r = ri[p];
        while (k < cp[j + 1] && ri[k] < r) ++k;
        if (k >= cp[j + 1] || ri[k] != r)
          return set_error(GLU_MATRIX_INVALID, "fill pattern is not closed: L(%u,%u) has no "
                           "target in column %u", r, c, j);
        hp.tmap.push_back((int32_t)hp.pos2slot[k]);
      }
      if (j >= t) {   // rows >= t land in D; check they exist in the pattern of column j
        for (uint32_t p = l0 + nmap; p < l1; ++p) {
          const uint32_t r = ri[p];
          while (k < cp[j + 1] && ri[k] < r) ++k;
          if (k >= cp[j + 1] || ri[k] != r)
            return set_error(GLU_MATRIX_INVALID, "fill pattern is not closed at (%u,%u)", r, j);
        }
      }
    }
  }

  if (hp.tmap.size() >= ((size_t)1 << 31))
    return set_error(GLU_BUDGET_EXCEEDED, "position map needs %zu entries", hp.tmap.size());

  // ---- front maps: gather / write-back entries and Schur-complement targets ----
  for (size_t fi = 0; fi < hp.fronts.size(); ++fi) {
    Front& f = hp.fronts[fi];
    const uint32_t s0 = (uint32_t)f.s0, s1 = s0 + (uint32_t)f.w, last = s1 - 1;
    const uint32_t* R = ri + lp[last] + 1;          // rows below the front
    const uint32_t* J = ci + dp[last] + 1;          // columns right of the front
    f.g_off = (int64_t)hp.fg_slot.size();
    for (uint32_t x = s0; x < s1; ++x) {            // columns of S: rows s0.. then R
      uint32_t p = (uint32_t)(std::lower_bound(ri + cp[x], ri + cp[x + 1], s0) - ri);
      for (uint32_t i = s0; i < s1; ++i, ++p) {
        if (p >= cp[x + 1] || ri[p] != i)
          return set_error(GLU_MATRIX_INVALID, "front %zu: column %u misses row %u", fi, x, i);
        hp.fg_slot.push_back((int32_t)hp.pos2slot[p]);
        hp.fg_idx.push_back((int32_t)((i - s0) + (int64_t)(x - s0) * f.ld));
      }
      for (int32_t rr = 0; rr < f.m; ++rr, ++p) {
        if (p >= cp[x + 1] || ri[p] != R[rr])
          return set_error(GLU_MATRIX_INVALID, "front %zu: column %u misses a row of R", fi, x);
        hp.fg_slot.push_back((int32_t)hp.pos2slot[p]);
        hp.fg_idx.push_back((int32_t)((f.wp + rr) + (int64_t)(x - s0) * f.ld));
      }
    }
    for (int32_t jj = 0; jj < f.q; ++jj) {          // U(S, J)
      const uint32_t j = J[jj];
      uint32_t p = (uint32_t)(std::lower_bound(ri + cp[j], ri + cp[j + 1], s0) - ri);
      for (uint32_t i = s0; i < s1; ++i, ++p) {
        if (p >= cp[j + 1] || ri[p] != i)
          return set_error(GLU_MATRIX_INVALID, "front %zu: column %u misses row %u", fi, j, i);
        hp.fg_slot.push_back((int32_t)hp.pos2slot[p]);
        hp.fg_idx.push_back((int32_t)((i - s0) + (int64_t)(f.wp + jj) * f.ld));
      }
    }
    f.g_cnt = (int64_t)hp.fg_slot.size() - f.g_off;
    f.c_off = (int64_t)hp.fc_slot.size();
    for (int32_t jj = 0; jj < f.q; ++jj) {          // targets of C(R, J)
      const uint32_t j = J[jj];
      uint32_t k = (uint32_t)(std::lower_bound(ri + cp[j], ri + cp[j + 1], s1) - ri);
      for (int32_t rr = 0; rr < f.m; ++rr) {
        while (k < cp[j + 1] && ri[k] < R[rr]) ++k;
        if (k >= cp[j + 1] || ri[k] != R[rr])
          return set_error(GLU_MATRIX_INVALID, "fill pattern is not closed at (%u,%u)", R[rr], j);
        hp.fc_slot.push_back((int32_t)hp.pos2slot[k]);
        hp.fc_idx.push_back((int32_t)((f.wp + rr) + (int64_t)(f.wp + jj) * f.ld));
      }
    }
    f.c_cnt = (int64_t)hp.fc_slot.size() - f.c_off;
    f.h_off = (int64_t)hp.fhasl.size();
    for (int32_t kk = 0; kk < f.wp; ++kk)
      hp.fhasl.push_back(kk < f.w && lp[s0 + kk] + 1 < cp[s0 + kk + 1] ? 1 : 0);
    hp.front_max = std::max(hp.front_max, f.size);
    for (uint32_t x = s0; x < s1; ++x)
      hp.front_updates += (double)(cp[x + 1] - lp[x] - 1) * (double)(rp[x + 1] - dp[x] - 1);
  }
  if (hp.fc_slot.size() >= ((size_t)1 << 31) || hp.fg_slot.size() >= ((size_t)1 << 31))
    return set_error(GLU_BUDGET_EXCEEDED, "front maps too large");

  // ---- contributions of the sparse columns to the dense block ----
  // L21(:,c) * U12(c,:) for every c < t.  The columns with the largest outer products ("hubs")
  // are gathered into dense panels and applied as one GEMM; the rest are pulled per tail column.
  if (hp.nt > 0) {
    std::vector<int64_t> w(t, 0);
    std::vector<uint32_t> ut(t, 0);
    for (uint32_t c = 0; c < t; ++c) {
      if (front_of[c] >= 0) continue;        // fronts add their part of L21*U12 themselves
      const uint32_t lt = (cp[c + 1] - lp[c] - 1) - hp.lsplit[c];
      for (int64_t q = hp.pair_ptr[c]; q < hp.pair_ptr[c + 1]; ++q)
        if ((uint32_t)hp.pair_j[q] >= t) ut[c]++;
      w[c] = (int64_t)lt * ut[c];
      hp.dense_updates += (double)w[c];
    }
    std::vector<int32_t> order;
    for (uint32_t c = 0; c < t; ++c)
      if (w[c] > 0) order.push_back((int32_t)c);
    std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
      return w[a] != w[b] ? w[a] > w[b] : a < b;
    });
    // a column becomes a hub when its outer product is at least hub_min_frac of a dense rank-1
    // update of the block (the GEMM then wastes at most 1/hub_min_frac of its work)
    const double frac = opt.hub_min_frac > 0 ? opt.hub_min_frac : 0.02;
    const int32_t cap = opt.hub_max > 0 ? opt.hub_max : 256;
    const double dense_rank1 = (double)hp.ntp * hp.ntp;
    std::vector<uint8_t> is_hub(t, 0);
    for (int32_t c : order) {
      if ((int32_t)hp.hubs.size() >= cap || (double)w[c] < frac * dense_rank1) break;
      is_hub[c] = 1;
      hp.hub_updates += (double)w[c];
      hp.hubs.push_back(c);
    }
    hp.hubs_p = hp.hubs.empty() ? 0 : (int32_t)((hp.hubs.size() + 15) / 16 * 16);
    for (size_t hi = 0; hi < hp.hubs.size(); ++hi) {
      const uint32_t c = (uint32_t)hp.hubs[hi];
      for (uint32_t p = lp[c] + 1 + hp.lsplit[c]; p < cp[c + 1]; ++p) {
        hp.gl_src.push_back((int32_t)p);
        hp.gl_dst.push_back((int32_t)((ri[p] - t) + (int64_t)hi * hp.ntp));
      }
      for (int64_t q = hp.pair_ptr[c]; q < hp.pair_ptr[c + 1]; ++q) {
        const uint32_t j = (uint32_t)hp.pair_j[q];
        if (j < t) continue;
        hp.gu_src.push_back(hp.pair_uslot[q]);
        hp.gu_dst.push_back((int32_t)(hi + (int64_t)(j - t) * hp.hubs_p));
      }
    }
    hp.pull_ptr.assign((size_t)hp.nt + 1, 0);
    for (uint32_t c = 0; c < t; ++c) {
      if (is_hub[c] || w[c] == 0) continue;
      for (int64_t q = hp.pair_ptr[c]; q < hp.pair_ptr[c + 1]; ++q)
        if ((uint32_t)hp.pair_j[q] >= t) hp.pull_ptr[hp.pair_j[q] - t + 1]++;
    }
    for (uint32_t jt = 0; jt < hp.nt; ++jt) hp.pull_ptr[jt + 1] += hp.pull_ptr[jt];
    hp.pull_lb.assign(hp.pull_ptr[hp.nt], 0);
    hp.pull_le.assign(hp.pull_ptr[hp.nt], 0);
    hp.pull_uslot.assign(hp.pull_ptr[hp.nt], 0);
    std::vector<int64_t> fill(hp.pull_ptr.begin(), hp.pull_ptr.end() - 1);
    for (uint32_t c = 0; c < t; ++c) {
      if (is_hub[c] || w[c] == 0) continue;
      for (int64_t q = hp.pair_ptr[c]; q < hp.pair_ptr[c + 1]; ++q) {
        const uint32_t j = (uint32_t)hp.pair_j[q];
        if (j < t) continue;
        const int64_t e = fill[j - t]++;
        hp.pull_lb[e] = hp.lp[c] + 1 + hp.lsplit[c];
        hp.pull_le[e] = hp.cp[c + 1];
        hp.pull_uslot[e] = hp.pair_uslot[q];
      }
    }
    // Columns whose pulls carry far more updates than the average keep a prefix of about twice
    // the average for their own CTA; the rest of their entries become chunks of that size for
    // extra CTAs, which add into the written column afterwards (one matrix leaves the GPU a few
    // waves of column CTAs, and the heaviest column would otherwise set the kernel's time).
    int64_t total = 0;
    for (size_t e = 0; e < hp.pull_lb.size(); ++e) total += hp.pull_le[e] - hp.pull_lb[e];
    const int64_t chunk = std::max<int64_t>(1024, hp.nt ? 2 * total / hp.nt : 0);
    hp.pull_mend.assign(hp.nt, 0);
    hp.pull_xcol.clear();
    hp.pull_xe.clear();
    for (uint32_t jt = 0; jt < hp.nt; ++jt) {
      int64_t e = hp.pull_ptr[jt], acc = 0;
      const int64_t e1 = hp.pull_ptr[jt + 1];
      while (e < e1 && acc < chunk) acc += hp.pull_le[e] - hp.pull_lb[e], ++e;
      hp.pull_mend[jt] = e;
      while (e < e1) {
        const int64_t c0 = e;
        for (acc = 0; e < e1 && acc < chunk; ++e) acc += hp.pull_le[e] - hp.pull_lb[e];
        hp.pull_xcol.push_back((int32_t)jt);
        hp.pull_xe.push_back(c0);
        hp.pull_xe.push_back(e);
      }
    }
    if (hp.pull_xcol.empty()) hp.pull_mend.clear();
  }

  // ---- sparse factor levels ----
  // Without fronts: the reference's level sets restricted to c < t.  With fronts: levels of the
  // "units" (a front or a single column), computed with the reference's dependency rules
  // (symbolic.cc:106-151) on the graph where each front's columns are one node.  Dependencies
  // always point to lower column indices, so collapsing a contiguous run keeps the graph acyclic.
  std::vector<std::vector<int32_t>> lev_cols;
  std::vector<std::vector<int32_t>> lev_fronts;
  if (hp.fronts.empty()) {
    for (int32_t l = 0; l < num_lev; ++l) {
      std::vector<int32_t> cols;
      for (int32_t q = level_ptr[l]; q < level_ptr[l + 1]; ++q)
        if ((uint32_t)level_idx[q] < t) cols.push_back(level_idx[q]);
      lev_cols.push_back(std::move(cols));
      lev_fronts.emplace_back();
    }
  } else {
    std::vector<int32_t> ulev(t, 0), facc(hp.fronts.size(), 0);
    auto lvl = [&](uint32_t k) { return front_of[k] >= 0 ? hp.fronts[front_of[k]].level : ulev[k]; };
    int32_t maxl = -1;
    for (uint32_t c = 0; c < t; ++c) {
      const int32_t F = front_of[c];
      int32_t m = -1;
      for (uint32_t p = cp[c]; p < lp[c]; ++p) {
        const uint32_t k = ri[p];
        if (lp[k] + 1 != cp[k + 1] && (F < 0 || front_of[k] != F)) m = std::max(m, lvl(k));
      }
      for (uint32_t q = rp[c]; q < dp[c]; ++q) {
        const uint32_t k = ci[q];
        if (F < 0 || front_of[k] != F) m = std::max(m, lvl(k));
      }
      if (F < 0) {
        ulev[c] = m + 1;
        maxl = std::max(maxl, ulev[c]);
      } else {
        facc[F] = std::max(facc[F], m + 1);
        if ((int32_t)c == hp.fronts[F].s0 + hp.fronts[F].w - 1) {
          hp.fronts[F].level = facc[F];
          maxl = std::max(maxl, facc[F]);
        }
      }
    }
    lev_cols.assign(maxl + 1, {});
    lev_fronts.assign(maxl + 1, {});
    for (uint32_t c = 0; c < t; ++c)
      if (front_of[c] < 0) lev_cols[ulev[c]].push_back((int32_t)c);
    for (size_t fi = 0; fi < hp.fronts.size(); ++fi)
      lev_fronts[hp.fronts[fi].level].push_back((int32_t)fi);
    // keep fronts ordered by level in the array
    std::vector<Front> sorted;
    std::vector<int32_t> remap(hp.fronts.size());
    for (auto& lf : lev_fronts)
      for (int32_t& fi : lf) {
        remap[fi] = (int32_t)sorted.size();
        sorted.push_back(hp.fronts[fi]);
        fi = remap[fi];
      }
    hp.fronts.swap(sorted);
    // the fronts of one level are independent (every dependency through a row or a column puts
    // the later unit on a later level), so each gets its own buffer and they may run concurrently
    hp.front_area = 0;
    for (const auto& lf : lev_fronts) {
      int64_t off = 0;
      for (int32_t fi : lf) {
        hp.fronts[fi].foff = off;
        off += (hp.fronts[fi].size + 31) / 32 * 32;
      }
      hp.front_area = std::max(hp.front_area, off);
    }
    if (hp.front_area >= ((int64_t)1 << 31))
      return set_error(GLU_BUDGET_EXCEEDED, "front buffers of one level exceed 2^31 doubles");
    // the maps in level order (so a level's entries are consecutive), with indices within an
    // instance's front area
    std::vector<int32_t> gs, gx, cs, cx;
    std::vector<uint8_t> hs;
    gs.reserve(hp.fg_slot.size());
    cs.reserve(hp.fc_slot.size());
    hp.fg_aidx.clear();
    hp.fc_aidx.clear();
    hp.fgeom.clear();
    for (Front& f : hp.fronts) {
      const int64_t g0 = (int64_t)gs.size(), c0 = (int64_t)cs.size(), h0 = (int64_t)hs.size();
      for (int64_t e = f.g_off; e < f.g_off + f.g_cnt; ++e) {
        gs.push_back(hp.fg_slot[e]);
        gx.push_back(hp.fg_idx[e]);
        hp.fg_aidx.push_back((int32_t)(f.foff + hp.fg_idx[e]));
      }
      for (int64_t e = f.c_off; e < f.c_off + f.c_cnt; ++e) {
        cs.push_back(hp.fc_slot[e]);
        cx.push_back(hp.fc_idx[e]);
        hp.fc_aidx.push_back((int32_t)(f.foff + hp.fc_idx[e]));
      }
      hs.insert(hs.end(), hp.fhasl.begin() + f.h_off, hp.fhasl.begin() + f.h_off + f.wp);
      f.g_off = g0;
      f.c_off = c0;
      f.h_off = h0;
      hp.fgeom.push_back(FrontGeom{f.foff, f.h_off, f.ld, f.wp + f.qp, f.w, f.wp});
    }
    hp.fg_slot.swap(gs);
    hp.fg_idx.swap(gx);
    hp.fc_slot.swap(cs);
    hp.fc_idx.swap(cx);
    hp.fhasl.swap(hs);
  }
  hp.scols.clear();
  hp.slevels.clear();
  const int32_t wpc = opt.sparse_warps_per_col;
  int32_t fcur = 0;
  for (int32_t l = 0; l < (int32_t)lev_cols.size(); ++l) {
    const int32_t begin = (int32_t)hp.scols.size();
    int64_t work = 0;
    int32_t max_nl = 0, max_pairs = 0;
    for (int32_t c : lev_cols[l]) {
      hp.scols.push_back(c);
      work += (int64_t)(cp[c + 1] - lp[c]) * (int64_t)(rp[c + 1] - dp[c]);
      max_nl = std::max(max_nl, (int32_t)(cp[c + 1] - lp[c] - 1));
      max_pairs = std::max(max_pairs, (int32_t)(hp.pair_ptr[c + 1] - hp.pair_ptr[c]));
    }
    const int32_t ncols = (int32_t)hp.scols.size() - begin;
    const int32_t nf = (int32_t)lev_fronts[l].size();
    if (ncols == 0 && nf == 0) continue;
    if (ncols == 0) {
      hp.slevels.push_back({begin, 0, 0, l, fcur, fcur + nf});
      fcur += nf;
      continue;
    }
    // narrow levels (few columns, much work per column) get a CTA's warps per column so their
    // work spreads over the SMs; wide levels get a warp per column (src/numeric.cu:423-545 makes
    // the same split with fixed thresholds)
    const int32_t wide = opt.wide_level_cols > 0 ? opt.wide_level_cols : 4 * 148;
    const int32_t cwork = opt.narrow_col_work > 0 ? opt.narrow_col_work : 256;
    int32_t w = wpc;
    const bool by_level = w != 1 && w != 2 && w != 4 && w != 8;
    if (by_level) w = (ncols < wide && work / ncols > cwork) ? 8 : 1;
    w = std::min(w, hp.sparse_block / 32);
    hp.slevels.push_back({begin, ncols, w > 1 ? 1 : 0, l, fcur, fcur + nf, max_nl, max_pairs, w});
    hp.slevels.back().lanes = w == 1 ? column_lanes(opt.sparse_col_lanes, cp, lp, hp.pair_ptr,
                                                    hp.scols.data() + begin, ncols)
                                     : 32;
    hp.slevels.back().grow = by_level && w == 1 && work / ncols > cwork ? 1 : 0;
    fcur += nf;
  }

  // ---- fronts of each level, handled together ----
  hp.flevels.assign(hp.slevels.size(), FrontLevel{});
  for (size_t li = 0; li < hp.slevels.size(); ++li) {
    const LevelLaunch& L = hp.slevels[li];
    if (L.f1 <= L.f0) continue;
    FrontLevel& F = hp.flevels[li];
    F.f0 = L.f0;
    F.nf = L.f1 - L.f0;
    const Front& a = hp.fronts[L.f0];
    const Front& z = hp.fronts[L.f1 - 1];
    F.g0 = a.g_off;
    F.g1 = z.g_off + z.g_cnt;
    F.c0 = a.c_off;
    F.c1 = z.c_off + z.c_cnt;
    int32_t wmax = 0;
    for (int32_t fi = L.f0; fi < L.f1; ++fi) {
      const Front& f = hp.fronts[fi];
      F.area = std::max(F.area, f.foff + f.size);
      wmax = std::max(wmax, f.w);
    }
    for (int32_t k = 0; k < wmax; k += 64) {
      int32_t mm = 0, nn = 0, t4 = 0, t1 = 0;
      for (int32_t fi = L.f0; fi < L.f1; ++fi) {
        const Front& f = hp.fronts[fi];
        if (k >= f.w) continue;
        const int32_t m = f.ld - k - 64, q = f.wp + f.qp - k - 64;
        mm = std::max(mm, m);
        nn = std::max(nn, q);
        t4 = std::max(t4, (m + 127) / 128 + (q + 127) / 128);
        t1 = std::max(t1, (m + 31) / 32 + (q + 31) / 32);
      }
      F.mmax.push_back(mm);
      F.nmax.push_back(nn);
      F.tiles4.push_back(t4);
      F.tiles1.push_back(t1);
    }
  }

  // ---- deterministic mode: each level's pairs grouped by target column ----
  if (hp.deterministic) {
    hp.det_q.clear();
    hp.det_c.clear();
    hp.det_tptr.assign(1, 0);
    std::vector<std::tuple<int32_t, int32_t, int64_t>> v;   // (target j, rank of c, pair)
    for (LevelLaunch& L : hp.slevels) {
      L.t0 = (int64_t)hp.det_tptr.size() - 1;
      v.clear();
      for (int32_t k = 0; k < L.ncols; ++k) {
        const int32_t c = hp.scols[L.begin + k];
        for (int64_t q = hp.pair_ptr[c]; q < hp.pair_ptr[c + 1]; ++q)
          v.emplace_back(hp.pair_j[q], k, q);
      }
      std::sort(v.begin(), v.end());
      for (size_t i = 0; i < v.size(); ++i) {
        if (i > 0 && std::get<0>(v[i]) != std::get<0>(v[i - 1]))
          hp.det_tptr.push_back((int64_t)hp.det_q.size());
        hp.det_q.push_back(std::get<2>(v[i]));
        hp.det_c.push_back(hp.scols[L.begin + std::get<1>(v[i])]);
      }
      if (!v.empty()) hp.det_tptr.push_back((int64_t)hp.det_q.size());
      L.t1 = (int64_t)hp.det_tptr.size() - 1;
    }
    // slot of every CSR entry outside the dense block (-1 inside it): rows are walked in column
    // order, exactly as the CSR mirror was built (symbolic.cc:55-79)
    if (hp.S >= ((int64_t)1 << 31))
      return set_error(GLU_BUDGET_EXCEEDED, "deterministic mode needs < 2^31 sparse slots");
    hp.csr_slot.assign(nnz, -1);
    std::vector<uint32_t> fill(rp, rp + n);
    for (uint32_t j = 0; j < n; ++j)
      for (uint32_t p = cp[j]; p < cp[j + 1]; ++p) {
        const int64_t sl = hp.pos2slot[p];
        hp.csr_slot[fill[ri[p]]++] = sl < hp.dbase ? (int32_t)sl : -1;
      }
  }

  // ---- dense block: which columns have an L part (perturbation applies only there) ----
  hp.dhasl.assign(hp.ntp, 0);
  for (uint32_t j = t; j < n; ++j) hp.dhasl[j - t] = (lp[j] + 1 < cp[j + 1]) ? 1 : 0;

  // ---- solve schedules over the sparse columns ----
  // Single columns by level; a front is one unit (its columns solved in order by one CTA).
  {
    const int32_t nf = (int32_t)hp.fronts.size();
    std::vector<int32_t> fid(t, -1);
    hp.fs0.assign(nf, 0);
    hp.fw.assign(nf, 0);
    for (int32_t f = 0; f < nf; ++f) {
      hp.fs0[f] = hp.fronts[f].s0;
      hp.fw[f] = hp.fronts[f].w;
      for (int32_t x = 0; x < hp.fronts[f].w; ++x) fid[hp.fronts[f].s0 + x] = f;
    }
    auto build = [&](bool lower, std::vector<int32_t>& cols, std::vector<int32_t>& ptr,
                     std::vector<int32_t>& fr, std::vector<int32_t>& frptr) {
      std::vector<int32_t> lev(t, 0), flev(nf, 0);
      auto lv = [&](uint32_t k) { return fid[k] >= 0 ? flev[fid[k]] : lev[k]; };
      int32_t maxl = -1;
      for (uint32_t step = 0; step < t; ++step) {
        const uint32_t c = lower ? step : t - 1 - step;
        const int32_t F = fid[c];
        int32_t m = -1;
        if (lower) {                 // c after every k with L(c, k) != 0
          for (uint32_t q = rp[c]; q < dp[c]; ++q)
            if (F < 0 || fid[ci[q]] != F) m = std::max(m, lv(ci[q]));
        } else {                     // c after every j < t with U(c, j) != 0
          for (uint32_t q = dp[c] + 1; q < rp[c + 1]; ++q)
            if (ci[q] < t && (F < 0 || fid[ci[q]] != F)) m = std::max(m, lv(ci[q]));
        }
        if (F < 0) {
          lev[c] = m + 1;
        } else {
          flev[F] = std::max(flev[F], m + 1);
        }
        maxl = std::max(maxl, m + 1);
      }
      ptr.assign(maxl + 2, 0);
      frptr.assign(maxl + 2, 0);
      for (uint32_t c = 0; c < t; ++c)
        if (fid[c] < 0) ptr[lev[c] + 1]++;
      for (int32_t f = 0; f < nf; ++f) frptr[flev[f] + 1]++;
      for (int32_t l = 0; l <= maxl; ++l) {
        ptr[l + 1] += ptr[l];
        frptr[l + 1] += frptr[l];
      }
      cols.assign(ptr[maxl + 1], 0);
      fr.assign(nf, 0);
      std::vector<int32_t> fc(ptr.begin(), ptr.end() - 1), ff(frptr.begin(), frptr.end() - 1);
      for (uint32_t c = 0; c < t; ++c)
        if (fid[c] < 0) cols[fc[lev[c]]++] = (int32_t)c;
      for (int32_t f = 0; f < nf; ++f) fr[ff[flev[f]]++] = f;
    };
    build(true, hp.lcols, hp.lptr, hp.lfr, hp.lfr_ptr);
    build(false, hp.ucols, hp.uptr, hp.ufr, hp.ufr_ptr);
  }
  hp.bord_ptr.assign((size_t)hp.nt + 1, 0);
  hp.bord_row.clear();
  hp.bord_slot.clear();
  for (uint32_t j = t; j < n; ++j) {
    for (uint32_t p = cp[j]; p < cp[j + 1] && ri[p] < t; ++p) {
      hp.bord_row.push_back((int32_t)ri[p]);
      hp.bord_slot.push_back((int32_t)hp.pos2slot[p]);
    }
    hp.bord_ptr[j - t + 1] = (int64_t)hp.bord_row.size();
  }
  // the border of the forward solve in chunks of at most kBorderChunk entries, a warp each, so a
  // long column is shared by several warps
  constexpr int64_t kBorderChunk = 1024;
  hp.bord_ckcol.clear();
  hp.bord_ck0.clear();
  for (uint32_t jt = 0; jt < hp.nt; ++jt)
    for (int64_t e = hp.bord_ptr[jt]; e < hp.bord_ptr[jt + 1]; e += kBorderChunk) {
      hp.bord_ckcol.push_back((int32_t)jt);
      hp.bord_ck0.push_back(e);
    }
  return GLU_OK;
}

}  // namespace glu
