// Fast symbolic analysis with the same output, bit for bit, as the reference's
// Symbolic_Matrix::fill_in / csr / leveling (src/symbolic.cc:11-151).
//
// fill_in (src/symbolic.cc:11-53) grows column i by repeated std::set_union with the L part of
// every column k < i already in its pattern; that costs a merge of the whole column per union
// and took minutes at n = 20,000.  The pattern it produces is the reach of A(:,i) in the graph
// of L restricted to expansion through nodes k < i.  Here the reach is computed by an iterative
// depth-first search over a *pruned* L graph (Eisenstat & Liu symmetric pruning: once column i
// has U(j,i) != 0 and L(i,j) != 0, rows of L(:,j) below i are reachable through i and are
// dropped from j's adjacency), then sorted.  The set is identical, so the sorted columns,
// l_col_ptr, the CSR mirror and the levels are identical.
//
// csr (src/symbolic.cc:55-79) and leveling (src/symbolic.cc:106-151) are restated directly:
// they are already linear in nnz.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include "glu_b200.h"
#include "internal.h"

struct glu_symbolic_s {
  uint32_t n = 0;
  uint32_t nnz = 0;
  int32_t num_lev = 0;
  std::vector<uint32_t> cp, ri, lp, rp, ci, dp;
  std::vector<int32_t> lev_ptr, lev_idx;
};

namespace glu {

int symbolic_fill(uint32_t n, const uint32_t* ap, const uint32_t* ai, std::vector<uint32_t>& cp,
                  std::vector<uint32_t>& ri, std::vector<uint32_t>& lp) {
  cp.assign(1, 0);
  cp.reserve(n + 1);
  lp.clear();
  lp.reserve(n);
  ri.clear();
  ri.reserve((size_t)ap[n] * 4);
  std::vector<uint32_t> prune_end(n, 0);  // end of the (pruned) L adjacency of column k in ri
  std::vector<uint8_t> pruned(n, 0);
  std::vector<int64_t> mark(n, -1);
  std::vector<uint32_t> pat;
  std::vector<uint32_t> stack;
  pat.reserve(1024);
  stack.reserve(1024);
  for (uint32_t i = 0; i < n; ++i) {
    pat.clear();
    for (uint32_t e = ap[i]; e < ap[i + 1]; ++e) {
      const uint32_t r0 = ai[e];
      if (r0 >= n) return set_error(GLU_MATRIX_INVALID, "row index out of range in column %u", i);
      if (mark[r0] == (int64_t)i) continue;
      mark[r0] = i;
      pat.push_back(r0);
      if (r0 >= i) continue;
      stack.push_back(r0);
      while (!stack.empty()) {
        const uint32_t k = stack.back();
        stack.pop_back();
        for (uint32_t p = lp[k] + 1; p < prune_end[k]; ++p) {
          const uint32_t r = ri[p];
          if (mark[r] == (int64_t)i) continue;
          mark[r] = i;
          pat.push_back(r);
          if (r < i) stack.push_back(r);
        }
      }
    }
    std::sort(pat.begin(), pat.end());
    const uint32_t base = cp.back();
    auto d = std::lower_bound(pat.begin(), pat.end(), i);
    if (d == pat.end() || *d != i)
      return set_error(GLU_MATRIX_STRUCTURAL_SINGULAR, "column %u has no structural diagonal", i);
    lp.push_back(base + (uint32_t)(d - pat.begin()));
    ri.insert(ri.end(), pat.begin(), pat.end());
    cp.push_back(base + (uint32_t)pat.size());
    prune_end[i] = cp.back();
    // symmetric pruning of every L(:,j) with U(j,i) != 0 and L(i,j) != 0
    for (auto it = pat.begin(); it != d; ++it) {
      const uint32_t j = *it;
      if (pruned[j]) continue;
      const uint32_t* b = ri.data() + lp[j] + 1;
      const uint32_t* e = ri.data() + cp[j + 1];
      const uint32_t* f = std::lower_bound(b, e, i);
      if (f != e && *f == i) {
        prune_end[j] = (uint32_t)(f - ri.data()) + 1;
        pruned[j] = 1;
      }
    }
    if (cp.back() < base) return set_error(GLU_MATRIX_INVALID, "nnz of L+U overflows 32 bits");
  }
  return GLU_OK;
}

void symbolic_csr(uint32_t n, const std::vector<uint32_t>& cp, const std::vector<uint32_t>& ri,
                  std::vector<uint32_t>& rp, std::vector<uint32_t>& ci,
                  std::vector<uint32_t>& dp) {
  const uint32_t nnz = cp[n];
  rp.assign(n + 1, 0);
  for (uint32_t p = 0; p < nnz; ++p) rp[ri[p] + 1]++;
  for (uint32_t i = 0; i < n; ++i) rp[i + 1] += rp[i];
  ci.assign(nnz, 0);
  dp.assign(n, 0);
  std::vector<uint32_t> fill(rp.begin(), rp.end() - 1);
  for (uint32_t j = 0; j < n; ++j) {
    for (uint32_t p = cp[j]; p < cp[j + 1]; ++p) {
      const uint32_t r = ri[p];
      const uint32_t q = fill[r]++;
      ci[q] = j;
      if (r == j) dp[r] = q;
    }
  }
}

int32_t symbolic_levels(uint32_t n, const std::vector<uint32_t>& cp,
                        const std::vector<uint32_t>& ri, const std::vector<uint32_t>& lp,
                        const std::vector<uint32_t>& rp, const std::vector<uint32_t>& ci,
                        const std::vector<uint32_t>& dp, std::vector<int32_t>& lev_ptr,
                        std::vector<int32_t>& lev_idx) {
  // symbolic.cc:106-151: level(i) = 1 + max level over (a) rows k of U(:,i) whose L part is
  // non-empty and (b) columns k of L(i,:).
  std::vector<int32_t> inlevel(n, 0);
  std::vector<int32_t> size(n + 1, 0);
  int32_t num_lev = 0;
  for (uint32_t i = 0; i < n; ++i) {
    int32_t mx = -1;
    for (uint32_t p = cp[i]; p < lp[i]; ++p) {
      const uint32_t k = ri[p];
      if (lp[k] + 1 != cp[k + 1] && inlevel[k] > mx) mx = inlevel[k];
    }
    for (uint32_t q = rp[i]; q < dp[i]; ++q) {
      const uint32_t k = ci[q];
      if (inlevel[k] > mx) mx = inlevel[k];
    }
    inlevel[i] = mx + 1;
    size[mx + 1]++;
    if (mx + 1 > num_lev) num_lev = mx + 1;
  }
  num_lev += (n > 0) ? 1 : 0;
  lev_ptr.assign(num_lev + 1, 0);
  for (int32_t l = 0; l < num_lev; ++l) lev_ptr[l + 1] = lev_ptr[l] + size[l];
  lev_idx.assign(n, 0);
  std::vector<int32_t> t(lev_ptr.begin(), lev_ptr.end());
  for (uint32_t i = 0; i < n; ++i) lev_idx[t[inlevel[i]]++] = (int32_t)i;
  return num_lev;
}

}  // namespace glu

extern "C" {

int glu_symbolic_create(uint32_t n, const uint32_t* ap, const uint32_t* ai, glu_symbolic_t* out) {
  if (!ap || !ai || !out) return glu::set_error(GLU_ARGUMENT_ERROR, "null argument");
  *out = nullptr;
  glu_symbolic_s* s = new (std::nothrow) glu_symbolic_s();
  if (!s) return glu::set_error(GLU_MEMORY_OVERFLOW, "host allocation failed");
  try {
    s->n = n;
    int st = glu::symbolic_fill(n, ap, ai, s->cp, s->ri, s->lp);
    if (st != GLU_OK) {
      delete s;
      return st;
    }
    s->nnz = s->cp[n];
    glu::symbolic_csr(n, s->cp, s->ri, s->rp, s->ci, s->dp);
    s->num_lev = glu::symbolic_levels(n, s->cp, s->ri, s->lp, s->rp, s->ci, s->dp, s->lev_ptr,
                                      s->lev_idx);
  } catch (const std::bad_alloc&) {
    delete s;
    return glu::set_error(GLU_MEMORY_OVERFLOW, "host allocation failed in symbolic analysis");
  }
  *out = s;
  return GLU_OK;
}

int glu_symbolic_sizes(glu_symbolic_t s, uint32_t* nnz, int32_t* num_lev) {
  if (!s) return glu::set_error(GLU_ARGUMENT_ERROR, "null handle");
  if (nnz) *nnz = s->nnz;
  if (num_lev) *num_lev = s->num_lev;
  return GLU_OK;
}

int glu_symbolic_get(glu_symbolic_t s, uint32_t* sym_c_ptr, uint32_t* sym_r_idx,
                     uint32_t* l_col_ptr, uint32_t* csr_r_ptr, uint32_t* csr_c_idx,
                     uint32_t* csr_diag_ptr, int32_t* level_ptr, int32_t* level_idx) {
  if (!s) return glu::set_error(GLU_ARGUMENT_ERROR, "null handle");
  const size_t n = s->n, z = s->nnz;
  if (sym_c_ptr) memcpy(sym_c_ptr, s->cp.data(), 4 * (n + 1));
  if (sym_r_idx) memcpy(sym_r_idx, s->ri.data(), 4 * z);
  if (l_col_ptr) memcpy(l_col_ptr, s->lp.data(), 4 * n);
  if (csr_r_ptr) memcpy(csr_r_ptr, s->rp.data(), 4 * (n + 1));
  if (csr_c_idx) memcpy(csr_c_idx, s->ci.data(), 4 * z);
  if (csr_diag_ptr) memcpy(csr_diag_ptr, s->dp.data(), 4 * n);
  if (level_ptr) memcpy(level_ptr, s->lev_ptr.data(), 4 * (s->num_lev + 1));
  if (level_idx) memcpy(level_idx, s->lev_idx.data(), 4 * n);
  return GLU_OK;
}

int glu_symbolic_positions(glu_symbolic_t s, const uint32_t* ap, const uint32_t* ai,
                           int64_t* pos) {
  if (!s || !ap || !ai || !pos) return glu::set_error(GLU_ARGUMENT_ERROR, "null argument");
  const uint32_t n = s->n;
  std::vector<int64_t> where(n, -1);
  std::vector<int64_t> stamp(n, -1);
  for (uint32_t i = 0; i < n; ++i) {
    for (uint32_t p = s->cp[i]; p < s->cp[i + 1]; ++p) {
      where[s->ri[p]] = p;
      stamp[s->ri[p]] = i;
    }
    for (uint32_t e = ap[i]; e < ap[i + 1]; ++e) {
      const uint32_t r = ai[e];
      if (r < n && stamp[r] == (int64_t)i) {
        pos[e] = where[r];
        stamp[r] = -2 - (int64_t)i;  // later duplicates of (r, i) map to -1
      } else {
        pos[e] = -1;
      }
    }
  }
  return GLU_OK;
}

void glu_symbolic_destroy(glu_symbolic_t s) { delete s; }

}  // extern "C"
