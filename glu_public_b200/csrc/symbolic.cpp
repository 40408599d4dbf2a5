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
#include <cstdio>
#include <cstring>
#include <new>
#include <system_error>
#include <thread>
#include <vector>

#include "glu_b200.h"
#include "internal.h"

struct glu_symbolic_s {
  uint32_t n = 0;
  uint32_t nnz = 0;
  int32_t num_lev = 0;
  uint64_t nnz_a = 0;           // entries of the analysed pattern
  uint64_t pattern = 0;         // digest of the analysed pattern (ap, ai)
  std::vector<uint32_t> cp, ri, lp, rp, ci, dp;
  std::vector<int32_t> lev_ptr, lev_idx;
};

namespace {

// FNV-1a, 64 bit, over a byte range (continuing from h)
uint64_t fnv1a(const void* data, size_t bytes, uint64_t h = 1469598103934665603ull) {
  const unsigned char* p = static_cast<const unsigned char*>(data);
  for (size_t i = 0; i < bytes; ++i) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

uint64_t pattern_digest(uint32_t n, const uint32_t* ap, const uint32_t* ai) {
  uint64_t h = fnv1a(&n, sizeof(n));
  h = fnv1a(ap, sizeof(uint32_t) * ((size_t)n + 1), h);
  return fnv1a(ai, sizeof(uint32_t) * (size_t)ap[n], h);
}

constexpr char kMagic[8] = {'G', 'L', 'U', 'S', 'Y', 'M', 0, 1};   // format version 1

}  // namespace

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
  // a pruned column's (short) adjacency is also copied into padj, so the depth-first searches,
  // which mostly walk pruned columns, read a compact array instead of all of ri
  std::vector<uint32_t> padj;
  std::vector<uint64_t> pbeg(n, 0);
  std::vector<uint32_t> plen(n, 0);
  // rows of the current column's pattern as a bit set (all clear between columns)
  std::vector<uint64_t> bits(((size_t)n + 63) / 64, 0);
  auto seen = [&](uint32_t r) {                // test and set
    uint64_t& w = bits[r >> 6];
    const uint64_t m = 1ull << (r & 63);
    const bool was = (w & m) != 0;
    w |= m;
    return was;
  };
  std::vector<uint32_t> pat;
  std::vector<uint32_t> stack;
  pat.reserve(1024);
  stack.reserve(1024);
  for (uint32_t i = 0; i < n; ++i) {
    pat.clear();
    uint32_t lo = n, hi = 0;                     // row range of the pattern
    for (uint32_t e = ap[i]; e < ap[i + 1]; ++e) {
      const uint32_t r0 = ai[e];
      if (r0 >= n) return set_error(GLU_MATRIX_INVALID, "row index out of range in column %u", i);
      if (seen(r0)) continue;
      pat.push_back(r0);
      lo = std::min(lo, r0);
      hi = std::max(hi, r0);
      if (r0 >= i) continue;
      stack.push_back(r0);
      while (!stack.empty()) {
        const uint32_t k = stack.back();
        stack.pop_back();
        const uint32_t* adj = pruned[k] ? padj.data() + pbeg[k] : ri.data() + lp[k] + 1;
        const uint32_t len = pruned[k] ? plen[k] : prune_end[k] - lp[k] - 1;
        for (uint32_t q = 0; q < len; ++q) {
          const uint32_t r = adj[q];
          if (seen(r)) continue;
          pat.push_back(r);
          lo = std::min(lo, r);
          hi = std::max(hi, r);
          if (r < i) stack.push_back(r);
        }
      }
    }
    // sorted pattern, clearing the bit set: read off the set bits in order when the pattern is
    // not too sparse in its row range (one 64-bit word per 64 rows), sort it otherwise -- the
    // same sorted set either way
    if (!pat.empty()) {
      const uint32_t w0 = lo >> 6, w1 = hi >> 6;
      if ((uint64_t)(w1 - w0) + 1 <= 16ull * pat.size()) {
        size_t k = 0;
        for (uint32_t w = w0; w <= w1; ++w) {
          uint64_t x = bits[w];
          while (x) {
            pat[k++] = (w << 6) + (uint32_t)__builtin_ctzll(x);
            x &= x - 1;
          }
          bits[w] = 0;
        }
      } else {
        std::sort(pat.begin(), pat.end());
        for (uint32_t r : pat) bits[r >> 6] = 0;
      }
    }
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
        pbeg[j] = padj.size();
        plen[j] = (uint32_t)(f - b) + 1;
        padj.insert(padj.end(), b, f + 1);
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
  ci.assign(nnz, 0);
  dp.assign(n, 0);
  // large patterns: threads over column ranges of equal entry counts, each with its own row
  // counts; thread t's entries of row r go after those of threads < t, so every row keeps its
  // columns in increasing order, exactly as the one-thread transpose below
  const unsigned hw = std::thread::hardware_concurrency();
  const int T = nnz >= (1u << 22) ? (int)std::min(16u, std::max(1u, hw)) : 1;
  if (T > 1) {
    std::vector<uint32_t> cb(T + 1, n);
    cb[0] = 0;
    for (int t = 1; t < T; ++t)
      cb[t] = (uint32_t)(std::lower_bound(cp.begin(), cp.end(), (uint64_t)nnz * t / T) -
                         cp.begin());
    for (int t = 1; t <= T; ++t) cb[t] = std::max(cb[t], cb[t - 1]);
    std::vector<std::vector<uint32_t>> cnt(T, std::vector<uint32_t>(n, 0));
    // threads that cannot be started (resource limits) run their share on this thread
    auto run = [&](auto&& body) {
      std::vector<std::thread> th;
      th.reserve(T);
      int t = 0;
      try {
        for (; t < T; ++t) th.emplace_back(body, t);
      } catch (const std::system_error&) {
      }
      for (int u = t; u < T; ++u) body(u);
      for (auto& x : th) x.join();
    };
    run([&](int t) {
      for (uint32_t p = cp[cb[t]]; p < cp[cb[t + 1]]; ++p) cnt[t][ri[p]]++;
    });
    for (uint32_t r = 0; r < n; ++r) {       // row pointers, and each thread's start in each row
      uint32_t at = rp[r];
      for (int t = 0; t < T; ++t) {
        const uint32_t c = cnt[t][r];
        cnt[t][r] = at;
        at += c;
      }
      rp[r + 1] = at;
    }
    run([&](int t) {
      std::vector<uint32_t>& fill = cnt[t];
      for (uint32_t j = cb[t]; j < cb[t + 1]; ++j)
        for (uint32_t p = cp[j]; p < cp[j + 1]; ++p) {
          const uint32_t r = ri[p];
          const uint32_t q = fill[r]++;
          ci[q] = j;
          if (r == j) dp[r] = q;
        }
    });
    return;
  }
  for (uint32_t p = 0; p < nnz; ++p) rp[ri[p] + 1]++;
  for (uint32_t i = 0; i < n; ++i) rp[i + 1] += rp[i];
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
    s->nnz_a = ap[n];
    s->pattern = pattern_digest(n, ap, ai);
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

int glu_symbolic_order(glu_symbolic_t s, uint32_t* n) {
  if (!s || !n) return glu::set_error(GLU_ARGUMENT_ERROR, "null argument");
  *n = s->n;
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

int glu_symbolic_save(glu_symbolic_t s, const char* path) {
  if (!s || !path) return glu::set_error(GLU_ARGUMENT_ERROR, "null argument");
  std::vector<char> buf;
  auto put = [&](const void* p, size_t bytes) {
    const char* c = static_cast<const char*>(p);
    buf.insert(buf.end(), c, c + bytes);
  };
  put(kMagic, sizeof(kMagic));
  const uint32_t hdr[4] = {s->n, s->nnz, (uint32_t)s->num_lev, 0u};
  put(hdr, sizeof(hdr));
  put(&s->nnz_a, 8);
  put(&s->pattern, 8);
  put(s->cp.data(), 4 * s->cp.size());
  put(s->ri.data(), 4 * s->ri.size());
  put(s->lp.data(), 4 * s->lp.size());
  put(s->rp.data(), 4 * s->rp.size());
  put(s->ci.data(), 4 * s->ci.size());
  put(s->dp.data(), 4 * s->dp.size());
  put(s->lev_ptr.data(), 4 * s->lev_ptr.size());
  put(s->lev_idx.data(), 4 * s->lev_idx.size());
  const uint64_t sum = fnv1a(buf.data(), buf.size());
  put(&sum, 8);
  FILE* f = fopen(path, "wb");
  if (!f) return glu::set_error(GLU_FILE_CANNOT_OPEN, "cannot open %s for writing", path);
  const bool ok = fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  if (fclose(f) != 0 || !ok)
    return glu::set_error(GLU_FILE_CANNOT_OPEN, "cannot write %s", path);
  return GLU_OK;
}

int glu_symbolic_load(const char* path, uint32_t n, const uint32_t* ap, const uint32_t* ai,
                      glu_symbolic_t* out) {
  if (!path || !out) return glu::set_error(GLU_ARGUMENT_ERROR, "null argument");
  *out = nullptr;
  FILE* f = fopen(path, "rb");
  if (!f) return glu::set_error(GLU_FILE_CANNOT_OPEN, "cannot open %s", path);
  std::vector<char> buf;
  try {
    char chunk[1 << 16];
    size_t got;
    while ((got = fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
  } catch (const std::bad_alloc&) {
    fclose(f);
    return glu::set_error(GLU_MEMORY_OVERFLOW, "host allocation failed reading %s", path);
  }
  fclose(f);
  const size_t head = sizeof(kMagic) + 16 + 16;
  if (buf.size() < head + 8 || memcmp(buf.data(), kMagic, sizeof(kMagic)) != 0)
    return glu::set_error(GLU_MATRIX_INVALID, "%s is not a symbolic analysis file", path);
  uint32_t hdr[4];
  uint64_t nnz_a, pattern, sum;
  memcpy(hdr, buf.data() + 8, 16);
  memcpy(&nnz_a, buf.data() + 24, 8);
  memcpy(&pattern, buf.data() + 32, 8);
  const uint64_t fn = hdr[0], fz = hdr[1], fl = hdr[2];
  const uint64_t words = (fn + 1) + fz + fn + (fn + 1) + fz + fn + (fl + 1) + fn;
  if (fl > fn || buf.size() != head + 4 * words + 8)
    return glu::set_error(GLU_MATRIX_INVALID, "%s: sizes do not match its length", path);
  memcpy(&sum, buf.data() + buf.size() - 8, 8);
  if (fnv1a(buf.data(), buf.size() - 8) != sum)
    return glu::set_error(GLU_MATRIX_INVALID, "%s: checksum mismatch (damaged file)", path);
  if (ap && ai) {
    if (n != fn || (uint64_t)ap[n] != nnz_a || pattern_digest(n, ap, ai) != pattern)
      return glu::set_error(GLU_MATRIX_INVALID,
                            "%s was made from another pattern (n, entries or their order differ)",
                            path);
  }
  glu_symbolic_s* s = new (std::nothrow) glu_symbolic_s();
  if (!s) return glu::set_error(GLU_MEMORY_OVERFLOW, "host allocation failed");
  try {
    s->n = (uint32_t)fn;
    s->nnz = (uint32_t)fz;
    s->num_lev = (int32_t)fl;
    s->nnz_a = nnz_a;
    s->pattern = pattern;
    const char* p = buf.data() + head;
    auto take_u = [&](std::vector<uint32_t>& v, uint64_t cnt) {
      v.resize(cnt);
      memcpy(v.data(), p, 4 * cnt);
      p += 4 * cnt;
    };
    auto take_i = [&](std::vector<int32_t>& v, uint64_t cnt) {
      v.resize(cnt);
      memcpy(v.data(), p, 4 * cnt);
      p += 4 * cnt;
    };
    take_u(s->cp, fn + 1);
    take_u(s->ri, fz);
    take_u(s->lp, fn);
    take_u(s->rp, fn + 1);
    take_u(s->ci, fz);
    take_u(s->dp, fn);
    take_i(s->lev_ptr, fl + 1);
    take_i(s->lev_idx, fn);
  } catch (const std::bad_alloc&) {
    delete s;
    return glu::set_error(GLU_MEMORY_OVERFLOW, "host allocation failed reading %s", path);
  }
  // index ranges (the plan re-validates the structure in full)
  bool ok = s->cp[0] == 0 && s->cp[fn] == fz && s->rp[0] == 0 && s->rp[fn] == fz &&
            s->lev_ptr[0] == 0 && (uint64_t)s->lev_ptr[fl] == fn;
  for (uint64_t i = 0; ok && i < fn; ++i)
    ok = s->cp[i] <= s->cp[i + 1] && s->rp[i] <= s->rp[i + 1] && s->lp[i] >= s->cp[i] &&
         s->lp[i] < s->cp[i + 1] && s->dp[i] >= s->rp[i] && s->dp[i] < s->rp[i + 1] &&
         s->lev_idx[i] >= 0 && (uint64_t)s->lev_idx[i] < fn;
  for (uint64_t p = 0; ok && p < fz; ++p) ok = s->ri[p] < fn && s->ci[p] < fn;
  for (uint64_t l = 0; ok && l < fl; ++l) ok = s->lev_ptr[l] <= s->lev_ptr[l + 1];
  if (!ok) {
    delete s;
    return glu::set_error(GLU_MATRIX_INVALID, "%s: indices out of range", path);
  }
  *out = s;
  return GLU_OK;
}

}  // extern "C"
