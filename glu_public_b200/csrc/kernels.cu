// Device kernels of the GLU numeric phase for sm_100a (FP64 throughout).
//
// Factorization = sparse phase + dense phase:
//  * sparse phase: one launch per level of the reference's level sets restricted to the
//    columns before the dense trailing block (src/symbolic.cc:106-151 builds those levels).  A
//    warp (narrow levels: a CTA) owns one column c: it divides L(:,c) by the pivot
//    (src/numeric.cu:37-47) and then, for every U(c,j) != 0, subtracts L(:,c)*U(c,j) from
//    column j (src/numeric.cu:51-89).  The target slots come from the precomputed position map
//    instead of the reference's scan of the whole of column j, so each update costs one load of
//    the map entry.  Columns of one level may hit the same target, so updates are FP64 atomics,
//    as in the reference.  Targets inside the dense block are left to dense.cu.
//  * dense phase (dense.cu): right-looking blocked LU without pivoting of the trailing block that
//    fill has made dense, with FP64 DMMA tensor-core trailing updates.
//
// Every kernel takes the instance index from blockIdx.y / blockIdx.z, so one launch covers a
// whole batch of value sets of the same pattern.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "glu_b200.h"
#include "kernels.cuh"
#include "residual.cuh"

namespace glu {

namespace {

constexpr int kWarp = 32;

__device__ __forceinline__ void set_flag(int32_t* status, int b, int32_t f) {
  atomicOr(status + b, f);
}

__device__ __forceinline__ void pivot_flags(int32_t* status, int b, double d, bool perturbed) {
  if (d == 0.0) set_flag(status, b, GLU_INST_ZERO_PIVOT);
  else if (!(fabs(d) <= 1.79769313486231570e308)) set_flag(status, b, GLU_INST_NAN_PIVOT);
  if (perturbed) set_flag(status, b, GLU_INST_PERTURBED);
}

// ---------------------------------------------------------------------------------------------
// value handling
// ---------------------------------------------------------------------------------------------

__global__ void k_pad_identity(PlanDev P, double* vals, int first) {
  double* D = vals + (int64_t)(first + blockIdx.y) * P.blob + P.dbase;
  for (uint32_t i = P.nt + blockIdx.x * blockDim.x + threadIdx.x; i < P.ntp;
       i += gridDim.x * blockDim.x)
    D[(int64_t)i * P.ntp + i] = 1.0;
}

__global__ void k_zero_slots(PlanDev P, double* vals, int first) {
  double* V = vals + (int64_t)(first + blockIdx.y) * P.blob;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < P.nasm_zero;
       e += (int64_t)gridDim.x * blockDim.x)
    V[P.asm_zero[e]] = 0.0;
}

__global__ void k_ingest(PlanDev P, double* vals, int first, const double* __restrict__ a) {
  const int b = blockIdx.y;
  double* V = vals + (int64_t)(first + b) * P.blob;
  const double* ab = a + (int64_t)b * P.nnz_a;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < P.nnz_a;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = P.ing_slot[e];
    if (s >= 0) V[s] = P.ing_scale ? ab[e] * P.ing_scale[e] : ab[e];
  }
}

__global__ void k_load_lu(PlanDev P, double* vals, int first, const double* __restrict__ val) {
  const int b = blockIdx.y;
  double* V = vals + (int64_t)(first + b) * P.blob;
  const double* vb = val + (int64_t)b * P.nnz;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P.nnz;
       p += (int64_t)gridDim.x * blockDim.x)
    V[P.pos2slot[p]] = vb[p];
}

__global__ void k_export_lu(PlanDev P, const double* vals, int inst, double* __restrict__ val) {
  const double* V = vals + (int64_t)inst * P.blob;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P.nnz;
       p += (int64_t)gridDim.x * blockDim.x)
    val[p] = V[P.pos2slot[p]];
}

// 1-norm of every instance (max column abs sum over the filled pattern, src/numeric.cu:405-417),
// accumulated as the bit pattern of a non-negative double so atomicMax orders it correctly.
__global__ void k_norm1(PlanDev P, const double* vals, unsigned long long* norm_bits) {
  const int b = blockIdx.y;
  const double* V = vals + (int64_t)b * P.blob;
  const int lane = threadIdx.x % kWarp;
  const int warps = blockDim.x / kWarp;
  for (uint32_t j = blockIdx.x * warps + threadIdx.x / kWarp; j < P.n; j += gridDim.x * warps) {
    double s = 0.0;
    for (uint32_t p = P.cp[j] + lane; p < P.cp[j + 1]; p += kWarp) s += fabs(V[P.pos2slot[p]]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) atomicMax(norm_bits + b, (unsigned long long)__double_as_longlong(s));
  }
}

__global__ void k_pert_finish(int count, const unsigned long long* norm_bits, double* pert) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < count) pert[b] = 3.45e-4 * __longlong_as_double((long long)norm_bits[b]);
}

__global__ void k_fill(int count, double v, double* out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < count) out[b] = v;
}

// ---------------------------------------------------------------------------------------------
// sparse phase: one level
// ---------------------------------------------------------------------------------------------

// The threads that share one column: `gsize` threads (whole warps) of which this is thread
// `gtid` in warp `wig` of `nwg`; `bar` says how they synchronise: 0 one warp (__syncwarp), -1 the
// whole CTA (__syncthreads), k > 0 the named barrier k (several warps of a larger CTA).
// `ilane` / `istride`: the lane and lane count that walk one pair's L rows (the whole warp, or the
// group's own lanes when a group is a fraction of a warp); `mask`: those lanes when bar == 0.
struct ColGroup {
  int gtid, gsize, wig, nwg, bar, ilane, istride;
  unsigned mask;
};

__device__ __forceinline__ void group_sync(const ColGroup& g) {
  if (g.bar == 0) __syncwarp(g.mask);
  else if (g.bar < 0) __syncthreads();
  else asm volatile("bar.sync %0, %1;" ::"r"(g.bar), "r"(g.gsize) : "memory");
}

__device__ __forceinline__ ColGroup warp_group() {
  const int lane = threadIdx.x % kWarp;
  return ColGroup{lane, kWarp, 0, 1, 0, lane, kWarp, 0xffffffffu};
}

__device__ __forceinline__ ColGroup cta_group() {
  return ColGroup{(int)threadIdx.x, (int)blockDim.x, (int)(threadIdx.x / kWarp),
                  (int)(blockDim.x / kWarp), -1, (int)(threadIdx.x % kWarp), kWarp, 0xffffffffu};
}

// One column c of a sparse level for instance b, by the threads of group g (their warps split the
// U(c,:) pairs): pivot (perturbed if |d| < pert and the column has an L part,
// src/numeric.cu:139-140), L(:,c) /= d (src/numeric.cu:37-47), then for every U(c,j) != 0 the
// targets of column j take -L(:,c) * U(c,j) through the position map (src/numeric.cu:51-89).
// Columns of one level may hit the same target, hence the FP64 atomics (as in the reference).
// SCALE_ONLY: pivot and scaling only (the updates are applied by sparse_split_part or, in the
// deterministic mode, by k_sparse_pull).
// Ls (optional, |L(:,c)| doubles of shared memory, whole-CTA groups only): the scaled L(:,c) is
// also kept there and the updates read it from there instead of from global memory.
template <bool SCALE_ONLY>
__device__ __forceinline__ void sparse_column(const PlanDev& P, double* __restrict__ V, double pv,
                                              int32_t* status, int b, uint32_t c,
                                              const ColGroup& g, double* Ls = nullptr) {
  const uint32_t dslot = P.lp[c];
  const uint32_t l0 = dslot + 1;
  const uint32_t nL = P.cp[c + 1] - l0;
  const double d0 = V[dslot];
  double d = d0;
  const bool perturbed = pv > 0.0 && nL > 0 && fabs(d0) < pv;   // numeric.cu:139-140
  if (perturbed) d = pv;
  group_sync(g);
  if (g.gtid == 0) {
    if (perturbed) V[dslot] = d;
    pivot_flags(status, b, d, perturbed);
  }
  for (uint32_t k = g.gtid; k < nL; k += g.gsize) {
    const double l = V[l0 + k] / d;
    V[l0 + k] = l;
    if (Ls) Ls[k] = l;
  }
  group_sync(g);

  if (SCALE_ONLY) return;
  const double* __restrict__ Lc = Ls ? Ls : V + l0;
  const int64_t q1 = P.pair_ptr[c + 1];
  const uint32_t nsplit = P.lsplit[c];
  for (int64_t q = P.pair_ptr[c] + g.wig; q < q1; q += g.nwg) {
    const uint32_t j = (uint32_t)P.pair_j[q];
    const double u = V[P.pair_uslot[q]];
    const int32_t* __restrict__ tm = P.tmap + P.pair_moff[q];
    // rows >= t of a tail column j belong to the dense block: they are applied afterwards by
    // the hub GEMM and the per-column pull, so only sparse targets are touched here
    const uint32_t nsp = j < P.t ? nL : nsplit;
    for (uint32_t k = g.ilane; k < nsp; k += g.istride) atomicAdd(V + tm[k], -(Lc[k] * u));
  }
}

// Part `part` of `splits` of column c's pairs (c, j), by the whole CTA: L(:,c) = A(:,c) / d is
// formed in shared memory (Ls, |L(:,c)| doubles; the pivot perturbed as in sparse_column) and
// the part's pairs are applied from there; the column itself is scaled afterwards by
// sparse_column<true>, so no CTA writes what another reads.  Each update is the same L * u
// product as in sparse_column, from the same rounded L.
__device__ __forceinline__ void sparse_split_part(const PlanDev& P, double* __restrict__ V,
                                                  double pv, uint32_t c, int part, int splits,
                                                  double* Ls) {
  const int lane = threadIdx.x % kWarp, wig = threadIdx.x / kWarp, nwg = blockDim.x / kWarp;
  const uint32_t dslot = P.lp[c];
  const uint32_t l0 = dslot + 1;
  const uint32_t nL = P.cp[c + 1] - l0;
  const double d0 = V[dslot];
  const double d = (pv > 0.0 && nL > 0 && fabs(d0) < pv) ? pv : d0;   // numeric.cu:139-140
  __syncthreads();                             // Ls may still be read by the previous item
  for (uint32_t k = threadIdx.x; k < nL; k += blockDim.x) Ls[k] = V[l0 + k] / d;
  __syncthreads();
  const int64_t q1 = P.pair_ptr[c + 1];
  const uint32_t nsplit = P.lsplit[c];
  for (int64_t q = P.pair_ptr[c] + part * nwg + wig; q < q1; q += (int64_t)splits * nwg) {
    const uint32_t j = (uint32_t)P.pair_j[q];
    const double u = V[P.pair_uslot[q]];
    const int32_t* __restrict__ tm = P.tmap + P.pair_moff[q];
    const uint32_t nsp = j < P.t ? nL : nsplit;
    for (uint32_t k = lane; k < nsp; k += kWarp) atomicAdd(V + tm[k], -(Ls[k] * u));
  }
}

// One launch per sparse level: groups of `wpc` warps share a column (wpc = 1: a warp per
// column; wpc = blockDim/32: the whole CTA), or, with wpc = 1 and lanes < 32, groups of `lanes`
// lanes of a warp (8 or 16: columns whose L parts are that short leave most of a warp idle);
// each group takes `cpw` consecutive columns of the level in turn.  Grid
// (ceil(ncols / (groups per CTA * cpw)), count).  stage: whole-CTA groups keep the scaled L(:,c)
// in dynamic shared memory (the launch sizes it for the level's longest L part) and every warp's
// updates read it from there.
__global__ void __launch_bounds__(256) k_sparse_level(PlanDev P, double* vals,
                                                      const double* __restrict__ pert,
                                                      int32_t* status, int begin, int ncols,
                                                      int wpc, int cpw, int stage, int lanes) {
  extern __shared__ double Lsm[];
  const int b = blockIdx.y;
  const int gsz = wpc == 1 ? lanes : kWarp * wpc;
  const int groups = blockDim.x / gsz;
  const int gi = threadIdx.x / gsz;
  const int gtid = (int)(threadIdx.x % gsz);
  const unsigned sub = gsz >= kWarp ? 0xffffffffu
                                    : (((1u << gsz) - 1u) << ((threadIdx.x % kWarp) / gsz * gsz));
  const ColGroup g{gtid, gsz, wpc == 1 ? 0 : (int)((threadIdx.x / kWarp) % wpc), wpc,
                   wpc == 1 ? 0 : (groups == 1 ? -1 : 1 + gi),
                   gsz >= kWarp ? (int)(threadIdx.x % kWarp) : gtid, gsz >= kWarp ? kWarp : gsz,
                   sub};
  double* V = vals + (int64_t)b * P.blob;
  const int first = (blockIdx.x * groups + gi) * cpw;
  for (int k = 0; k < cpw; ++k) {
    const int col = first + k;
    if (col >= ncols) break;                   // the same for every thread of the group
    sparse_column<false>(P, V, pert[b], status, b, (uint32_t)P.scols[begin + col], g,
                         stage ? Lsm : nullptr);
  }
}

// Pivot and scaling of a level's columns (a CTA per column): after k_sparse_split, and in the
// deterministic mode before k_sparse_pull.
__global__ void __launch_bounds__(256) k_sparse_scale(PlanDev P, double* vals,
                                                      const double* __restrict__ pert,
                                                      int32_t* status, int begin) {
  const int b = blockIdx.y;
  sparse_column<true>(P, vals + (int64_t)b * P.blob, pert[b], status, b,
                      (uint32_t)P.scols[begin + blockIdx.x], cta_group());
}

// A narrow level's columns with their updates split over `splits` CTAs each (grid
// (ncols * splits, count)); k_sparse_scale scales the columns afterwards.
__global__ void __launch_bounds__(256) k_sparse_split(PlanDev P, double* vals,
                                                      const double* __restrict__ pert, int begin,
                                                      int splits) {
  extern __shared__ double Ls[];
  const int b = blockIdx.y;
  const int col = blockIdx.x / splits, part = blockIdx.x % splits;
  sparse_split_part(P, vals + (int64_t)b * P.blob, pert[b], (uint32_t)P.scols[begin + col], part,
                    splits, Ls);
}

// Deterministic level, after k_sparse_scale: one warp per target column j of the level applies
// the level's pairs (c, j) in the level's column order, -L(:,c) * U(c,j) into column j's slots,
// without atomics: the rows of one L(:,c) are distinct, the pairs of one target follow each
// other, and no two warps share a target column.  Same products and sums as sparse_column, in a
// fixed order.  Grid (ceil(targets / 8), count), targets [t0, t0 + ntargets) of det_tptr.
__global__ void __launch_bounds__(256) k_sparse_pull(PlanDev P, double* vals, int64_t t0,
                                                     int64_t ntargets) {
  const int64_t w = (int64_t)blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp;
  if (w >= ntargets) return;
  const int lane = threadIdx.x % kWarp;
  double* __restrict__ V = vals + (int64_t)blockIdx.y * P.blob;
  const int64_t e1 = P.det_tptr[t0 + w + 1];
  for (int64_t e = P.det_tptr[t0 + w]; e < e1; ++e) {
    const int64_t q = P.det_q[e];
    const uint32_t c = (uint32_t)P.det_c[e];
    const uint32_t j = (uint32_t)P.pair_j[q];
    const uint32_t l0 = P.lp[c] + 1;
    const uint32_t nL = P.cp[c + 1] - l0;
    const double u = V[P.pair_uslot[q]];
    const int32_t* __restrict__ tm = P.tmap + P.pair_moff[q];
    const uint32_t nsp = j < P.t ? nL : P.lsplit[c];
    for (uint32_t k = lane; k < nsp; k += kWarp) V[tm[k]] += -(V[l0 + k] * u);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------------------------
// sparse phase: a run of consecutive levels in ONE cooperative launch
// ---------------------------------------------------------------------------------------------

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Barrier among the CTAs of one group: every CTA adds one arrival to the group's counter and
// waits until it reaches `target`.  The wait is bounded: after `budget_ns` of waiting, or as soon
// as another CTA has reported a failure in *err, it gives up, records the failure in *err and
// returns false.  All threads of the CTA must call it.
__device__ bool group_barrier(unsigned* ctr, int* err, unsigned target,
                              unsigned long long budget_ns) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();                           // this CTA's writes before its arrival
    atomicAdd(ctr, 1u);
    const unsigned long long t0 = global_ns();
    while (ld_acquire_u32(ctr) < target) {
      if (*(volatile int*)err) {
        ok = 0;
        break;
      }
      if (global_ns() - t0 > budget_ns) {
        atomicExch(err, 1);
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// A run of consecutive sparse levels (no fronts among them) for every instance, in one
// cooperative launch: the grid is split into `count` groups of gridDim.x / count CTAs (or, with
// more instances than CTAs, every CTA is a group of one and walks its instances b, b + gridDim.x,
// ... one after another).  A group walks the levels of its instance in order; per level its CTAs
// share the level's columns in the mode the plan chose (desc[l] = {begin, ncols, mode, splits}:
// mode 0 a warp per column, 1 a CTA per column, 3 the column's pairs split over `splits` CTA
// items, then scaled by a CTA each after the level's barrier), with the same per-column code as
// the per-level kernels.  Between levels the group's CTAs meet at a device-side barrier (a
// group of one CTA needs only __syncthreads); instances never depend on each other, so no
// barrier spans groups.  Every wait is bounded (group_barrier): on expiry the CTA marks its
// instances GLU_INST_TIMEOUT, *err becomes non-zero, and every CTA returns.  `extra` arrivals are
// added to every barrier target (0 in use; a test sets 1 to make the first barrier unreachable).
__global__ void __launch_bounds__(256) k_sparse_persistent(PlanDev P, double* vals,
                                                           const double* __restrict__ pert,
                                                           int32_t* status,
                                                           const int4* __restrict__ desc,
                                                           int nlev, int count, unsigned* bar,
                                                           int* err, unsigned long long budget_ns,
                                                           int extra) {
  extern __shared__ double Ls[];
  __shared__ int s_abort;
  const int G = count < (int)gridDim.x ? count : (int)gridDim.x;
  const int cpg = gridDim.x / G;               // CTAs per group
  const int g = blockIdx.x / cpg;
  if (g >= G) return;                          // CTAs beyond G * cpg have no group
  const int r = blockIdx.x % cpg;
  const int warp = threadIdx.x / kWarp, nw = blockDim.x / kWarp;
  unsigned epoch = 0;
  for (int b = g; b < count; b += G) {
    double* V = vals + (int64_t)b * P.blob;
    const double pv = pert[b];
    int4 pending = make_int4(0, 0, -1, 0);     // a split level whose columns still need scaling
    for (int l = 0; l < nlev; ++l) {
      if (threadIdx.x == 0) s_abort = *(volatile int*)err;   // another group gave up
      __syncthreads();
      if (s_abort) {
        if (threadIdx.x == 0 && r == 0)
          for (int bb = b; bb < count; bb += G) atomicOr(status + bb, GLU_INST_TIMEOUT);
        return;
      }
      if (pending.z == 3) {                    // scale the previous split level's columns: no
        for (int col = r; col < pending.y; col += cpg)   // later level reads or writes them
          sparse_column<true>(P, V, pv, status, b, (uint32_t)P.scols[pending.x + col],
                              cta_group());
        pending.z = -1;
      }
      const int4 d = desc[l];
      if (d.z == 0) {
        for (int col = r * nw + warp; col < d.y; col += cpg * nw)
          sparse_column<false>(P, V, pv, status, b, (uint32_t)P.scols[d.x + col], warp_group());
      } else if (d.z == 1) {
        for (int col = r; col < d.y; col += cpg)
          sparse_column<false>(P, V, pv, status, b, (uint32_t)P.scols[d.x + col], cta_group());
      } else {
        for (int it = r; it < d.y * d.w; it += cpg)
          sparse_split_part(P, V, pv, (uint32_t)P.scols[d.x + it / d.w], it % d.w, d.w, Ls);
        pending = d;
      }
      if (cpg > 1) {
        ++epoch;
        if (!group_barrier(bar + g, err, epoch * (unsigned)cpg + (unsigned)extra, budget_ns)) {
          if (threadIdx.x == 0)
            for (int bb = b; bb < count; bb += G) atomicOr(status + bb, GLU_INST_TIMEOUT);
          return;
        }
      } else {
        __syncthreads();
        if (extra > 0) {                       // a group of one CTA has no barrier to miss: the
          if (threadIdx.x == 0) {              // unreachable-target test times out here instead
            const unsigned long long t0 = global_ns();
            while (global_ns() - t0 <= budget_ns && !*(volatile int*)err) __nanosleep(1000);
            atomicExch(err, 1);
            for (int bb = b; bb < count; bb += G) atomicOr(status + bb, GLU_INST_TIMEOUT);
          }
          return;
        }
      }
    }
    if (pending.z == 3) {
      for (int col = r; col < pending.y; col += cpg)
        sparse_column<true>(P, V, pv, status, b, (uint32_t)P.scols[pending.x + col], cta_group());
    }
    if (cpg == 1) __syncthreads();             // Ls and V reuse by the next instance
  }
}

// ---------------------------------------------------------------------------------------------
// solves
// ---------------------------------------------------------------------------------------------

__global__ void k_permute_in(PlanDev P, int nrhs, const double* __restrict__ Bm, double* y,
                             int64_t ylen, int transpose) {
  const int64_t v = blockIdx.y;                 // instance * nrhs + rhs
  const double* bv = Bm + v * P.n;
  double* yv = y + v * ylen;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < ylen;
       k += (int64_t)gridDim.x * blockDim.x) {
    double out = 0.0;
    if (k < P.n) {
      if (!transpose) {          // symbolic.cc:211-219 with pivot = identity
        const uint32_t src = P.col_perm[k];
        out = P.col_scale_perm ? bv[src] * P.col_scale_perm[k] : bv[src];
      } else {                   // g'[i] = row_scale[row_perm[i]] * g[row_perm[i]]
        const uint32_t src = P.row_perm[k];
        out = P.row_scale ? P.row_scale[src] * bv[src] : bv[src];
      }
    }
    yv[k] = out;
  }
}

__global__ void k_permute_out(PlanDev P, int nrhs, const double* __restrict__ y, double* X,
                              int64_t ylen, int transpose) {
  const int64_t v = blockIdx.y;
  const double* yv = y + v * ylen;
  double* xv = X + v * P.n;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < P.n;
       k += (int64_t)gridDim.x * blockDim.x) {
    if (!transpose) {            // symbolic.cc:238-245
      const double b = yv[P.row_perm_inv[k]];
      xv[k] = P.row_scale ? b * P.row_scale[k] : b;
    } else {                     // lambda[col_perm[k]] = col_scale_perm[k] * w[k]
      xv[P.col_perm[k]] = P.col_scale_perm ? P.col_scale_perm[k] * yv[k] : yv[k];
    }
  }
}

// Right-hand sides one warp handles together in the push-form sparse solves: the column's
// indices and values are loaded once for all of them.
constexpr int kSolveVecs = 4;

// L solve, column oriented with unit diagonal (symbolic.cc:221-226), one warp per column and
// group of up to kSolveVecs right-hand sides of one instance (grid.y = instance * groups + group).
__global__ void k_sparse_lsolve(PlanDev P, const double* vals, int nrhs, double* y, int64_t ylen,
                                const int32_t* __restrict__ cols, int begin, int ncols) {
  const int w = blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp;
  if (w >= ncols) return;
  const int lane = threadIdx.x % kWarp;
  const int groups = (nrhs + kSolveVecs - 1) / kSolveVecs;
  const int64_t inst = blockIdx.y / groups;
  const int k0 = (blockIdx.y % groups) * kSolveVecs;
  const int nk = min(kSolveVecs, nrhs - k0);
  const double* V = vals + inst * P.blob;
  double* y0 = y + (inst * nrhs + k0) * ylen;
  const uint32_t c = (uint32_t)cols[begin + w];
  double yc[kSolveVecs];
#pragma unroll
  for (int k = 0; k < kSolveVecs; ++k) yc[k] = k < nk ? y0[k * ylen + c] : 0.0;
  for (uint32_t p = P.lp[c] + 1 + lane; p < P.cp[c + 1]; p += kWarp) {
    const uint32_t r = P.ri[p];
    const double l = V[p];
#pragma unroll
    for (int k = 0; k < kSolveVecs; ++k)
      if (k < nk) atomicAdd(y0 + k * ylen + r, -(l * yc[k]));
  }
}

// U solve (symbolic.cc:228-236), one warp per column and group of right-hand sides.
__global__ void k_sparse_usolve(PlanDev P, const double* vals, int nrhs, double* y, int64_t ylen,
                                const int32_t* __restrict__ cols, int begin, int ncols) {
  const int w = blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp;
  if (w >= ncols) return;
  const int lane = threadIdx.x % kWarp;
  const int groups = (nrhs + kSolveVecs - 1) / kSolveVecs;
  const int64_t inst = blockIdx.y / groups;
  const int k0 = (blockIdx.y % groups) * kSolveVecs;
  const int nk = min(kSolveVecs, nrhs - k0);
  const double* V = vals + inst * P.blob;
  double* y0 = y + (inst * nrhs + k0) * ylen;
  const uint32_t c = (uint32_t)cols[begin + w];
  const double d = V[P.lp[c]];
  double xc[kSolveVecs];
#pragma unroll
  for (int k = 0; k < kSolveVecs; ++k) xc[k] = k < nk ? y0[k * ylen + c] / d : 0.0;
  __syncwarp();
  if (lane < nk) {                             // lane k stores x_c of right-hand side k
    double xv = xc[0];
#pragma unroll
    for (int k = 1; k < kSolveVecs; ++k)
      if (lane == k) xv = xc[k];
    y0[lane * ylen + c] = xv;
  }
  for (uint32_t p = P.cp[c] + lane; p < P.lp[c]; p += kWarp) {
    const uint32_t r = P.ri[p];
    const double u = V[p];
#pragma unroll
    for (int k = 0; k < kSolveVecs; ++k)
      if (k < nk) atomicAdd(y0 + k * ylen + r, -(u * xc[k]));
  }
}

// U^T solve (row j of U^T = column j of U), pull form, one warp per column.
__global__ void k_sparse_utsolve(PlanDev P, const double* vals, int nrhs, double* y, int64_t ylen,
                                 const int32_t* __restrict__ cols, int begin, int ncols) {
  const int w = blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp;
  if (w >= ncols) return;
  const int lane = threadIdx.x % kWarp;
  const int64_t v = blockIdx.y;
  const double* V = vals + (v / nrhs) * P.blob;
  double* yv = y + v * ylen;
  const uint32_t j = (uint32_t)cols[begin + w];
  double s = 0.0;
  for (uint32_t p = P.cp[j] + lane; p < P.lp[j]; p += kWarp) s += V[p] * yv[P.ri[p]];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) yv[j] = (yv[j] - s) / V[P.lp[j]];
}

// L^T solve (row j of L^T = column j of L), pull form, unit diagonal.
__global__ void k_sparse_ltsolve(PlanDev P, const double* vals, int nrhs, double* y, int64_t ylen,
                                 const int32_t* __restrict__ cols, int begin, int ncols) {
  const int w = blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp;
  if (w >= ncols) return;
  const int lane = threadIdx.x % kWarp;
  const int64_t v = blockIdx.y;
  const double* V = vals + (v / nrhs) * P.blob;
  double* yv = y + v * ylen;
  const uint32_t j = (uint32_t)cols[begin + w];
  double s = 0.0;
  for (uint32_t p = P.lp[j] + 1 + lane; p < P.cp[j + 1]; p += kWarp) s += V[p] * yv[P.ri[p]];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) yv[j] = yv[j] - s;
}

// A front in a triangular solve: one CTA per (front, vector) walks the front's columns in
// order, so the chain of pivots inside the front costs barriers instead of launches.
// which: 0 = L push (forward), 1 = U push (backward), 2 = U^T pull (forward), 3 = L^T pull
// (backward) -- the column forms of the single-column kernels above.
__global__ void __launch_bounds__(256) k_front_solve(PlanDev P, const double* vals, int nrhs,
                                                     double* y, int64_t ylen,
                                                     const int32_t* __restrict__ fids, int which) {
  __shared__ double red[8];
  __shared__ double bcast;
  const int f = fids[blockIdx.x];
  const int64_t v = blockIdx.y;
  const double* V = vals + (v / nrhs) * P.blob;
  double* yv = y + v * ylen;
  const int s0 = P.fs0[f], w = P.fw[f];
  const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp;
  for (int step = 0; step < w; ++step) {
    const bool fwd = (which == 0 || which == 2);
    const uint32_t x = (uint32_t)(fwd ? s0 + step : s0 + w - 1 - step);
    if (which == 0) {
      __syncthreads();
      const double yx = yv[x];
      for (uint32_t p = P.lp[x] + 1 + tid; p < P.cp[x + 1]; p += blockDim.x)
        atomicAdd(yv + P.ri[p], -(V[p] * yx));
    } else if (which == 1) {
      __syncthreads();
      const double xx = yv[x] / V[P.lp[x]];
      __syncthreads();
      if (tid == 0) yv[x] = xx;
      for (uint32_t p = P.cp[x] + tid; p < P.lp[x]; p += blockDim.x)
        atomicAdd(yv + P.ri[p], -(V[p] * xx));
    } else {
      double sum = 0.0;
      const uint32_t p0 = which == 2 ? P.cp[x] : P.lp[x] + 1;
      const uint32_t p1 = which == 2 ? P.lp[x] : P.cp[x + 1];
      for (uint32_t p = p0 + tid; p < p1; p += blockDim.x) sum += V[p] * yv[P.ri[p]];
      for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
      if (lane == 0) red[warp] = sum;
      __syncthreads();
      if (tid == 0) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x / kWarp); ++q) t += red[q];
        yv[x] = which == 2 ? (yv[x] - t) / V[P.lp[x]] : yv[x] - t;
      }
      __syncthreads();
    }
  }
}

// k_front_solve for the push forms (which 0: L forward, 1: U backward) with the front's own
// unknowns in shared memory: a step reads the pivot value from shared memory instead of global
// memory, applies updates to the front's rows there (the rows of one column are distinct, so no
// atomics) and pushes the rest to global memory with atomics, off the step-to-step chain; each
// thread's first PF entries of a column (and the pivot) are loaded one step ahead, so the chain
// from column to column is a barrier and a few shared-memory operations.  Same products and
// quotients as k_front_solve.
__global__ void __launch_bounds__(256) k_front_solve_push(PlanDev P, const double* vals, int nrhs,
                                                          double* y, int64_t ylen,
                                                          const int32_t* __restrict__ fids,
                                                          int which) {
  extern __shared__ double fsm[];
  const int f = fids[blockIdx.x];
  const int64_t v = blockIdx.y;
  const double* __restrict__ V = vals + (v / nrhs) * P.blob;
  double* yv = y + v * ylen;
  const int s0 = P.fs0[f], w = P.fw[f];
  double* ys = fsm;                                          // running values of the front's rows
  double* xs = fsm + P.fw_max;                               // U: the solved values
  uint32_t* pb = reinterpret_cast<uint32_t*>(fsm + 2 * P.fw_max);   // entry range per column
  uint32_t* pe = pb + P.fw_max;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int x = tid; x < w; x += nt) {
    const uint32_t c = (uint32_t)(s0 + x);
    ys[x] = yv[c];
    pb[x] = which == 0 ? P.lp[c] + 1 : P.cp[c];
    pe[x] = which == 0 ? P.cp[c + 1] : P.lp[c];
  }
  __syncthreads();
  constexpr int PF = 4;
  uint32_t rn[PF];
  double vn[PF], dn = 1.0;
  auto prefetch = [&](int step) {                            // entries of the step's column
    const int x = which == 0 ? step : w - 1 - step;
    const uint32_t b0 = pb[x], e0 = pe[x];
#pragma unroll
    for (int k = 0; k < PF; ++k) {
      const uint32_t p = b0 + tid + k * nt;
      rn[k] = p < e0 ? P.ri[p] : 0xffffffffu;
      vn[k] = p < e0 ? V[p] : 0.0;
    }
    dn = which == 1 ? V[e0] : 1.0;                           // U(x, x) sits at lp[c] = pe[x]
  };
  prefetch(0);
  for (int step = 0; step < w; ++step) {
    const int x = which == 0 ? step : w - 1 - step;
    uint32_t r[PF];
    double m[PF];
#pragma unroll
    for (int k = 0; k < PF; ++k) {
      r[k] = rn[k];
      m[k] = vn[k];
    }
    const double d = dn;
    if (step + 1 < w) prefetch(step + 1);
    __syncthreads();                                         // the previous step's updates
    double xv = ys[x];
    if (which == 1) {
      xv = xv / d;
      if (tid == 0) xs[x] = xv;
    }
    auto apply = [&](uint32_t rr, double mm) {
      if (rr >= (uint32_t)s0 && rr < (uint32_t)(s0 + w)) ys[rr - s0] -= mm * xv;
      else atomicAdd(yv + rr, -(mm * xv));
    };
#pragma unroll
    for (int k = 0; k < PF; ++k)
      if (r[k] != 0xffffffffu) apply(r[k], m[k]);
    const uint32_t e0 = pe[x];
    for (uint32_t p = pb[x] + tid + PF * nt; p < e0; p += nt) apply(P.ri[p], V[p]);
  }
  __syncthreads();
  for (int x = tid; x < w; x += nt) yv[s0 + x] = which == 0 ? ys[x] : xs[x];
}

// Row-wise (pull) forward solves of the deterministic mode, one warp per row; each sum is
// formed lane by lane over the row's entries and reduced by shuffles, in a fixed order.
// which 0 (L, unit diagonal): y_r -= sum L(r, c) y_c over the row's entries with c < min(r, t);
// which 1 (U): y_c = (y_c - sum_{j > c} U(c, j) y_j) / U(c, c), the border columns j >= t
// included.  rows: a level's rows rows[begin .. begin + nrows), or nullptr for rows
// begin .. begin + nrows - 1.
__global__ void __launch_bounds__(256) k_rows_solve(PlanDev P, const double* vals, int nrhs,
                                                    double* y, int64_t ylen,
                                                    const int32_t* __restrict__ rows, int begin,
                                                    int nrows, int which) {
  const int w = blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp;
  if (w >= nrows) return;
  const int lane = threadIdx.x % kWarp;
  const int64_t v = blockIdx.y;
  const double* __restrict__ V = vals + (v / nrhs) * P.blob;
  double* yv = y + v * ylen;
  const uint32_t r = rows ? (uint32_t)rows[begin + w] : (uint32_t)(begin + w);
  double s = 0.0;
  if (which == 0) {
    for (uint32_t q = P.rp[r] + lane; q < P.dp[r]; q += kWarp) {
      const uint32_t c = P.ci[q];
      if (c < P.t) s += V[P.csr_slot[q]] * yv[c];
    }
  } else {
    for (uint32_t q = P.dp[r] + 1 + lane; q < P.rp[r + 1]; q += kWarp)
      s += V[P.csr_slot[q]] * yv[P.ci[q]];
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) yv[r] = which == 0 ? yv[r] - s : (yv[r] - s) / V[P.lp[r]];
}

// Border U(r < t, j >= t): push x_j into rows r (solve) or pull w_r into w_j (transpose).
__global__ void k_border(PlanDev P, const double* vals, int nrhs, double* y, int64_t ylen,
                         int transpose) {
  const int jt = blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp;
  if (jt >= (int)P.nt) return;
  const int lane = threadIdx.x % kWarp;
  const int64_t v = blockIdx.y;
  const double* V = vals + (v / nrhs) * P.blob;
  double* yv = y + v * ylen;
  const int64_t e0 = P.bord_ptr[jt], e1 = P.bord_ptr[jt + 1];
  if (!transpose) {
    const double xj = yv[P.t + jt];
    for (int64_t e = e0 + lane; e < e1; e += kWarp)
      atomicAdd(yv + P.bord_row[e], -(V[P.bord_slot[e]] * xj));
  } else {
    double s = 0.0;
    for (int64_t e = e0 + lane; e < e1; e += kWarp) s += V[P.bord_slot[e]] * yv[P.bord_row[e]];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) yv[P.t + jt] -= s;
  }
}

// The forward solve's border y_r -= U(r, j) x_j (r < t <= j) in chunks of at most 1024 entries
// of one tail column, a warp per chunk (grid (ceil(chunks / 8), vectors)), so the long border
// columns of a mesh's top separator are shared by many warps.
__global__ void k_border_chunks(PlanDev P, const double* vals, int nrhs, double* y, int64_t ylen) {
  const int64_t k = (int64_t)blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp;
  if (k >= P.nbordck) return;
  const int lane = threadIdx.x % kWarp;
  const int jt = P.bord_ckcol[k];
  const int64_t v = blockIdx.y;
  const double* V = vals + (v / nrhs) * P.blob;
  double* yv = y + v * ylen;
  const int64_t e0 = P.bord_ck0[k], e1 = min(e0 + 1024, P.bord_ptr[jt + 1]);
  const double xj = yv[P.t + jt];
  for (int64_t e = e0 + lane; e < e1; e += kWarp)
    atomicAdd(yv + P.bord_row[e], -(V[P.bord_slot[e]] * xj));
}

// Copies the 64 x 64 diagonal block at (kb, kb) of a column-major matrix into shared memory
// (Ds[i + 64 j]) with 16-byte asynchronous copies, all in flight at once; the caller waits with
// cp.async.wait_group and a barrier.  kb, ld and the instance offsets are even, so every copied
// row pair is 16-byte aligned.
__device__ __forceinline__ void stage_diag_block(const double* __restrict__ D, int64_t ld, int kb,
                                                 double* Ds, int tid, int nthreads) {
  for (int idx = tid; idx < 64 * 32; idx += nthreads) {
    const int i = (idx % 32) * 2, j = idx / 32;
    const unsigned dst = (unsigned)__cvta_generic_to_shared(Ds + i + j * 64);
    const double* src = D + (int64_t)(kb + i) + (int64_t)(kb + j) * ld;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src));
  }
  asm volatile("cp.async.commit_group;\n" ::);
}
__device__ __forceinline__ void stage_wait() { asm volatile("cp.async.wait_group 0;\n" ::); }

// The 64x64 diagonal block of a dense triangular solve, by one warp in registers (rows lane and
// lane + 32), the block read from shared memory (Ds[i + 64 j], see stage_diag_block).
// which: 0 = L (unit lower, forward), 1 = U (backward), 2 = U^T (forward), 3 = L^T (backward).
// yb[0 .. 64) must already hold every contribution from outside the block.
__device__ __forceinline__ void dense_block_solve(int which, const double* __restrict__ Ds,
                                                  double* yb, int lane, double* xs) {
  constexpr int TB = 64;
  double r0 = yb[lane], r1 = yb[lane + 32];
  if (which == 0) {
    for (int i = 0; i < TB; ++i) {
      const double xi = __shfl_sync(0xffffffffu, i < 32 ? r0 : r1, i & 31);
      const double* col = Ds + i * TB;
      if (lane > i) r0 -= col[lane] * xi;
      if (lane + 32 > i) r1 -= col[lane + 32] * xi;
    }
  } else if (which == 1) {
    for (int i = TB - 1; i >= 0; --i) {
      const double* col = Ds + i * TB;
      if (lane == (i & 31)) {
        if (i < 32) r0 = r0 / col[i]; else r1 = r1 / col[i];
      }
      const double xi = __shfl_sync(0xffffffffu, i < 32 ? r0 : r1, i & 31);
      if (lane < i) r0 -= col[lane] * xi;
      if (lane + 32 < i) r1 -= col[lane + 32] * xi;
    }
  } else if (which == 2) {
    // w_j = (w_j - sum_{kb <= i < j} U(i,j) w_i) / U(j,j), forward
    for (int j = 0; j < TB; ++j) {
      const double* col = Ds + j * TB;
      double s = 0.0;
      const double w0 = r0, w1 = r1;
      if (lane < j) s += col[lane] * w0;
      if (lane + 32 < j) s += col[lane + 32] * w1;
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == (j & 31)) {
        if (j < 32) r0 = (r0 - s) / col[j]; else r1 = (r1 - s) / col[j];
      }
    }
  } else {
    // w_j = w_j - sum_{j < i < kb+64} L(i,j) w_i, backward
    for (int j = TB - 1; j >= 0; --j) {
      const double* col = Ds + j * TB;
      double s = 0.0;
      if (lane > j) s += col[lane] * r0;
      if (lane + 32 > j) s += col[lane + 32] * r1;
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == (j & 31)) {
        if (j < 32) r0 -= s; else r1 -= s;
      }
    }
  }
  yb[lane] = r0;
  yb[lane + 32] = r1;
  if (xs) {
    xs[lane] = r0;
    xs[lane + 32] = r1;
  }
}

// The 64 x 64 diagonal block of a front's columns [xb, xb + 64) (column x's rows s0 + xb ..
// s0 + xb + 63 start at position pz[x] + xb: a front's diagonal block is dense) copied into D
// (D[i + 64 j]) with 8-byte asynchronous copies, committed as one group; only for a block that
// lies inside the front.  dense_block_solve reads only the triangle it needs, so the other
// triangle's values may stay in D.
__device__ __forceinline__ void front_stage_async(const double* __restrict__ V,
                                                  const long long* pz, int xb, double* D, int tid,
                                                  int nt) {
  for (int idx = tid; idx < 64 * 64; idx += nt) {
    const int i = idx % 64, j = idx / 64;
    const unsigned dst = (unsigned)__cvta_generic_to_shared(D + idx);
    const double* src = V + pz[xb + j] + xb + i;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src));
  }
  asm volatile("cp.async.commit_group;\n" ::);
}

// The same block when it runs past the front (nb < 64 columns): the triangle's values and the
// identity on the padding, by plain loads.
__device__ __forceinline__ void front_stage_edge(const double* __restrict__ V, const long long* pz,
                                                 int xb, int nb, int which, double* D, int tid,
                                                 int nt) {
  for (int idx = tid; idx < 64 * 64; idx += nt) {
    const int i = idx % 64, j = idx / 64;
    double val = 0.0;
    if (i < nb && j < nb) {
      if (which == 0 ? i > j : i <= j) val = V[pz[xb + j] + xb + i];
    } else if (i == j) {
      val = 1.0;                                    // padding: identity
    }
    D[idx] = val;
  }
}

// A front in the push-form solves (which 0: L forward, 1: U backward), blocked: one CTA per
// (front, vector).  The front's unknowns y_S stay in shared memory; its columns are taken 64 at a
// time: the 64 x 64 triangle of the block (a front's diagonal block is dense, so column x's rows
// s0 .. s1-1 sit contiguously from position lp[x] - (x - s0)) is staged in shared memory and
// solved by one warp (dense_block_solve), then every thread pushes the block into the front's
// remaining rows.  After the last block the updates leaving the front go out: for L, the rows R
// below the front take y_R -= L(R, S) y_S, one sum and one atomic per row (R is the same row list
// in every column of the front); for U, the entries above row s0 of every column, one atomic
// each.  The chain from block to block is a triangle and two barriers instead of one barrier
// per column; each push is the sum of the block's products subtracted at once.
__global__ void __launch_bounds__(256) k_front_solve_blk(PlanDev P, const double* vals, int nrhs,
                                                         double* y, int64_t ylen,
                                                         const int32_t* __restrict__ fids,
                                                         int which, int tail) {
  constexpr int TB = 64;
  extern __shared__ double fsm[];
  const int f = fids[blockIdx.x];
  const int s0 = P.fs0[f], w = P.fw[f];
  const int wpad = (w + TB - 1) / TB * TB;
  double* Ds = fsm;                                 // [2][TB * TB] the blocks' triangles
  double* xs = Ds + 2 * TB * TB;                    // [TB] the block's solved values
  double* ys = xs + TB;                             // [wpad] the front's unknowns
  long long* pz = reinterpret_cast<long long*>(ys + ((P.fw_max + TB - 1) / TB) * TB);
  const int64_t v = blockIdx.y;
  const double* __restrict__ V = vals + (v / nrhs) * P.blob;
  double* yv = y + v * ylen;
  const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp, nt = blockDim.x;
  for (int x = tid; x < wpad; x += nt) {
    ys[x] = x < w ? yv[s0 + x] : 0.0;
    if (x < w) pz[x] = (long long)P.lp[s0 + x] - x;  // position of row s0 in column s0 + x
  }
  __syncthreads();
  const int nblk = wpad / TB;
  // block bi's triangle goes to Ds[bi & 1]; the next block's is copied in while this one is
  // solved and pushed
  const int xb0 = (which == 0 ? 0 : nblk - 1) * TB;
  if (xb0 + TB <= w) front_stage_async(V, pz, xb0, Ds, tid, nt);
  for (int bi = 0; bi < nblk; ++bi) {
    const int xb = (which == 0 ? bi : nblk - 1 - bi) * TB;
    const int nb = min(TB, w - xb);
    double* D = Ds + (bi & 1) * TB * TB;
    if (nb == TB) asm volatile("cp.async.wait_group 0;\n" ::);
    else front_stage_edge(V, pz, xb, nb, which, D, tid, nt);
    __syncthreads();
    if (bi + 1 < nblk) {
      const int xn = (which == 0 ? bi + 1 : nblk - 2 - bi) * TB;
      if (xn + TB <= w) front_stage_async(V, pz, xn, Ds + ((bi + 1) & 1) * TB * TB, tid, nt);
    }
    if (warp == 0) dense_block_solve(which, D, ys + xb, lane, xs);
    __syncthreads();
    const int lo = which == 0 ? xb + nb : 0, hi = which == 0 ? w : xb;
    for (int r = lo + tid; r < hi; r += nt) {
      double sum = 0.0;
      for (int j = 0; j < nb; ++j) sum += V[pz[xb + j] + r] * xs[j];
      ys[r] -= sum;
    }
    __syncthreads();
  }
  for (int x = tid; x < w; x += nt) yv[s0 + x] = ys[x];
  if (!tail) return;                                // k_front_solve_tail applies the rest
  if (which == 0) {
    const int64_t q0 = pz[0] + w;                   // the rows R in column s0
    const int m = (int)((int64_t)P.cp[s0 + 1] - q0);
    for (int i = tid; i < m; i += nt) {
      double sum = 0.0;
      for (int x = 0; x < w; ++x) sum += V[pz[x] + w + i] * ys[x];
      atomicAdd(yv + P.ri[q0 + i], -sum);
    }
  } else {
    for (int x = warp; x < w; x += nt / kWarp) {
      const double xx = ys[x];
      for (int64_t p = P.cp[s0 + x] + lane; p < pz[x]; p += kWarp)
        atomicAdd(yv + P.ri[p], -(V[p] * xx));
    }
  }
}

// A wide front in the push-form solves (which 0: L forward, 1: U backward) by a cluster of kFsC
// CTAs (grid (fronts * kFsC, vectors)): the front's unknowns are dealt out in 64-row blocks,
// block k to CTA k % kFsC, and every CTA keeps the front's unknowns in its shared memory but
// updates only its own blocks.  Per 64-column block: the CTA that owns it stages its triangle,
// solves it with one warp and writes the 64 values into every CTA's xs buffer (distributed shared
// memory, two buffers in turn); after one cluster barrier every CTA pushes the block into its own
// rows.  So the push over the rest of the front, which one CTA per front does alone in
// k_front_solve_blk, is spread over kFsC SMs.  The arithmetic of every unknown is the same as
// there (same triangle code, each row's sum over the block's columns in the same order).  The
// rows outside the front are left to k_front_solve_tail.  Every CTA of a cluster walks the same
// blocks, so all reach every barrier.
constexpr int kFsC = 8;

__global__ void __cluster_dims__(kFsC, 1, 1) __launch_bounds__(256)
    k_front_solve_cluster(PlanDev P, const double* vals, int nrhs, double* y, int64_t ylen,
                          const int32_t* __restrict__ fids, int which) {
  namespace cg = cooperative_groups;
  constexpr int TB = 64;
  extern __shared__ double fsm[];
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int f = fids[blockIdx.x / kFsC];
  const int s0 = P.fs0[f], w = P.fw[f];
  const int wpad = (w + TB - 1) / TB * TB;
  const int fwp = (P.fw_max + TB - 1) / TB * TB;
  double* Ds = fsm;                                 // [2][TB * TB] the owner's triangles
  double* xs = Ds + 2 * TB * TB;                    // [2][TB] solved values of a block
  double* ys = xs + 2 * TB;                         // [fwp] the front's unknowns
  long long* pz = reinterpret_cast<long long*>(ys + fwp);
  const int64_t v = blockIdx.y;
  const double* __restrict__ V = vals + (v / nrhs) * P.blob;
  double* yv = y + v * ylen;
  const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp, nt = blockDim.x;
  for (int x = tid; x < wpad; x += nt) {
    ys[x] = x < w ? yv[s0 + x] : 0.0;
    if (x < w) pz[x] = (long long)P.lp[s0 + x] - x;  // position of row s0 in column s0 + x
  }
  __syncthreads();
  const int nblk = wpad / TB;
  // this CTA's blocks kb (kb % kFsC == rank) take Ds[(kb / kFsC) & 1] in turn; the next one's
  // triangle is copied in while the cluster works on the blocks in between
  {
    const int k0 = which == 0 ? rank : nblk - 1 - ((nblk - 1 - rank) % kFsC + kFsC) % kFsC;
    if (k0 >= 0 && k0 < nblk && (k0 + 1) * TB <= w)
      front_stage_async(V, pz, k0 * TB, Ds + ((k0 / kFsC) & 1) * TB * TB, tid, nt);
  }
  for (int bi = 0; bi < nblk; ++bi) {
    const int kb = which == 0 ? bi : nblk - 1 - bi;
    const int xb = kb * TB;
    const int nb = min(TB, w - xb);
    double* xbuf = xs + (bi & 1) * TB;
    if (kb % kFsC == rank) {
      double* D = Ds + ((kb / kFsC) & 1) * TB * TB;
      if (nb == TB) asm volatile("cp.async.wait_group 0;\n" ::);
      else front_stage_edge(V, pz, xb, nb, which, D, tid, nt);
      __syncthreads();
      const int kn = which == 0 ? kb + kFsC : kb - kFsC;
      if (kn >= 0 && kn < nblk && (kn + 1) * TB <= w)
        front_stage_async(V, pz, kn * TB, Ds + ((kn / kFsC) & 1) * TB * TB, tid, nt);
      if (warp == 0) {
        dense_block_solve(which, D, ys + xb, lane, nullptr);
        __syncwarp();
        const double a = ys[xb + lane], b = ys[xb + lane + 32];
        for (int k = 0; k < kFsC; ++k) {
          double* dst = cl.map_shared_rank(xbuf, k);
          dst[lane] = a;
          dst[lane + 32] = b;
        }
      }
    }
    cl.sync();
    // this CTA's row blocks in [lo, hi): 64 rows per block, four blocks at a time
    const int lo = which == 0 ? xb + nb : 0, hi = which == 0 ? w : xb;
    if (lo < hi) {
      const int b_lo = lo / TB, b_hi = (hi + TB - 1) / TB;
      const int first = b_lo + ((rank - b_lo % kFsC) % kFsC + kFsC) % kFsC;
      for (int bb = first + (tid / TB) * kFsC; bb < b_hi; bb += (nt / TB) * kFsC) {
        const int r = bb * TB + tid % TB;
        if (r < lo || r >= hi) continue;
        double sum = 0.0;
        for (int j = 0; j < nb; ++j) sum += V[pz[xb + j] + r] * xbuf[j];
        ys[r] -= sum;
      }
    }
    __syncthreads();
  }
  for (int x = tid; x < w; x += nt)
    if ((x / TB) % kFsC == rank) yv[s0 + x] = ys[x];
}

// The part of a front's push solve outside the front, after k_front_solve_blk or
// k_front_solve_cluster has written the front's unknowns x_S: L: y_R -= L(R, S) x_S; U:
// y_r -= U(r, S) x_S for the rows r < s0 above the front.  One CTA per 64 columns of S (grid
// (ceil(max w / 64), fronts, vectors)), so a wide front's rows R or its long U columns are spread
// over many SMs instead of one CTA per front; each CTA adds its 64 columns' share of a row with
// one atomic.  (Grouping a CTA's work over several vectors was measured slower: fewer CTAs.)
__global__ void __launch_bounds__(256) k_front_solve_tail(PlanDev P, const double* vals, int nrhs,
                                                          double* y, int64_t ylen,
                                                          const int32_t* __restrict__ fids,
                                                          int which) {
  constexpr int TC = 64;
  __shared__ double xs[TC];
  __shared__ long long pzs[TC];
  const int f = fids[blockIdx.y];
  const int s0 = P.fs0[f], w = P.fw[f];
  const int x0 = blockIdx.x * TC;
  if (x0 >= w) return;                              // the same for every thread of the CTA
  const int nx = min(TC, w - x0);
  const int64_t v = blockIdx.z;
  const double* __restrict__ V = vals + (v / nrhs) * P.blob;
  double* yv = y + v * ylen;
  const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp, nt = blockDim.x;
  if (tid < nx) {
    xs[tid] = yv[s0 + x0 + tid];
    pzs[tid] = (long long)P.lp[s0 + x0 + tid] - (x0 + tid);   // row s0 in column s0 + x0 + tid
  }
  __syncthreads();
  if (which == 0) {
    const int64_t q0 = (int64_t)P.lp[s0] + w;       // the rows R in column s0
    const int m = (int)((int64_t)P.cp[s0 + 1] - q0);
    for (int i = tid; i < m; i += nt) {
      double sum = 0.0;
      for (int x = 0; x < nx; ++x) sum += V[pzs[x] + w + i] * xs[x];
      atomicAdd(yv + P.ri[q0 + i], -sum);
    }
  } else {
    for (int x = warp; x < nx; x += nt / kWarp) {
      const double xx = xs[x];
      for (int64_t p = P.cp[s0 + x0 + x] + lane; p < pzs[x]; p += kWarp)
        atomicAdd(yv + P.ri[p], -(V[p] * xx));
    }
  }
}

// Dense triangular solves on the ntp x ntp block, one CTA (256 threads) per vector, in 64-row
// blocks: the 64x64 diagonal block is solved by warp 0 in registers (rows lane, lane+32), the
// rest of the block column/row is applied by all threads with coalesced column reads.  Used when
// the batch has enough vectors to fill the GPU.
// which: 0 = L (unit lower, forward), 1 = U (backward), 2 = U^T (forward), 3 = L^T (backward)
__global__ void __launch_bounds__(256) k_dense_trsv(PlanDev P, const double* vals, int nrhs,
                                                    double* y, int64_t ylen, int which) {
  constexpr int TB = 64;
  __shared__ double xs[TB];
  __shared__ __align__(16) double Ds[TB * TB];
  const int64_t v = blockIdx.x;
  const double* __restrict__ D = vals + (v / nrhs) * P.blob + P.dbase;
  double* yd = y + v * ylen + P.t;
  const int64_t ld = P.ntp;
  const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp;
  const int nblk = (int)(P.ntp / TB);
  for (int bi = 0; bi < nblk; ++bi) {
    const int kb = (which == 0 || which == 2) ? bi * TB : (nblk - 1 - bi) * TB;
    stage_diag_block(D, ld, kb, Ds, tid, blockDim.x);
    if (which >= 2) {
      // pull the already-solved part into the block: w_j -= sum_i M(i, j) w_i
      for (int jj = warp; jj < TB; jj += 8) {
        const int j = kb + jj;
        double s = 0.0;
        if (which == 2) {
          for (int i = lane; i < kb; i += kWarp) s += D[i + (int64_t)j * ld] * yd[i];
        } else {
          for (int i = kb + TB + lane; i < (int)P.ntp; i += kWarp) s += D[i + (int64_t)j * ld] * yd[i];
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) yd[j] -= s;
      }
      __syncthreads();
    }
    stage_wait();
    __syncthreads();
    if (warp == 0) dense_block_solve(which, Ds, yd + kb, lane, xs);
    __syncthreads();
    if (which == 0) {          // rows below the block: y_r -= L(r, blk) x_blk
      for (int r = kb + TB + tid; r < (int)P.ntp; r += blockDim.x) {
        double s = 0.0;
#pragma unroll 8
        for (int i = 0; i < TB; ++i) s += D[r + (int64_t)(kb + i) * ld] * xs[i];
        yd[r] -= s;
      }
    } else if (which == 1) {   // rows above the block: y_r -= U(r, blk) x_blk
      for (int r = tid; r < kb; r += blockDim.x) {
        double s = 0.0;
#pragma unroll 8
        for (int i = 0; i < TB; ++i) s += D[r + (int64_t)(kb + i) * ld] * xs[i];
        yd[r] -= s;
      }
    }
    __syncthreads();
  }
}

// Blocked variant for few vectors (one matrix, few right-hand sides): per 64-block, one launch
// solves the diagonal block of every vector (a warp each), one launch pushes the solved block
// into the rest of the vector with many CTAs, so the triangle is read once at full bandwidth.
// Grid (instances, ceil(nrhs / 8)): the CTA stages its instance's diagonal block once and each
// warp solves one right-hand side.
__global__ void __launch_bounds__(256) k_trsv_blk_diag(PlanDev P, const double* vals, int nrhs,
                                                       double* y, int64_t ylen, int which, int kb) {
  __shared__ __align__(16) double Ds[64 * 64];
  const int64_t inst = blockIdx.x;
  const int k = blockIdx.y * 8 + threadIdx.x / kWarp;
  stage_diag_block(vals + inst * P.blob + P.dbase, P.ntp, kb, Ds, threadIdx.x, blockDim.x);
  stage_wait();
  __syncthreads();
  if (k >= nrhs) return;
  dense_block_solve(which, Ds, y + (inst * nrhs + k) * ylen + P.t + kb, threadIdx.x % kWarp,
                    nullptr);
}

// Push of a solved block kb: which 0/1 update rows (y_r -= M(r, blk) x_blk), which 2/3 update
// columns (w_j -= sum_i M(i, j) w_i over the block's rows); rows/columns [lo, hi); grid
// (chunks of 32, instances), 256 threads.  Vectors of one instance are processed 8 at a time
// from shared memory, so each matrix element is loaded once per 8 right-hand sides.  Rows: each
// of the 32 rows of a CTA is summed by 8 threads over 8 columns each (coalesced column reads),
// partial sums reduced in shared memory in a fixed order; columns: a warp per column of M reads
// the block's 64 rows of it (coalesced) and reduces with shuffles.
__global__ void __launch_bounds__(256) k_trsv_blk_update(PlanDev P, const double* vals, int nrhs,
                                                         double* y, int64_t ylen, int which,
                                                         int kb, int lo, int hi) {
  constexpr int TB = 64, VC = 8, RW = 32;
  __shared__ double xs[VC][TB];
  __shared__ double part[8][VC][RW];
  const int64_t inst = blockIdx.y;
  const double* __restrict__ D = vals + inst * P.blob + P.dbase;
  const int64_t ld = P.ntp;
  const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp;
  for (int vc = 0; vc < nrhs; vc += VC) {
    const int nv = nrhs - vc < VC ? nrhs - vc : VC;
    __syncthreads();
    for (int idx = tid; idx < VC * TB; idx += blockDim.x) {
      const int v = idx / TB, i = idx % TB;
      xs[v][i] = v < nv ? y[(inst * nrhs + vc + v) * ylen + P.t + kb + i] : 0.0;
    }
    __syncthreads();
    if (which < 2) {
      const int r = lo + blockIdx.x * RW + lane, g = warp;   // row, column group of 8
      double acc[VC];
#pragma unroll
      for (int v = 0; v < VC; ++v) acc[v] = 0.0;
      if (r < hi) {
#pragma unroll
        for (int ii = 0; ii < 8; ++ii) {
          const int i = g * 8 + ii;
          const double m = D[r + (int64_t)(kb + i) * ld];
#pragma unroll
          for (int v = 0; v < VC; ++v) acc[v] += m * xs[v][i];
        }
      }
#pragma unroll
      for (int v = 0; v < VC; ++v) part[g][v][lane] = acc[v];
      __syncthreads();
      if (tid < VC * RW) {
        const int v = tid / RW, rr = tid % RW, row = lo + blockIdx.x * RW + rr;
        if (v < nv && row < hi) {
          double sum = 0.0;
#pragma unroll
          for (int gg = 0; gg < 8; ++gg) sum += part[gg][v][rr];
          y[(inst * nrhs + vc + v) * ylen + P.t + row] -= sum;
        }
      }
    } else {
      for (int jj = warp; jj < RW; jj += 8) {
        const int r = lo + blockIdx.x * RW + jj;
        if (r >= hi) break;
        const double* colp = D + (int64_t)r * ld + kb;
        const double m0 = colp[lane], m1 = colp[lane + 32];
        for (int v = 0; v < nv; ++v) {
          double sum = m0 * xs[v][lane] + m1 * xs[v][lane + 32];
          for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
          if (lane == 0) y[(inst * nrhs + vc + v) * ylen + P.t + r] -= sum;
        }
      }
    }
  }
}

__global__ void k_grad(PlanDev P, int nrhs, const double* __restrict__ lambda,
                       const double* __restrict__ x, double* __restrict__ ga) {
  const int64_t b = blockIdx.y;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < P.nnz_g;
       e += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t r = P.g_row[e], c = P.g_col[e];
    double s = 0.0;
    for (int k = 0; k < nrhs; ++k) {
      const int64_t v = (b * nrhs + k) * P.n;
      s += lambda[v + r] * x[v + c];
    }
    ga[b * P.nnz_g + e] = -s;
  }
}

// r = b - A x (or b - A^T x) for every (instance, rhs) vector on the ORIGINAL matrix, and the
// infinity norms ||r||, ||x||, ||b||, ||A|| of each vector (as non-negative double bits) for
// ||r|| / (||A|| ||x|| + ||b||), the acceptance test of the solves.  Grid (chunks, vectors).
__global__ void k_residual(PlanDev P, int nrhs, const double* __restrict__ a,
                           const double* __restrict__ X, const double* __restrict__ Bm,
                           double* __restrict__ R, unsigned long long* norms, int transpose) {
  residual_rows(P, nrhs, a, X, Bm, R, norms, transpose, blockIdx.y, blockIdx.x, gridDim.x);
}

__global__ void k_resid_finish(int64_t nv, const unsigned long long* norms, double* out) {
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (v < nv) out[v] = residual_ratio(norms + 4 * v);
}

__global__ void k_axpy(int64_t n, const double* __restrict__ dx, double* __restrict__ x) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] += dx[i];
}

inline int grid1(int64_t work, int threads, int cap = 148 * 16) {
  int64_t g = (work + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// launch wrappers
// ---------------------------------------------------------------------------------------------

void launch_prepare_blob(const PlanDev& P, double* vals, int first, int count, bool assemble,
                         cudaStream_t s, LaunchCounter& lc) {
  if (assemble) {
    if (P.dbase > 0)
      cudaMemset2DAsync(vals + (int64_t)first * P.blob, sizeof(double) * P.blob, 0,
                        sizeof(double) * P.dbase, count, s);
    if (P.nasm_zero > 0) {
      k_zero_slots<<<dim3(grid1(P.nasm_zero, 256, 256), count), 256, 0, s>>>(P, vals, first);
      lc.n++;
    }
    return;
  }
  cudaMemsetAsync(vals + (int64_t)first * P.blob, 0, sizeof(double) * P.blob * count, s);
  if (P.ntp > P.nt) {
    k_pad_identity<<<dim3(1, count), 64, 0, s>>>(P, vals, first);
    lc.n++;
  }
}

void launch_ingest(const PlanDev& P, double* vals, int first, int count, const double* a,
                   cudaStream_t s, LaunchCounter& lc) {
  k_ingest<<<dim3(grid1(P.nnz_a, 256, 1024), count), 256, 0, s>>>(P, vals, first, a);
  lc.n++;
}

void launch_load_lu(const PlanDev& P, double* vals, int first, int count, const double* val,
                    cudaStream_t s, LaunchCounter& lc) {
  k_load_lu<<<dim3(grid1(P.nnz, 256, 1024), count), 256, 0, s>>>(P, vals, first, val);
  lc.n++;
}

void launch_export_lu(const PlanDev& P, const double* vals, int inst, double* val, cudaStream_t s,
                      LaunchCounter& lc) {
  k_export_lu<<<grid1(P.nnz, 256), 256, 0, s>>>(P, vals, inst, val);
  lc.n++;
}

void launch_pert(const PlanDev& P, const double* vals, int count, double pert, double* pert_dev,
                 cudaStream_t s, LaunchCounter& lc) {
  if (pert >= 0.0) {
    k_fill<<<(count + 127) / 128, 128, 0, s>>>(count, pert, pert_dev);
    lc.n++;
    return;
  }
  // pert_dev doubles as the bit accumulator (non-negative doubles order like their bits)
  unsigned long long* bits = reinterpret_cast<unsigned long long*>(pert_dev);
  cudaMemsetAsync(bits, 0, sizeof(double) * count, s);
  k_norm1<<<dim3(grid1(P.n, 8, 512), count), 256, 0, s>>>(P, vals, bits);
  k_pert_finish<<<(count + 127) / 128, 128, 0, s>>>(count, bits, pert_dev);
  lc.n += 2;
}

void launch_sparse_level(const PlanDev& P, double* vals, int count, const double* pert,
                         int32_t* status, int begin, int ncols, int wpc, int max_nl,
                         int max_pairs, int block, int cpw, int lanes, int grow, int occ,
                         cudaStream_t s, LaunchCounter& lc) {
  // a wide level of heavy columns whose columns of the batch are fewer than half the warps the
  // GPU should hold (occ per SM): 2, 4 or 8 warps per column, so the pairs of each column are
  // shared instead of walked by one warp
  const int64_t want = (int64_t)occ * sm_count();
  if (grow && occ > 0 && wpc == 1)
    while (wpc < 8 && (int64_t)ncols * count * wpc * 2 <= want && max_pairs > 4 * wpc) wpc *= 2;
  // a level whose CTA-per-column grid covers fewer CTAs than the GPU should hold (occ warps per
  // SM, two CTAs per SM when occ = 0) and whose columns have more pairs than one CTA's warps:
  // split each column's pairs over several CTAs
  constexpr int kSplitMaxL = 6144;               // L(:,c) staged in 48 KB of shared memory
  const int64_t ctas = (int64_t)ncols * count;
  const int64_t target = occ > 0 ? std::max<int64_t>(want / 8, 2 * (int64_t)sm_count())
                                 : 2 * (int64_t)sm_count();
  if (wpc > 1 && ctas < target && max_pairs > 16 && max_nl <= kSplitMaxL) {
    int splits = (int)std::min<int64_t>((target + ctas - 1) / ctas, (max_pairs + 7) / 8);
    k_sparse_split<<<dim3(ncols * splits, count), 256, sizeof(double) * std::max(max_nl, 1), s>>>(
        P, vals, pert, begin, splits);
    k_sparse_scale<<<dim3(ncols, count), 256, 0, s>>>(P, vals, pert, status, begin);
    lc.n += 2;
    return;
  }
  if (block != 128) block = 256;
  wpc = std::max(1, std::min(wpc, block / kWarp));
  if (wpc > 1 || (lanes != 8 && lanes != 16)) lanes = kWarp;
  const int groups = block / (wpc == 1 ? lanes : kWarp * wpc);
  const int per_cta = groups * std::max(1, cpw);
  // a CTA per column: its L(:,c) staged in shared memory when eight CTAs of it still fit on an
  // SM (at most 24 KB each), so the staging costs no occupancy
  constexpr int kStageMaxL = 3072;
  const bool stage = groups == 1 && max_nl > 0 && max_nl <= kStageMaxL;
  const size_t smem = stage ? sizeof(double) * max_nl : 0;
  k_sparse_level<<<dim3((ncols + per_cta - 1) / per_cta, count), block, smem, s>>>(
      P, vals, pert, status, begin, ncols, wpc, std::max(1, cpw), stage ? 1 : 0, lanes);
  lc.n++;
}

void launch_sparse_level_det(const PlanDev& P, double* vals, int count, const double* pert,
                             int32_t* status, int begin, int ncols, int64_t t0, int64_t t1,
                             cudaStream_t s, LaunchCounter& lc) {
  k_sparse_scale<<<dim3(ncols, count), 256, 0, s>>>(P, vals, pert, status, begin);
  lc.n++;
  const int64_t nt = t1 - t0;
  if (nt > 0) {
    k_sparse_pull<<<dim3((unsigned)((nt + 7) / 8), count), 256, 0, s>>>(P, vals, t0, nt);
    lc.n++;
  }
}

void launch_rows_solve(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                       int64_t ylen, const int32_t* rows, int begin, int nrows, int which,
                       cudaStream_t s, LaunchCounter& lc) {
  if (nrows <= 0) return;
  k_rows_solve<<<dim3((nrows + 7) / 8, count * nrhs), 256, 0, s>>>(P, vals, nrhs, y, ylen, rows,
                                                                   begin, nrows, which);
  lc.n++;
}

int persistent_grid(size_t smem) {
  int dev = 0, per_sm = 0;
  cudaGetDevice(&dev);
  ensure_smem_limit((const void*)k_sparse_persistent, smem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sparse_persistent, 256, smem) !=
          cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    return 0;
  }
  return per_sm * sm_count();
}

void launch_sparse_persistent(const PlanDev& P, double* vals, int count, const double* pert,
                              int32_t* status, const int4* desc, int nlev, unsigned* bar,
                              int groups, int* err, double budget_ms, int extra, int grid,
                              size_t smem, cudaStream_t s, LaunchCounter& lc) {
  cudaMemsetAsync(bar, 0, sizeof(unsigned) * groups, s);
  cudaMemsetAsync(err, 0, sizeof(int), s);
  ensure_smem_limit((const void*)k_sparse_persistent, smem);
  const unsigned long long budget = (unsigned long long)(budget_ms * 1e6);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;      // every CTA resident at once
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k_sparse_persistent, P, vals, pert, status, desc, nlev, count, bar, err,
                     budget, extra);
  lc.n++;
}

void launch_solve_permute_in(const PlanDev& P, int count, int nrhs, const double* B, double* y,
                             int64_t ylen, int transpose, cudaStream_t s, LaunchCounter& lc) {
  k_permute_in<<<dim3(grid1(ylen, 256, 256), count * nrhs), 256, 0, s>>>(P, nrhs, B, y, ylen,
                                                                        transpose);
  lc.n++;
}

void launch_solve_permute_out(const PlanDev& P, int count, int nrhs, const double* y, double* X,
                              int64_t ylen, int transpose, cudaStream_t s, LaunchCounter& lc) {
  k_permute_out<<<dim3(grid1(P.n, 256, 256), count * nrhs), 256, 0, s>>>(P, nrhs, y, X, ylen,
                                                                        transpose);
  lc.n++;
}

#define GLU_SOLVE_LAUNCH(KERNEL)                                                             \
  k_##KERNEL<<<dim3((ncols + 7) / 8, count * nrhs), 256, 0, s>>>(P, vals, nrhs, y, ylen, cols, \
                                                                 begin, ncols);              \
  lc.n++;
// the push forms take kSolveVecs right-hand sides per warp
#define GLU_SOLVE_LAUNCH_GROUPED(KERNEL)                                                      \
  k_##KERNEL<<<dim3((ncols + 7) / 8, count * ((nrhs + kSolveVecs - 1) / kSolveVecs)), 256, 0,  \
               s>>>(P, vals, nrhs, y, ylen, cols, begin, ncols);                              \
  lc.n++;

void launch_sparse_lsolve(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                          int64_t ylen, const int32_t* cols, int begin, int ncols,
                          cudaStream_t s, LaunchCounter& lc) {
  GLU_SOLVE_LAUNCH_GROUPED(sparse_lsolve)
}
void launch_sparse_usolve(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                          int64_t ylen, const int32_t* cols, int begin, int ncols,
                          cudaStream_t s, LaunchCounter& lc) {
  GLU_SOLVE_LAUNCH_GROUPED(sparse_usolve)
}
void launch_sparse_utsolve(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                           int64_t ylen, const int32_t* cols, int begin, int ncols,
                           cudaStream_t s, LaunchCounter& lc) {
  GLU_SOLVE_LAUNCH(sparse_utsolve)
}
void launch_sparse_ltsolve(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                           int64_t ylen, const int32_t* cols, int begin, int ncols,
                           cudaStream_t s, LaunchCounter& lc) {
  GLU_SOLVE_LAUNCH(sparse_ltsolve)
}

void launch_front_solve(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                        int64_t ylen, const int32_t* fids, int nfronts, int max_w, int which,
                        cudaStream_t s, LaunchCounter& lc) {
  if (nfronts <= 0) return;
  const size_t fwp = ((size_t)P.fw_max + 63) / 64 * 64;
  const size_t smem_blk = sizeof(double) * (2 * 64 * 64 + 64 + fwp) + sizeof(long long) * fwp;
  if (which <= 1 && smem_blk <= 200 * 1024) {
    // fronts wider than two blocks leave the rows outside the front to k_front_solve_tail;
    // a level with a front of at least four blocks solves its fronts by clusters of CTAs
    const bool split = max_w > 128;
    const size_t smem_cl = sizeof(double) * (2 * 64 * 64 + 2 * 64 + fwp) + sizeof(long long) * fwp;
    if (max_w >= 256 && smem_cl <= 200 * 1024) {
      ensure_smem_limit((const void*)k_front_solve_cluster, smem_cl);
      k_front_solve_cluster<<<dim3((unsigned)(nfronts * kFsC), (unsigned)(count * nrhs)), 256,
                              smem_cl, s>>>(P, vals, nrhs, y, ylen, fids, which);
    } else {
      ensure_smem_limit((const void*)k_front_solve_blk, smem_blk);
      k_front_solve_blk<<<dim3((unsigned)nfronts, (unsigned)(count * nrhs)), 256, smem_blk, s>>>(
          P, vals, nrhs, y, ylen, fids, which, split ? 0 : 1);
    }
    lc.n++;
    if (split) {
      k_front_solve_tail<<<dim3((unsigned)((max_w + 63) / 64), (unsigned)nfronts,
                                (unsigned)(count * nrhs)), 256, 0, s>>>(P, vals, nrhs, y, ylen,
                                                                        fids, which);
      lc.n++;
    }
    return;
  }
  const size_t smem = (2 * sizeof(double) + 2 * sizeof(uint32_t)) * (size_t)P.fw_max;
  if (which <= 1 && smem <= 96 * 1024) {
    ensure_smem_limit((const void*)k_front_solve_push, smem);
    k_front_solve_push<<<dim3((unsigned)nfronts, (unsigned)(count * nrhs)), 256, smem, s>>>(
        P, vals, nrhs, y, ylen, fids, which);
  } else {
    k_front_solve<<<dim3((unsigned)nfronts, (unsigned)(count * nrhs)), 256, 0, s>>>(
        P, vals, nrhs, y, ylen, fids, which);
  }
  lc.n++;
}

void launch_border(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                   int64_t ylen, int transpose, cudaStream_t s, LaunchCounter& lc) {
  if (P.nt == 0) return;
  if (!transpose && P.nbordck > 0)
    k_border_chunks<<<dim3((unsigned)((P.nbordck + 7) / 8), count * nrhs), 256, 0, s>>>(
        P, vals, nrhs, y, ylen);
  else
    k_border<<<dim3((P.nt + 7) / 8, count * nrhs), 256, 0, s>>>(P, vals, nrhs, y, ylen, transpose);
  lc.n++;
}

void launch_dense_trsv(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                       int64_t ylen, int which, cudaStream_t s, LaunchCounter& lc) {
  if (P.ntp == 0) return;
  const int64_t nvec = (int64_t)count * nrhs;
  if (nvec >= 256 || P.ntp < 1024) {       // enough vectors to fill the GPU: one CTA each
    k_dense_trsv<<<(unsigned)nvec, 256, 0, s>>>(P, vals, nrhs, y, ylen, which);
    lc.n++;
    return;
  }
  const int nblk = (int)(P.ntp / 64);
  for (int bi = 0; bi < nblk; ++bi) {
    const int kb = (which == 0 || which == 2) ? bi * 64 : (nblk - 1 - bi) * 64;
    k_trsv_blk_diag<<<dim3((unsigned)count, (unsigned)((nrhs + 7) / 8)), 256, 0, s>>>(
        P, vals, nrhs, y, ylen, which, kb);
    const int lo = (which == 0 || which == 2) ? kb + 64 : 0;
    const int hi = (which == 0 || which == 2) ? (int)P.ntp : kb;
    if (hi > lo)
      k_trsv_blk_update<<<dim3((unsigned)((hi - lo + 31) / 32), (unsigned)count), 256, 0, s>>>(
          P, vals, nrhs, y, ylen, which, kb, lo, hi);
    lc.n += hi > lo ? 2 : 1;
  }
}

void launch_residual(const PlanDev& P, int count, int nrhs, const double* a, const double* X,
                     const double* B, double* R, unsigned long long* norms, double* resid,
                     int transpose, cudaStream_t s, LaunchCounter& lc) {
  const int64_t nv = (int64_t)count * nrhs;
  cudaMemsetAsync(norms, 0, sizeof(unsigned long long) * 4 * nv, s);
  k_residual<<<dim3(grid1(P.n, 256, 64), (unsigned)nv), 256, 0, s>>>(P, nrhs, a, X, B, R, norms,
                                                                    transpose);
  lc.n++;
  if (resid) {
    k_resid_finish<<<(unsigned)((nv + 127) / 128), 128, 0, s>>>(nv, norms, resid);
    lc.n++;
  }
}

void launch_axpy(int64_t n, const double* dx, double* x, cudaStream_t s, LaunchCounter& lc) {
  k_axpy<<<grid1(n, 256, 4096), 256, 0, s>>>(n, dx, x);
  lc.n++;
}

void launch_grad(const PlanDev& P, int count, int nrhs, const double* lambda, const double* x,
                 double* ga, cudaStream_t s, LaunchCounter& lc) {
  k_grad<<<dim3(grid1(P.nnz_g, 256, 1024), count), 256, 0, s>>>(P, nrhs, lambda, x, ga);
  lc.n++;
}

}  // namespace glu
