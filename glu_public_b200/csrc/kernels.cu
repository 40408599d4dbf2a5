// Device kernels of the GLU numeric phase for sm_100a (FP64 throughout).
//
// Factorization = sparse phase + dense phase:
//  * sparse phase: one launch per level of the reference's level sets restricted to the
//    columns before the dense trailing block (src/symbolic.cc:106-151 builds those levels).  A
//    warp (narrow levels: a CTA) owns one column c: it divides L(:,c) by the pivot
//    (src/numeric.cu:37-47) and then, for every U(c,j) != 0, subtracts L(:,c)*U(c,j) from
//    column j (src/numeric.cu:51-89).  The target slots come from the precomputed position map
//    instead of the reference's scan of the whole of column j, so each update costs one load of
//    the map entry; targets inside the dense block are addressed arithmetically.  Columns of
//    one level may hit the same target, so updates are FP64 atomics, as in the reference.
//  * dense phase: right-looking blocked LU without pivoting of the trailing block that fill has
//    made dense: per panel step one launch factors the nb x nb diagonal block (redundantly in
//    every CTA's shared memory), solves the L21 row blocks and U12 column blocks, and one launch
//    applies the rank-nb trailing update with FP64 DMMA (mma.sync m8n8k4 f64) tensor-core tiles.
//
// Every kernel takes the instance index from blockIdx.y / blockIdx.z, so one launch covers a
// whole batch of value sets of the same pattern.
#include <cuda_runtime.h>

#include <cstdint>

#include "glu_b200.h"
#include "kernels.cuh"

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

// MODE 0: each warp owns one column (blockDim/32 columns per CTA).
// MODE 1: the whole CTA owns one column; its warps split the U(c,:) pairs.
template <int MODE>
__global__ void __launch_bounds__(256) k_sparse_level(PlanDev P, double* vals,
                                                      const double* __restrict__ pert,
                                                      int32_t* status, int begin, int ncols) {
  const int b = blockIdx.y;
  double* __restrict__ V = vals + (int64_t)b * P.blob;
  const int lane = threadIdx.x % kWarp;
  int col, gtid, gsize, wig, nwg;
  if (MODE == 0) {
    col = blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp;
    if (col >= ncols) return;
    gtid = lane;
    gsize = kWarp;
    wig = 0;
    nwg = 1;
  } else {
    col = blockIdx.x;
    gtid = threadIdx.x;
    gsize = blockDim.x;
    wig = threadIdx.x / kWarp;
    nwg = blockDim.x / kWarp;
  }
  const uint32_t c = (uint32_t)P.scols[begin + col];
  const uint32_t dslot = P.lp[c];
  const uint32_t l0 = dslot + 1;
  const uint32_t nL = P.cp[c + 1] - l0;
  const double d0 = V[dslot];
  const double pv = pert[b];
  double d = d0;
  const bool perturbed = pv > 0.0 && nL > 0 && fabs(d0) < pv;   // numeric.cu:139-140
  if (perturbed) d = pv;
  if (MODE == 0) __syncwarp(); else __syncthreads();
  if (gtid == 0) {
    if (perturbed) V[dslot] = d;
    pivot_flags(status, b, d, perturbed);
  }
  for (uint32_t k = gtid; k < nL; k += gsize) V[l0 + k] = V[l0 + k] / d;
  if (MODE == 0) __syncwarp(); else __syncthreads();

  const int64_t q1 = P.pair_ptr[c + 1];
  const uint32_t nsplit = P.lsplit[c];
  for (int64_t q = P.pair_ptr[c] + wig; q < q1; q += nwg) {
    const uint32_t j = (uint32_t)P.pair_j[q];
    const double u = V[P.pair_uslot[q]];
    const int32_t* __restrict__ tm = P.tmap + P.pair_moff[q];
    const uint32_t nsp = j < P.t ? nL : nsplit;
    const int64_t dcol = P.dbase + (int64_t)(j - P.t) * P.ntp - (int64_t)P.t;
    for (uint32_t k = lane; k < nL; k += kWarp) {
      const double l = V[l0 + k];
      const int64_t tgt = (k < nsp) ? (int64_t)tm[k] : dcol + (int64_t)P.ri[l0 + k];
      atomicAdd(V + tgt, -(l * u));
    }
  }
}

// ---------------------------------------------------------------------------------------------
// dense phase: panel step k (diagonal block factor + L21 row blocks + U12 column blocks)
// ---------------------------------------------------------------------------------------------

template <int NB>
__global__ void __launch_bounds__(256) k_dense_panel(PlanDev P, double* vals,
                                                     const double* __restrict__ pert,
                                                     int32_t* status, int k, int nrb) {
  constexpr int S = NB + 1;          // smem column stride of the diagonal block
  constexpr int RB = 64;             // rows (or columns) of one L21 (U12) block
  constexpr int SB = (RB > NB ? RB : NB) + 1;
  extern __shared__ double sm[];
  double* A11 = sm;                  // NB x NB, column-major, stride S
  double* Bs = sm + NB * S;          // RB x NB (row block) or NB x RB (column block), stride SB
  const int b = blockIdx.y;
  const int tid = threadIdx.x;
  const int64_t ld = P.ntp;
  double* __restrict__ D = vals + (int64_t)b * P.blob + P.dbase;
  const double pv = pert[b];

  for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
    const int i = idx % NB, j = idx / NB;
    A11[i + j * S] = D[(int64_t)(k + i) + (int64_t)(k + j) * ld];
  }
  // prefetch this CTA's off-diagonal block while the diagonal block is factored
  const int role = blockIdx.x;       // 0: diagonal writer, 1..nrb: row block, rest: column block
  if (role >= 1 && role <= nrb) {
    const int r0 = k + NB + (role - 1) * RB;
    for (int idx = tid; idx < RB * NB; idx += blockDim.x) {
      const int i = idx % RB, j = idx / RB;
      Bs[i + j * SB] = D[(int64_t)(r0 + i) + (int64_t)(k + j) * ld];
    }
  } else if (role > nrb) {
    const int c0 = k + NB + (role - 1 - nrb) * RB;
    for (int idx = tid; idx < NB * RB; idx += blockDim.x) {
      const int i = idx % NB, j = idx / NB;
      Bs[i + j * SB] = D[(int64_t)(k + i) + (int64_t)(c0 + j) * ld];
    }
  }
  __syncthreads();

  // unblocked right-looking LU of the diagonal block (src/numeric.cu:28-89 on a dense block)
  for (int kk = 0; kk < NB; ++kk) {
    const double d0 = A11[kk + kk * S];
    const bool perturbed = pv > 0.0 && P.dhasl[k + kk] && fabs(d0) < pv;
    const double d = perturbed ? pv : d0;
    const int m = NB - kk - 1;
    for (int i = tid; i < m; i += blockDim.x) A11[kk + 1 + i + kk * S] /= d;
    __syncthreads();
    for (int idx = tid; idx < m * m; idx += blockDim.x) {
      const int i = kk + 1 + idx % m, j = kk + 1 + idx / m;
      A11[i + j * S] -= A11[i + kk * S] * A11[kk + j * S];
    }
    if (tid == 0) {
      A11[kk + kk * S] = d;
      if (role == 0) pivot_flags(status, b, d, perturbed);
    }
    __syncthreads();
  }

  if (role == 0) {
    for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
      const int i = idx % NB, j = idx / NB;
      D[(int64_t)(k + i) + (int64_t)(k + j) * ld] = A11[i + j * S];
    }
    return;
  }
  const int lane4 = tid % 4;
  const int line = tid / 4;          // 64 lines (rows or columns) x 4 threads, same warp
  if (role <= nrb) {
    // L21 = B * U11^-1: row `line`, columns j = lane4 (mod 4)
    for (int kk = 0; kk < NB; ++kk) {
      if ((kk & 3) == lane4) Bs[line + kk * SB] = Bs[line + kk * SB] / A11[kk + kk * S];
      __syncwarp();
      const double x = Bs[line + kk * SB];
      for (int j = kk + 1 + ((lane4 - kk - 1) & 3); j < NB; j += 4)
        Bs[line + j * SB] -= x * A11[kk + j * S];
      __syncwarp();
    }
    __syncthreads();
    const int r0 = k + NB + (role - 1) * RB;
    for (int idx = tid; idx < RB * NB; idx += blockDim.x) {
      const int i = idx % RB, j = idx / RB;
      D[(int64_t)(r0 + i) + (int64_t)(k + j) * ld] = Bs[i + j * SB];
    }
  } else {
    // U12 = L11^-1 * B: column `line`, rows i = lane4 (mod 4); unit diagonal
    for (int kk = 0; kk < NB; ++kk) {
      __syncwarp();
      const double y = Bs[kk + line * SB];
      for (int i = kk + 1 + ((lane4 - kk - 1) & 3); i < NB; i += 4)
        Bs[i + line * SB] -= A11[i + kk * S] * y;
    }
    __syncthreads();
    const int c0 = k + NB + (role - 1 - nrb) * RB;
    for (int idx = tid; idx < NB * RB; idx += blockDim.x) {
      const int i = idx % NB, j = idx / NB;
      D[(int64_t)(k + i) + (int64_t)(c0 + j) * ld] = Bs[i + j * SB];
    }
  }
}

// ---------------------------------------------------------------------------------------------
// DMMA GEMM: C -= A * B, column-major, 64x64 CTA tile, 4 warps of 32x32, K in chunks of 32,
// two-stage cp.async pipeline.  Tensor-core instruction: mma.sync.m8n8k4.f64 (FP64 DMMA).
// ---------------------------------------------------------------------------------------------

constexpr int GM = 64, GN = 64, GK = 32;
constexpr int AS = GM + 4;     // As[k][m] stride (== 4 mod 16 doubles: conflict-free fragments)
constexpr int BS = GK + 4;     // Bs[n][k] stride
constexpr int kGemmSmem = 2 * (GK * AS + GN * BS) * 8;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(128) k_gemm_sub(int M, int N, int K, const double* A, int lda,
                                                  const double* B, int ldb, double* C, int ldc,
                                                  int64_t sA, int64_t sB, int64_t sC) {
  extern __shared__ double sm[];
  double* As = sm;                     // [2][GK][AS]
  double* Bs = sm + 2 * GK * AS;       // [2][GN][BS]
  const int z = blockIdx.z;
  A += z * sA;
  B += z * sB;
  C += z * sC;
  const int m0 = blockIdx.x * GM, n0 = blockIdx.y * GN;
  const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;

  auto load = [&](int stage, int k0) {
    double* as = As + stage * GK * AS;
    double* bs = Bs + stage * GN * BS;
    for (int idx = tid; idx < GK * (GM / 2); idx += 128) {
      const int kc = idx / (GM / 2), mc = (idx % (GM / 2)) * 2;
      const bool ok = (m0 + mc < M) && (k0 + kc < K);
      const double* src = ok ? A + (int64_t)(m0 + mc) + (int64_t)(k0 + kc) * lda : A;
      cp_async16(as + kc * AS + mc, src, ok);
    }
    for (int idx = tid; idx < GN * (GK / 2); idx += 128) {
      const int nc = idx / (GK / 2), kc = (idx % (GK / 2)) * 2;
      const bool ok = (n0 + nc < N) && (k0 + kc < K);
      const double* src = ok ? B + (int64_t)(k0 + kc) + (int64_t)(n0 + nc) * ldb : B;
      cp_async16(bs + nc * BS + kc, src, ok);
    }
  };

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  const int nk = (K + GK - 1) / GK;
  load(0, 0);
  cp_async_commit();
  for (int kt = 0; kt < nk; ++kt) {
    if (kt + 1 < nk) {
      load((kt + 1) & 1, (kt + 1) * GK);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double* as = As + (kt & 1) * GK * AS;
    const double* bs = Bs + (kt & 1) * GN * BS;
#pragma unroll
    for (int kk = 0; kk < GK; kk += 4) {
      double a[4], bf[4];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) a[mi] = as[(kk + (lane & 3)) * AS + wm + mi * 8 + (lane >> 2)];
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) bf[ni] = bs[(wn + ni * 8 + (lane >> 2)) * BS + kk + (lane & 3)];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) dmma884(acc[mi][ni][0], acc[mi][ni][1], a[mi], bf[ni]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mi = 0; mi < 4; ++mi) {
    const int row = m0 + wm + mi * 8 + (lane >> 2);
    if (row >= M) continue;
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int col = n0 + wn + ni * 8 + (lane & 3) * 2 + e;
        if (col < N) {
          double* cptr = C + (int64_t)row + (int64_t)col * ldc;
          *cptr = *cptr - acc[mi][ni][e];
        }
      }
    }
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

// L solve, column oriented with unit diagonal (symbolic.cc:221-226), one warp per column.
__global__ void k_sparse_lsolve(PlanDev P, const double* vals, int nrhs, double* y, int64_t ylen,
                                const int32_t* __restrict__ cols, int begin, int ncols) {
  const int w = blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp;
  if (w >= ncols) return;
  const int lane = threadIdx.x % kWarp;
  const int64_t v = blockIdx.y;
  const double* V = vals + (v / nrhs) * P.blob;
  double* yv = y + v * ylen;
  const uint32_t c = (uint32_t)cols[begin + w];
  const double yc = yv[c];
  for (uint32_t p = P.lp[c] + 1 + lane; p < P.cp[c + 1]; p += kWarp)
    atomicAdd(yv + P.ri[p], -(V[p] * yc));
}

// U solve (symbolic.cc:228-236), one warp per column.
__global__ void k_sparse_usolve(PlanDev P, const double* vals, int nrhs, double* y, int64_t ylen,
                                const int32_t* __restrict__ cols, int begin, int ncols) {
  const int w = blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp;
  if (w >= ncols) return;
  const int lane = threadIdx.x % kWarp;
  const int64_t v = blockIdx.y;
  const double* V = vals + (v / nrhs) * P.blob;
  double* yv = y + v * ylen;
  const uint32_t c = (uint32_t)cols[begin + w];
  const double xc = yv[c] / V[P.lp[c]];
  __syncwarp();
  if (lane == 0) yv[c] = xc;
  for (uint32_t p = P.cp[c] + lane; p < P.lp[c]; p += kWarp) atomicAdd(yv + P.ri[p], -(V[p] * xc));
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

// Dense triangular solves on the ntp x ntp block, one CTA (256 threads) per vector, in 64-row
// blocks: the 64x64 diagonal block is solved by warp 0 in registers (rows lane, lane+32), the
// rest of the block column/row is applied by all threads with coalesced column reads.
// which: 0 = L (unit lower, forward), 1 = U (backward), 2 = U^T (forward), 3 = L^T (backward)
__global__ void __launch_bounds__(256) k_dense_trsv(PlanDev P, const double* vals, int nrhs,
                                                    double* y, int64_t ylen, int which) {
  constexpr int TB = 64;
  __shared__ double xs[TB];
  const int64_t v = blockIdx.x;
  const double* __restrict__ D = vals + (v / nrhs) * P.blob + P.dbase;
  double* yd = y + v * ylen + P.t;
  const int64_t ld = P.ntp;
  const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp;
  const int nblk = (int)(P.ntp / TB);
  for (int bi = 0; bi < nblk; ++bi) {
    const int kb = (which == 0 || which == 2) ? bi * TB : (nblk - 1 - bi) * TB;
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
    if (warp == 0) {
      double r0 = yd[kb + lane], r1 = yd[kb + lane + 32];
      if (which == 0) {
        for (int i = 0; i < TB; ++i) {
          const double xi = __shfl_sync(0xffffffffu, i < 32 ? r0 : r1, i & 31);
          const double* col = D + (int64_t)(kb + i) * ld + kb;
          if (lane > i) r0 -= col[lane] * xi;
          if (lane + 32 > i) r1 -= col[lane + 32] * xi;
        }
      } else if (which == 1) {
        for (int i = TB - 1; i >= 0; --i) {
          const double* col = D + (int64_t)(kb + i) * ld + kb;
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
          const double* col = D + (int64_t)(kb + j) * ld + kb;
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
          const double* col = D + (int64_t)(kb + j) * ld + kb;
          double s = 0.0;
          if (lane > j) s += col[lane] * r0;
          if (lane + 32 > j) s += col[lane + 32] * r1;
          for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
          if (lane == (j & 31)) {
            if (j < 32) r0 -= s; else r1 -= s;
          }
        }
      }
      yd[kb + lane] = r0;
      yd[kb + lane + 32] = r1;
      xs[lane] = r0;
      xs[lane + 32] = r1;
    }
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

void launch_prepare_blob(const PlanDev& P, double* vals, int first, int count, cudaStream_t s,
                         LaunchCounter& lc) {
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
                         int32_t* status, int begin, int ncols, int mode, cudaStream_t s,
                         LaunchCounter& lc) {
  if (mode == 0) {
    k_sparse_level<0><<<dim3((ncols + 7) / 8, count), 256, 0, s>>>(P, vals, pert, status, begin,
                                                                   ncols);
  } else {
    k_sparse_level<1><<<dim3(ncols, count), 256, 0, s>>>(P, vals, pert, status, begin, ncols);
  }
  lc.n++;
}

void launch_dense_panel(const PlanDev& P, double* vals, int count, const double* pert,
                        int32_t* status, int k, int nb, cudaStream_t s, LaunchCounter& lc) {
  const int rest = (int)P.ntp - k - nb;
  const int nrb = rest / 64;
  const int grid = 1 + 2 * nrb;
  if (nb == 64) {
    const int smem = (64 * 65 + 64 * 65) * 8;
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(k_dense_panel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      attr = true;
    }
    k_dense_panel<64><<<dim3(grid, count), 256, smem, s>>>(P, vals, pert, status, k, nrb);
  } else {
    const int smem = (32 * 33 + 64 * 65) * 8;
    k_dense_panel<32><<<dim3(grid, count), 256, smem, s>>>(P, vals, pert, status, k, nrb);
  }
  lc.n++;
}

void launch_gemm_sub(int M, int N, int K, const double* A, int lda, const double* B, int ldb,
                     double* C, int ldc, int count, int64_t strideA, int64_t strideB,
                     int64_t strideC, cudaStream_t s, LaunchCounter& lc) {
  if (M <= 0 || N <= 0 || K <= 0 || count <= 0) return;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_gemm_sub, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem);
    attr = true;
  }
  dim3 grid((M + GM - 1) / GM, (N + GN - 1) / GN, count);
  k_gemm_sub<<<grid, 128, kGemmSmem, s>>>(M, N, K, A, lda, B, ldb, C, ldc, strideA, strideB,
                                          strideC);
  lc.n++;
}

void launch_dense_update(const PlanDev& P, double* vals, int count, int k, int nb,
                         cudaStream_t s, LaunchCounter& lc) {
  const int m = (int)P.ntp - k - nb;
  if (m <= 0) return;
  double* D = vals + P.dbase;
  const int64_t ld = P.ntp;
  launch_gemm_sub(m, m, nb, D + (k + nb) + (int64_t)k * ld, (int)ld, D + k + (int64_t)(k + nb) * ld,
                  (int)ld, D + (k + nb) + (int64_t)(k + nb) * ld, (int)ld, count, P.blob, P.blob,
                  P.blob, s, lc);
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

void launch_sparse_lsolve(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                          int64_t ylen, const int32_t* cols, int begin, int ncols,
                          cudaStream_t s, LaunchCounter& lc) {
  GLU_SOLVE_LAUNCH(sparse_lsolve)
}
void launch_sparse_usolve(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                          int64_t ylen, const int32_t* cols, int begin, int ncols,
                          cudaStream_t s, LaunchCounter& lc) {
  GLU_SOLVE_LAUNCH(sparse_usolve)
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

void launch_border(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                   int64_t ylen, int transpose, cudaStream_t s, LaunchCounter& lc) {
  if (P.nt == 0) return;
  k_border<<<dim3((P.nt + 7) / 8, count * nrhs), 256, 0, s>>>(P, vals, nrhs, y, ylen, transpose);
  lc.n++;
}

void launch_dense_trsv(const PlanDev& P, const double* vals, int count, int nrhs, double* y,
                       int64_t ylen, int which, cudaStream_t s, LaunchCounter& lc) {
  if (P.ntp == 0) return;
  k_dense_trsv<<<count * nrhs, 256, 0, s>>>(P, vals, nrhs, y, ylen, which);
  lc.n++;
}

void launch_grad(const PlanDev& P, int count, int nrhs, const double* lambda, const double* x,
                 double* ga, cudaStream_t s, LaunchCounter& lc) {
  k_grad<<<dim3(grid1(P.nnz_g, 256, 1024), count), 256, 0, s>>>(P, nrhs, lambda, x, ga);
  lc.n++;
}

}  // namespace glu
