// Dense-phase kernels for sm_100a (FP64): the trailing block that fill has made dense.
//
// Per panel step k (width NB):
//   k_dense_diag_rows / k_dense_diag
//                  one CTA per instance factors the NB x NB diagonal block (a row per thread in
//                  registers for NB = 64, 16 x 16 register tiles for NB = 128); per pivot the
//                  reference's column math: pivot (perturbed if |d| < pert and the column has
//                  an L part, src/numeric.cu:139-140), L(:,kk) /= d (src/numeric.cu:37-47), then
//                  the rank-1 update (src/numeric.cu:78-83).
//   k_dense_trsm_mma
//                  L21 = A21 U11^-1 and U12 = L11^-1 A12: 8-column blocks updated by DMMA, 8 x 8
//                  triangles solved one row per lane in the reference's order (k_dense_trsm, a
//                  warp-shuffle recurrence, serves NB = 128).
//   k_gemm_sub / k_gemm_sub16
//                  updates C -= A * B on the FP64 tensor cores (DMMA, mma.sync m8n8k4 or
//                  m16n8k8): accumulators start from -C and collect +A*B, the result is stored
//                  negated, so each output is C - a1*b1 - a2*b2 - ... in one FMA chain (the
//                  reference subtracts the same products one at a time).
// Panels are grouped (launch_dense_factor): inside a group each panel first takes the updates of
// the group's earlier panels, and the rest of the block takes the whole group's update at once.
// Before the first step, the contributions of the sparse columns to the dense block arrive in two
// forms: the few "hub" columns with large L21 x U12 outer products as one DMMA GEMM on gathered
// panels (k_gather + k_gemm_sub), the rest pulled per tail column through shared memory
// (k_dense_pull, which also assembles the block) -- no global atomics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <functional>
#include <map>
#include <mutex>
#include <utility>

#include "glu_b200.h"
#include "kernels.cuh"
#include "plan_host.h"

namespace glu {

namespace {

constexpr int kWarp = 32;

__device__ __forceinline__ void pivot_flags(int32_t* status, int b, double d, bool perturbed) {
  if (d == 0.0) atomicOr(status + b, GLU_INST_ZERO_PIVOT);
  else if (!(fabs(d) <= 1.79769313486231570e308)) atomicOr(status + b, GLU_INST_NAN_PIVOT);
  if (perturbed) atomicOr(status + b, GLU_INST_PERTURBED);
}

// ---------------------------------------------------------------------------------------------
// diagonal block: one CTA (256 threads) per instance
// ---------------------------------------------------------------------------------------------
template <int NB>
__global__ void __launch_bounds__(256) k_dense_diag(DenseView V,
                                                    const double* __restrict__ pert,
                                                    int32_t* status, int k) {
  constexpr int R = NB / 16;
  __shared__ double srow[2][NB];
  __shared__ double scol[2][NB];
  __shared__ double sd[2];
  const int b = blockIdx.x;
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  const int64_t ld = V.ld;
  double* __restrict__ D = V.base + (int64_t)b * V.stride + (int64_t)k + (int64_t)k * ld;
  const double pv = pert[b];
  double a[R][R];   // a[i][j] = A(tx + 16 i, ty + 16 j) of the diagonal block
#pragma unroll
  for (int i = 0; i < R; ++i)
#pragma unroll
    for (int j = 0; j < R; ++j) a[i][j] = D[(tx + 16 * i) + (int64_t)(ty + 16 * j) * ld];

  const int nv = min(NB, V.nvalid - k);         // pivots beyond are identity padding
  for (int kk = 0; kk < nv; ++kk) {
    const int buf = kk & 1;
    if (tx == (kk & 15)) {                       // row kk lives in a[kk/16][*] of these threads
#pragma unroll
      for (int i = 0; i < R; ++i) {
        if (i != (kk >> 4)) continue;
#pragma unroll
        for (int j = 0; j < R; ++j) {
          const int col = ty + 16 * j;
          if (col > kk) srow[buf][col] = a[i][j];
          if (col == kk) {
            const double d0 = a[i][j];
            const bool perturbed = pv > 0.0 && V.hasl[k + kk] && fabs(d0) < pv;
            const double d = perturbed ? pv : d0;
            a[i][j] = d;
            sd[buf] = d;
            pivot_flags(status, b, d, perturbed);
          }
        }
      }
    }
    __syncthreads();
    if (ty == (kk & 15)) {                       // column kk lives in a[*][kk/16]
      const double d = sd[buf];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        if (j != (kk >> 4)) continue;
#pragma unroll
        for (int i = 0; i < R; ++i) {
          const int row = tx + 16 * i;
          if (row > kk) {
            a[i][j] = a[i][j] / d;
            scol[buf][row] = a[i][j];
          }
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int row = tx + 16 * i;
      if (row <= kk) continue;
      const double l = scol[buf][row];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const int col = ty + 16 * j;
        if (col > kk) a[i][j] -= l * srow[buf][col];
      }
    }
  }
#pragma unroll
  for (int i = 0; i < R; ++i)
#pragma unroll
    for (int j = 0; j < R; ++j) D[(tx + 16 * i) + (int64_t)(ty + 16 * j) * ld] = a[i][j];
}

// Pivot step KK of k_dense_diag_rows, instantiated per pivot so that the row stays in registers
// (every index into a[] is a compile-time constant).
template <int KK>
__device__ __forceinline__ void diag_rows_step(double (&a)[64], double (&prow)[2][64], int i,
                                               double pv, const uint8_t* __restrict__ hasl,
                                               int32_t* status, int b, int nv) {
  if constexpr (KK < 64) {
    if (KK >= nv) return;                        // the rest is identity padding
    if constexpr (KK >= 0) {
      if (i > KK) {
        const double* __restrict__ r = prow[KK & 1];
        const double l = a[KK] / r[KK];
        a[KK] = l;
#pragma unroll
        for (int j = KK + 1; j < 64; ++j) a[j] -= l * r[j];
      }
    }
    if constexpr (KK + 1 < 64) {
      if (i == KK + 1) {                         // row KK + 1 is final: pivot and publish it
        const double d0 = a[KK + 1];
        const bool perturbed = pv > 0.0 && hasl[KK + 1] && fabs(d0) < pv;
        const double d = perturbed ? pv : d0;
        a[KK + 1] = d;
        pivot_flags(status, b, d, perturbed);
#pragma unroll
        for (int j = KK + 1; j < 64; ++j) prow[(KK + 1) & 1][j] = a[j];
      }
    }
    __syncthreads();
    diag_rows_step<KK + 1>(a, prow, i, pv, hasl, status, b, nv);
  }
}

// Same factorization of a 64 x 64 diagonal block with one thread per row, the row held in
// registers: per pivot kk every lower row divides by the pivot and applies the rank-1 update with
// the pivot row read from a double-buffered shared copy; the thread owning row kk + 1 -- the last
// writer of the next pivot -- applies the perturbation and publishes its row right away, so one
// barrier per pivot suffices.  Lower latency than the 16 x 16 tiled kernel above, which matters
// when one block sits on the critical path.
__device__ __forceinline__ void diag_rows_body(const DenseView& V, const double* __restrict__ pert,
                                               int32_t* status, int k, int b) {
  constexpr int NB = 64;
  __shared__ __align__(16) double prow[2][NB];
  const int i = threadIdx.x;
  const int64_t ld = V.ld;
  double* __restrict__ D = V.base + (int64_t)b * V.stride + (int64_t)k + (int64_t)k * ld;
  double a[NB];
#pragma unroll
  for (int j = 0; j < NB; ++j) a[j] = D[i + (int64_t)j * ld];
  diag_rows_step<-1>(a, prow, i, pert[b], V.hasl + k, status, b, min(NB, V.nvalid - k));
#pragma unroll
  for (int j = 0; j < NB; ++j) D[i + (int64_t)j * ld] = a[j];
}

__global__ void __launch_bounds__(64) k_dense_diag_rows(DenseView V, const double* __restrict__ pert,
                                                        int32_t* status, int k) {
  diag_rows_body(V, pert, status, k, blockIdx.x);
}

// The dense view of front f's buffer (instances `fstride` doubles apart in F).
__device__ __forceinline__ DenseView front_view(const PlanDev& P, const FrontGeom& g, double* F,
                                                int64_t fstride) {
  return DenseView{F + g.foff, fstride, g.ld, g.ld, g.cols, P.fhasl + g.h_off, g.w};
}

// Diagonal block at pivot k of every front f0 + blockIdx.y of a level (grid (count, fronts)) that
// still has a pivot there; the same body as k_dense_diag_rows.
__global__ void __launch_bounds__(64) k_front_diag(PlanDev P, double* F, int64_t fstride, int f0,
                                                  const double* __restrict__ pert,
                                                  int32_t* status, int k) {
  const FrontGeom g = P.fgeom[f0 + blockIdx.y];
  if (k >= g.w) return;
  diag_rows_body(front_view(P, g, F, fstride), pert, status, k, blockIdx.x);
}

// ---------------------------------------------------------------------------------------------
// L21 / U12 blocks of a panel step: grid (2 * nrb, count), 256 threads (8 warps).
// The factored diagonal block is staged in shared memory once; after that the warps work
// independently (no block-wide barrier inside the recurrences): rows of L21 and columns of U12
// are independent of each other, and within one row (column) the recurrence runs in registers
// with the pivot-column value broadcast by a warp shuffle.
// ---------------------------------------------------------------------------------------------
template <int NB>
__global__ void __launch_bounds__(256) k_dense_trsm(DenseView V, int k, int nrb) {
  constexpr int TS = NB + 1;
  constexpr int C = NB / 32;               // columns (rows) of the block per lane
  extern __shared__ double T[];            // factored diagonal block, T[i + j * TS]
  const int role = blockIdx.x, b = blockIdx.y;
  const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp;
  const int64_t ld = V.ld;
  double* __restrict__ D = V.base + (int64_t)b * V.stride;
  for (int idx = tid; idx < NB * NB; idx += 256) {
    const int i = idx % NB, j = idx / NB;
    T[i + j * TS] = D[(int64_t)(k + i) + (int64_t)(k + j) * ld];
  }
  if (role < nrb) {
    // X * U11 = A21 for 8 rows per warp: lane holds columns lane + 32 c of each row
    double* __restrict__ A = D + (int64_t)(k + NB + role * 64 + warp * 8) + (int64_t)k * ld;
    double x[8][C];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int c = 0; c < C; ++c) x[r][c] = A[r + (int64_t)(lane + 32 * c) * ld];
    __syncthreads();
#pragma unroll 1
    for (int kk = 0; kk < NB; ++kk) {
      const int owner = kk & 31, q = kk >> 5;
      const double d = T[kk + kk * TS];
      double u[C];
#pragma unroll
      for (int c = 0; c < C; ++c) u[c] = T[kk + (lane + 32 * c) * TS];
      // L(r, kk) = A(r, kk) / U(kk, kk): lane r (< 8) fetches row r's value from the owner lane
      // and divides, so each step costs one division sequence per warp
      double mine = 0.0;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        double v = 0.0;
#pragma unroll
        for (int c = 0; c < C; ++c)
          if (c == q) v = x[r][c];
        const double a = __shfl_sync(0xffffffffu, v, owner);
        if (lane == r) mine = a;
      }
      const double quot = mine / d;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const double xk = __shfl_sync(0xffffffffu, quot, r);
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const int col = lane + 32 * c;
          if (col == kk) x[r][c] = xk;
          else if (col > kk) x[r][c] -= xk * u[c];
        }
      }
    }
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int c = 0; c < C; ++c) A[r + (int64_t)(lane + 32 * c) * ld] = x[r][c];
  } else {
    // L11 * Y = A12 (unit diagonal) for 8 columns per warp: lane holds rows lane + 32 c
    double* __restrict__ A =
        D + (int64_t)k + (int64_t)(k + NB + (role - nrb) * 64 + warp * 8) * ld;
    double y[8][C];
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
      for (int c = 0; c < C; ++c) y[j][c] = A[(lane + 32 * c) + (int64_t)j * ld];
    __syncthreads();
#pragma unroll 1
    for (int kk = 0; kk < NB - 1; ++kk) {
      const int owner = kk & 31, q = kk >> 5;
      double l[C];
#pragma unroll
      for (int c = 0; c < C; ++c) l[c] = T[(lane + 32 * c) + kk * TS];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        double v = 0.0;
#pragma unroll
        for (int c = 0; c < C; ++c)
          if (c == q) v = y[j][c];
        const double yk = __shfl_sync(0xffffffffu, v, owner);          // final U(kk, col)
#pragma unroll
        for (int c = 0; c < C; ++c)
          if (lane + 32 * c > kk) y[j][c] -= l[c] * yk;
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
      for (int c = 0; c < C; ++c) A[(lane + 32 * c) + (int64_t)j * ld] = y[j][c];
  }
}

// ---------------------------------------------------------------------------------------------
// DMMA GEMM  C -= A * B  (column-major; M, K even; 16-byte aligned A, B with even lda, ldb)
// ---------------------------------------------------------------------------------------------
template <int BM, int BN, int WM, int WN, int STAGES, int BK_ = 32>
struct Gemm {
  static constexpr int WARPS_M = BM / WM, WARPS_N = BN / WN;
  static constexpr int THREADS = WARPS_M * WARPS_N * kWarp;
  static constexpr int MI = WM / 8, NI = WN / 8;
  static constexpr int BK = BK_;
  static constexpr int AST = BM + 4;         // == 4 (mod 16) doubles: conflict-free fragments
  static constexpr int BST = BK + 4;
  static constexpr int A_STAGE = BK * AST, B_STAGE = BN * BST;
  static constexpr int SMEM = STAGES * (A_STAGE + B_STAGE) * 8;
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
// -x by flipping the sign bit on the integer pipe (keeps the negation off the FP64 pipe)
__device__ __forceinline__ double neg(double x) {
  return __hiloint2double(__double2hiint(x) ^ 0x80000000, __double2loint(x));
}

__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// The trailing update at pivot k of the fronts of a level, as GEMM problems: blockIdx.z =
// front (from f0) * count + instance; M, N, K and the operands come from the front's geometry.
struct FrontGemm {
  const FrontGeom* geom;
  double* F;
  int64_t fstride;
  int f0, count, k;
};

template <int BM, int BN, int WM, int WN, int STAGES, int BK = 32, bool GROUPED = false>
__global__ void __launch_bounds__(Gemm<BM, BN, WM, WN, STAGES, BK>::THREADS)
    k_gemm_sub(int M, int N, int K, const double* A, int lda, const double* B, int ldb, double* C,
               int ldc, int64_t sA, int64_t sB, int64_t sC, FrontGemm fg) {
  using G = Gemm<BM, BN, WM, WN, STAGES, BK>;
  extern __shared__ double sm[];
  double* As = sm;
  double* Bs = sm + STAGES * G::A_STAGE;
  const int z = blockIdx.z;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  if (GROUPED) {
    const FrontGeom g = fg.geom[fg.f0 + z / fg.count];
    const int k = fg.k;
    M = g.ld - k - 64;
    N = g.cols - k - 64;
    K = min(64, g.w - k);                        // pivots past w are identity padding
    if (K <= 0 || m0 >= M || n0 >= N) return;
    double* D = fg.F + (int64_t)(z % fg.count) * fg.fstride + g.foff;
    lda = ldb = ldc = g.ld;
    A = D + (k + 64) + (int64_t)k * g.ld;
    B = D + k + (int64_t)(k + 64) * g.ld;
    C = D + (k + 64) + (int64_t)(k + 64) * g.ld;
  } else {
    A += z * sA;
    B += z * sB;
    C += z * sC;
  }
  const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp;
  const int wm = (warp % G::WARPS_M) * WM, wn = (warp / G::WARPS_M) * WN;

  auto load = [&](int stage, int k0) {
    double* as = As + stage * G::A_STAGE;
    double* bs = Bs + stage * G::B_STAGE;
    for (int idx = tid; idx < G::BK * (BM / 2); idx += G::THREADS) {
      const int kc = idx / (BM / 2), mc = (idx % (BM / 2)) * 2;
      const bool ok = (m0 + mc < M) && (k0 + kc < K);
      const double* src = ok ? A + (int64_t)(m0 + mc) + (int64_t)(k0 + kc) * lda : A;
      cp_async16(as + kc * G::AST + mc, src, ok);
    }
    for (int idx = tid; idx < BN * (G::BK / 2); idx += G::THREADS) {
      const int nc = idx / (G::BK / 2), kc = (idx % (G::BK / 2)) * 2;
      const bool ok = (n0 + nc < N) && (k0 + kc < K);
      const double* src = ok ? B + (int64_t)(k0 + kc) + (int64_t)(n0 + nc) * ldb : B;
      cp_async16(bs + nc * G::BST + kc, src, ok);
    }
  };

  const int nk = (K + G::BK - 1) / G::BK;
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk) load(s, s * G::BK);
    cp_async_commit();
  }
  // accumulators start from -C (the loads above are in flight meanwhile) and collect +A*B, so
  // the stored -acc is C - a1*b1 - a2*b2 - ... with exactly the rounding of subtracting the
  // products one FMA at a time, without negating any operand inside the main loop
  double acc[G::MI][G::NI][2];
#pragma unroll
  for (int mi = 0; mi < G::MI; ++mi) {
    const int row = m0 + wm + mi * 8 + (lane >> 2);
#pragma unroll
    for (int ni = 0; ni < G::NI; ++ni) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int col = n0 + wn + ni * 8 + (lane & 3) * 2 + e;
        acc[mi][ni][e] = (row < M && col < N) ? neg(C[(int64_t)row + (int64_t)col * ldc]) : 0.0;
      }
    }
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    if (kt + STAGES - 1 < nk) load((kt + STAGES - 1) % STAGES, (kt + STAGES - 1) * G::BK);
    cp_async_commit();
    const double* as = As + (kt % STAGES) * G::A_STAGE;
    const double* bs = Bs + (kt % STAGES) * G::B_STAGE;
#pragma unroll
    for (int kk = 0; kk < G::BK; kk += 4) {
      double a[G::MI], bf[G::NI];
#pragma unroll
      for (int mi = 0; mi < G::MI; ++mi)
        a[mi] = as[(kk + (lane & 3)) * G::AST + wm + mi * 8 + (lane >> 2)];
#pragma unroll
      for (int ni = 0; ni < G::NI; ++ni)
        bf[ni] = bs[(wn + ni * 8 + (lane >> 2)) * G::BST + kk + (lane & 3)];
#pragma unroll
      for (int mi = 0; mi < G::MI; ++mi)
#pragma unroll
        for (int ni = 0; ni < G::NI; ++ni) dmma884(acc[mi][ni][0], acc[mi][ni][1], a[mi], bf[ni]);
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int mi = 0; mi < G::MI; ++mi) {
    const int row = m0 + wm + mi * 8 + (lane >> 2);
    if (row >= M) continue;
#pragma unroll
    for (int ni = 0; ni < G::NI; ++ni) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int col = n0 + wn + ni * 8 + (lane & 3) * 2 + e;
        if (col < N) C[(int64_t)row + (int64_t)col * ldc] = neg(acc[mi][ni][e]);
      }
    }
  }
}

// DMMA GEMM on the m16n8k8 FP64 shape (fewer, larger tensor instructions than m8n8k4).
// Fragments (PTX ISA, mma.m16n8k8 .f64): g = lane / 4, t = lane % 4;
//   A 16x8: a0 (g, t), a1 (g+8, t), a2 (g, t+4), a3 (g+8, t+4)
//   B 8x8:  b0 (t, g), b1 (t+4, g)
//   C 16x8: c0 (g, 2t), c1 (g, 2t+1), c2 (g+8, 2t), c3 (g+8, 2t+1)
// CPRE: accumulators start at zero and C is fetched into separate registers while the first
// tiles load, then written as C - acc; otherwise the accumulators start from C.
__device__ __forceinline__ void dmma1688(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

template <int BM, int BN, int WM, int WN, int STAGES, bool CPRE, int BK = 32>
__global__ void __launch_bounds__(Gemm<BM, BN, WM, WN, STAGES, BK>::THREADS)
    k_gemm_sub16(int M, int N, int K, const double* A, int lda, const double* B, int ldb, double* C,
                 int ldc, int64_t sA, int64_t sB, int64_t sC) {
  using G = Gemm<BM, BN, WM, WN, STAGES, BK>;
  constexpr int MI = WM / 16, NI = WN / 8;
  extern __shared__ double sm[];
  double* As = sm;
  double* Bs = sm + STAGES * G::A_STAGE;
  const int z = blockIdx.z;
  A += z * sA;
  B += z * sB;
  C += z * sC;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp % G::WARPS_M) * WM, wn = (warp / G::WARPS_M) * WN;

  auto load = [&](int stage, int k0) {
    double* as = As + stage * G::A_STAGE;
    double* bs = Bs + stage * G::B_STAGE;
    for (int idx = tid; idx < G::BK * (BM / 2); idx += G::THREADS) {
      const int kc = idx / (BM / 2), mc = (idx % (BM / 2)) * 2;
      const bool ok = (m0 + mc < M) && (k0 + kc < K);
      const double* src = ok ? A + (int64_t)(m0 + mc) + (int64_t)(k0 + kc) * lda : A;
      cp_async16(as + kc * G::AST + mc, src, ok);
    }
    for (int idx = tid; idx < BN * (G::BK / 2); idx += G::THREADS) {
      const int nc = idx / (G::BK / 2), kc = (idx % (G::BK / 2)) * 2;
      const bool ok = (n0 + nc < N) && (k0 + kc < K);
      const double* src = ok ? B + (int64_t)(k0 + kc) + (int64_t)(n0 + nc) * ldb : B;
      cp_async16(bs + nc * G::BST + kc, src, ok);
    }
  };

  const int nk = (K + G::BK - 1) / G::BK;
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk) load(s, s * G::BK);
    cp_async_commit();
  }
  double acc[MI][NI][4];
  double cpre[CPRE ? MI : 1][CPRE ? NI : 1][4];
#pragma unroll
  for (int mi = 0; mi < MI; ++mi)
#pragma unroll
    for (int ni = 0; ni < NI; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int row = m0 + wm + mi * 16 + g + (e >> 1) * 8;
        const int col = n0 + wn + ni * 8 + 2 * t + (e & 1);
        const double cv = (row < M && col < N) ? C[(int64_t)row + (int64_t)col * ldc] : 0.0;
        if (CPRE) {
          cpre[CPRE ? mi : 0][CPRE ? ni : 0][e] = cv;
          acc[mi][ni][e] = 0.0;
        } else {
          acc[mi][ni][e] = neg(cv);          // -C + sum A*B, stored negated (see k_gemm_sub)
        }
      }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    if (kt + STAGES - 1 < nk) load((kt + STAGES - 1) % STAGES, (kt + STAGES - 1) * G::BK);
    cp_async_commit();
    const double* as = As + (kt % STAGES) * G::A_STAGE;
    const double* bs = Bs + (kt % STAGES) * G::B_STAGE;
#pragma unroll
    for (int kk = 0; kk < G::BK; kk += 8) {
      double a[MI][4], bf[NI][2];
#pragma unroll
      for (int mi = 0; mi < MI; ++mi) {
        const double* ap = as + (kk + t) * G::AST + wm + mi * 16 + g;
        a[mi][0] = ap[0];
        a[mi][1] = ap[8];
        a[mi][2] = ap[4 * G::AST];
        a[mi][3] = ap[4 * G::AST + 8];
      }
#pragma unroll
      for (int ni = 0; ni < NI; ++ni) {
        const double* bp = bs + (wn + ni * 8 + g) * G::BST + kk + t;
        bf[ni][0] = bp[0];
        bf[ni][1] = bp[4];
      }
#pragma unroll
      for (int mi = 0; mi < MI; ++mi)
#pragma unroll
        for (int ni = 0; ni < NI; ++ni) dmma1688(acc[mi][ni], a[mi], bf[ni]);
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int mi = 0; mi < MI; ++mi)
#pragma unroll
    for (int ni = 0; ni < NI; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int row = m0 + wm + mi * 16 + g + (e >> 1) * 8;
        const int col = n0 + wn + ni * 8 + 2 * t + (e & 1);
        if (row < M && col < N)
          C[(int64_t)row + (int64_t)col * ldc] =
              CPRE ? cpre[CPRE ? mi : 0][CPRE ? ni : 0][e] - acc[mi][ni][e] : neg(acc[mi][ni][e]);
      }
}

// ---------------------------------------------------------------------------------------------
// L21 = A21 U11^-1 and U12 = L11^-1 A12 with most of the work on the FP64 tensor cores.
// Grid (nrt + nct, count): CTAs [0, nrt) take 32 * WARPS rows of L21 each, the rest 32 * WARPS
// columns of U12, handled as rows of U12^T = A12^T L11^-T so both roles share one code path.
// Each warp owns 32 rows and walks the panel's NB columns in blocks of 8:
//   1. the block's columns receive the updates of all earlier blocks in one DMMA pass,
//        X(:, blk) -= X(:, <blk) T(<blk, blk)      (m16n8k8, accumulators start at X(:, blk))
//   2. the 8 x 8 triangle is solved one row per lane in the reference's order: per pivot c of
//      the block, x_c /= u_cc (L21 only: L11 has a unit diagonal), then x_j -= x_c * t_cj for
//      the block's later columns (src/numeric.cu:37-47 and 78-83, restricted to the panel).
//      The quotient comes from the pivot's reciprocal, taken once per CTA, and one FMA
//      correction (Markstein's division: q = x r, e = x - q d, q + e r; Muller et al., Handbook
//      of Floating-Point Arithmetic, 2nd ed., sec. 4.7), within an ulp of x / d and three
//      dependent operations long, which shortens the 64-pivot chain of every row.
// The rows stay in shared memory, column-major per warp and padded so that the MMA fragments
// and the row-per-lane accesses are free of bank conflicts.  After the diagonal block is staged
// the warps never wait for each other.
// ---------------------------------------------------------------------------------------------
template <int NB, int WARPS>
__device__ __forceinline__ void trsm_mma_body(const DenseView& V, int k, int nrt, int bx, int b) {
  constexpr int TS = NB + 4;                 // diagonal block: T(i, j) = T[i + j * TS]
  constexpr int XS = 36;                     // a warp's rows: X(r, c) = X[c * XS + r], r < 32
  constexpr int NBLK = NB / 8;
  extern __shared__ double sm[];
  double* T = sm;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const bool lower = bx < nrt;                // rows of L21; otherwise columns of U12
  const int first = (lower ? bx : bx - nrt) * (WARPS * 32) + warp * 32;
  const int extent = (lower ? V.rows : V.cols) - k - NB;
  const int64_t ld = V.ld;
  double* __restrict__ D = V.base + (int64_t)b * V.stride;
  double* __restrict__ X = sm + NB * TS + warp * (NB * XS);
  double* __restrict__ R = sm + NB * TS + WARPS * (NB * XS);   // reciprocals of the pivots
  // stage with asynchronous copies so that all loads are in flight at once (k, ld and the
  // instance stride are even, so the 16-byte copies of row pairs are aligned)
  for (int idx = tid; idx < NB * NB / 2; idx += WARPS * 32) {
    const int i = (idx % (NB / 2)) * 2, j = idx / (NB / 2);
    cp_async16(T + i + j * TS, D + (int64_t)(k + i) + (int64_t)(k + j) * ld, true);
  }
  // B operand of the block products: U(kk, n) for L21, L^T(kk, n) = L(n, kk) for U12^T
  const int sk = lower ? 1 : TS, sn = lower ? TS : 1;
  if (first < extent) {
    if (lower) {
      const bool ok = first + lane < extent;
      const double* src = ok ? D + (int64_t)(k + NB + first + lane) + (int64_t)k * ld : D;
      for (int c = 0; c < NB; ++c) cp_async8(X + c * XS + lane, ok ? src + (int64_t)c * ld : D, ok);
    } else {
      for (int r = 0; r < 32; ++r) {
        const bool ok = first + r < extent;
        const double* src = ok ? D + (int64_t)k + (int64_t)(k + NB + first + r) * ld : D;
        for (int c = lane; c < NB; c += 32) cp_async8(X + c * XS + r, ok ? src + c : D, ok);
      }
    }
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  if (lower)
    for (int c = tid; c < NB; c += WARPS * 32) R[c] = 1.0 / T[c * (TS + 1)];
  __syncthreads();
  if (first >= extent) return;
  __syncwarp();
  const int nblk = min(NBLK, (V.nvalid - k + 7) / 8);   // blocks past it: padding, stay zero
#pragma unroll 1
  for (int blk = 0; blk < nblk; ++blk) {
    const int c0 = blk * 8;
    if (blk > 0) {
      double acc[2][4];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const double* xp = X + (c0 + 2 * t) * XS + mt * 16 + g;
        acc[mt][0] = xp[0];
        acc[mt][1] = xp[XS];
        acc[mt][2] = xp[8];
        acc[mt][3] = xp[XS + 8];
      }
#pragma unroll 1
      for (int kk = 0; kk < c0; kk += 8) {
        const double bf[2] = {T[(kk + t) * sk + (c0 + g) * sn], T[(kk + t + 4) * sk + (c0 + g) * sn]};
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
          const double* ap = X + (kk + t) * XS + mt * 16 + g;
          const double a[4] = {neg(ap[0]), neg(ap[8]), neg(ap[4 * XS]), neg(ap[4 * XS + 8])};
          dmma1688(acc[mt], a, bf);
        }
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        double* xp = X + (c0 + 2 * t) * XS + mt * 16 + g;
        xp[0] = acc[mt][0];
        xp[XS] = acc[mt][1];
        xp[8] = acc[mt][2];
        xp[XS + 8] = acc[mt][3];
      }
      __syncwarp();
    }
    double x[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = X[(c0 + j) * XS + lane];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      if (lower) {
        const double d = T[(c0 + c) * (TS + 1)], r = R[c0 + c];
        const double q = x[c] * r;
        x[c] = fma(fma(-q, d, x[c]), r, q);
      }
#pragma unroll
      for (int j = c + 1; j < 8; ++j) x[j] -= x[c] * T[(c0 + c) * sk + (c0 + j) * sn];
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) X[(c0 + j) * XS + lane] = x[j];
    __syncwarp();
  }
  if (lower) {
    if (first + lane < extent) {
      double* dst = D + (int64_t)(k + NB + first + lane) + (int64_t)k * ld;
#pragma unroll 16
      for (int c = 0; c < NB; ++c) dst[(int64_t)c * ld] = X[c * XS + lane];
    }
  } else {
#pragma unroll 4
    for (int r = 0; r < 32; ++r) {
      if (first + r >= extent) break;
      double* dst = D + (int64_t)k + (int64_t)(k + NB + first + r) * ld;
#pragma unroll
      for (int c = lane; c < NB; c += 32) dst[c] = X[c * XS + r];
    }
  }
}

template <int NB, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_dense_trsm_mma(DenseView V, int k, int nrt) {
  trsm_mma_body<NB, WARPS>(V, k, nrt, blockIdx.x, blockIdx.y);
}

// L21 / U12 at pivot k of the fronts of a level: grid (most row + column tiles of a front,
// fronts * count); CTAs past their front's tiles, and fronts without a pivot at k, return.
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_front_trsm(PlanDev P, double* F, int64_t fstride,
                                                           int f0, int count, int k) {
  const FrontGeom g = P.fgeom[f0 + blockIdx.y / count];
  const int b = blockIdx.y % count;
  if (k >= g.w) return;
  constexpr int R = WARPS * 32;
  const int nrt = (g.ld - k - 64 + R - 1) / R, nct = (g.cols - k - 64 + R - 1) / R;
  if ((int)blockIdx.x >= nrt + nct) return;
  trsm_mma_body<64, WARPS>(front_view(P, g, F, fstride), k, nrt, blockIdx.x, b);
}

// ---------------------------------------------------------------------------------------------
// sparse-to-dense contributions
// ---------------------------------------------------------------------------------------------
__global__ void k_gather(const int32_t* __restrict__ src, const int32_t* __restrict__ dst,
                         int64_t nent, const double* vals, int64_t blob, double* G,
                         int64_t gstride) {
  const int64_t b = blockIdx.y;
  const double* V = vals + b * blob;
  double* g = G + b * gstride;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nent;
       e += (int64_t)gridDim.x * blockDim.x)
    g[dst[e]] = V[src[e]];
}

// One CTA per (tail column j, instance): D(:,j) is staged in shared memory and every non-hub
// sparse column c with U(c,j) != 0 subtracts L21(:,c) * U(c,j) there.
// ASM (assembly, grid over all ntp columns): for instances whose asm_flag is set, the dense
// block was not cleared before the ingest, so the column is built from scratch -- zeros, the
// entries the ingest wrote (asm_row), 1 on the diagonal of a padding column -- and every column
// of the block, padding included, is written exactly once.  Other instances (values loaded in
// filled-pattern order, block cleared) take the plain pull.
// DET: the pull entries of the column are applied one after another by the whole CTA (the rows
// of one entry are distinct), so every entry of D(:,j) takes its updates in a fixed order.
// split: the CTA pulls only the column's first entries (up to pull_mend); k_dense_pull_extra
// adds the others afterwards.
template <bool SMEM, bool ASM, bool DET = false>
__global__ void __launch_bounds__(256) k_dense_pull(PlanDev P, double* vals,
                                                    const uint8_t* __restrict__ asm_flag,
                                                    int split) {
  extern __shared__ double col[];
  const int jt = blockIdx.x, b = blockIdx.y;
  const int tid = threadIdx.x, lane = tid % kWarp, warp = tid / kWarp;
  double* V = vals + (int64_t)b * P.blob;
  double* Dj = V + P.dbase + (int64_t)jt * P.ntp;
  const bool pulls = jt < (int)P.nt && P.pull_ptr != nullptr;
  const int64_t e0 = pulls ? P.pull_ptr[jt] : 0;
  const int64_t e1 = pulls ? (split ? P.pull_mend[jt] : P.pull_ptr[jt + 1]) : 0;
  const bool build = ASM && asm_flag[b] != 0;
  if (!build && e0 == e1) return;
  // entry warp + nw * i of the column is processed by warp `warp`; lane i fetches its pull
  // bounds and U value now, so these loads overlap the assembly below instead of forming a
  // dependent chain per entry later (entries past 32 per warp are fetched when reached)
  const int nw = blockDim.x / kWarp;
  uint32_t m_lb = 0, m_le = 0;
  double m_u = 0.0;
  if (!DET) {
    const int64_t me = e0 + warp + (int64_t)nw * lane;
    if (me < e1) {
      m_lb = P.pull_lb[me];
      m_le = P.pull_le[me];
      m_u = V[P.pull_uslot[me]];
    }
  }
  double* tgt = Dj;
  if (build) {
    for (uint32_t r = tid; r < P.ntp; r += blockDim.x) col[r] = 0.0;
    __syncthreads();
    for (int32_t e = P.asm_ptr[jt] + tid; e < P.asm_ptr[jt + 1]; e += blockDim.x) {
      const int32_t r = P.asm_row[e];
      col[r] = Dj[r];
    }
    if (jt >= (int)P.nt && tid == 0) col[jt] = 1.0;
    __syncthreads();
    tgt = col;
  } else if (SMEM) {
    for (uint32_t r = tid; r < P.ntp; r += blockDim.x) col[r] = Dj[r];
    __syncthreads();
    tgt = col;
  }
  if (DET) {
    for (int64_t e = e0; e < e1; ++e) {
      const double u = V[P.pull_uslot[e]];
      const uint32_t l1 = P.pull_le[e];
      for (uint32_t p = P.pull_lb[e] + tid; p < l1; p += blockDim.x)
        tgt[P.ri[p] - P.t] += -(V[p] * u);
      __syncthreads();
    }
  } else {
    int i = 0;
    for (int64_t e = e0 + warp; e < e1; e += nw, ++i) {
      double u;
      uint32_t l0, l1;
      if (i < kWarp) {
        u = __shfl_sync(0xffffffffu, m_u, i);
        l0 = __shfl_sync(0xffffffffu, m_lb, i);
        l1 = __shfl_sync(0xffffffffu, m_le, i);
      } else {
        u = V[P.pull_uslot[e]];
        l0 = P.pull_lb[e];
        l1 = P.pull_le[e];
      }
      for (uint32_t p = l0 + lane; p < l1; p += kWarp)
        atomicAdd(tgt + (P.ri[p] - P.t), -(V[p] * u));
    }
  }
  if (SMEM || build) {
    __syncthreads();
    for (uint32_t r = tid; r < P.ntp; r += blockDim.x) Dj[r] = col[r];
  }
}

// The entries of heavy columns past pull_mend, one chunk per CTA (grid (npullx, count)), added
// into the column written by k_dense_pull with global atomics: warps take entries in turn,
// lanes the entry's rows.
__global__ void __launch_bounds__(256) k_dense_pull_extra(PlanDev P, double* vals) {
  const int64_t k = blockIdx.x;
  const int b = blockIdx.y, lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
  double* V = vals + (int64_t)b * P.blob;
  double* Dj = V + P.dbase + (int64_t)P.pull_xcol[k] * P.ntp;
  const int64_t e1 = P.pull_xe[2 * k + 1];
  for (int64_t e = P.pull_xe[2 * k] + warp; e < e1; e += blockDim.x / kWarp) {
    const double u = V[P.pull_uslot[e]];
    const uint32_t l1 = P.pull_le[e];
    for (uint32_t p = P.pull_lb[e] + lane; p < l1; p += kWarp)
      atomicAdd(Dj + (P.ri[p] - P.t), -(V[p] * u));
  }
}

template <int BM, int BN, int WM, int WN, int STAGES, int BK = 32>
void gemm_launch(int M, int N, int K, const double* A, int lda, const double* B, int ldb,
                 double* C, int ldc, int count, int64_t sA, int64_t sB, int64_t sC,
                 cudaStream_t s) {
  using G = Gemm<BM, BN, WM, WN, STAGES, BK>;
  ensure_smem_limit((const void*)k_gemm_sub<BM, BN, WM, WN, STAGES, BK>, G::SMEM);
  dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN, count);
  k_gemm_sub<BM, BN, WM, WN, STAGES, BK><<<grid, G::THREADS, G::SMEM, s>>>(
      M, N, K, A, lda, B, ldb, C, ldc, sA, sB, sC, FrontGemm{});
}

template <int BM, int BN, int WM, int WN, int STAGES, bool CPRE, int BK = 32>
void gemm16_launch(int M, int N, int K, const double* A, int lda, const double* B, int ldb,
                   double* C, int ldc, int count, int64_t sA, int64_t sB, int64_t sC,
                   cudaStream_t s) {
  using G = Gemm<BM, BN, WM, WN, STAGES, BK>;
  ensure_smem_limit((const void*)k_gemm_sub16<BM, BN, WM, WN, STAGES, CPRE, BK>, G::SMEM);
  dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN, count);
  k_gemm_sub16<BM, BN, WM, WN, STAGES, CPRE, BK><<<grid, G::THREADS, G::SMEM, s>>>(
      M, N, K, A, lda, B, ldb, C, ldc, sA, sB, sC);
}

}  // namespace

int gemm_variants() { return 14; }

// cudaFuncSetAttribute acts on the current device only, so the limit is recorded per
// (kernel, device); the table is shared by every thread of the process.  Requests within 1 KB of
// the default 48 KB are raised too, leaving room for the kernel's static shared memory.
void ensure_smem_limit(const void* func, size_t bytes) {
  if (bytes + 1024 <= 48 * 1024) return;
  bytes += 1024;
  int dev = 0;
  cudaGetDevice(&dev);
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> done;
  std::lock_guard<std::mutex> lock(mu);
  size_t& cur = done[{func, dev}];
  if (cur >= bytes) return;
  if (cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) ==
      cudaSuccess)
    cur = bytes;
}

void launch_gemm_sub(int M, int N, int K, const double* A, int lda, const double* B, int ldb,
                     double* C, int ldc, int count, int64_t strideA, int64_t strideB,
                     int64_t strideC, cudaStream_t s, LaunchCounter& lc, int variant) {
  if (M <= 0 || N <= 0 || K <= 0 || count <= 0) return;
  switch (variant) {
    case 1: gemm_launch<64, 64, 32, 32, 3>(M, N, K, A, lda, B, ldb, C, ldc, count, strideA, strideB, strideC, s); break;
    case 2: gemm_launch<128, 64, 32, 32, 3>(M, N, K, A, lda, B, ldb, C, ldc, count, strideA, strideB, strideC, s); break;
    case 3: gemm_launch<64, 128, 32, 32, 3>(M, N, K, A, lda, B, ldb, C, ldc, count, strideA, strideB, strideC, s); break;
    case 4: gemm_launch<128, 128, 64, 32, 3>(M, N, K, A, lda, B, ldb, C, ldc, count, strideA, strideB, strideC, s); break;
    case 5: gemm16_launch<64, 64, 32, 32, 2, false>(M, N, K, A, lda, B, ldb, C, ldc, count, strideA, strideB, strideC, s); break;
    case 6: gemm16_launch<128, 64, 32, 32, 2, false>(M, N, K, A, lda, B, ldb, C, ldc, count, strideA, strideB, strideC, s); break;
    case 7: gemm16_launch<128, 128, 64, 32, 2, false>(M, N, K, A, lda, B, ldb, C, ldc, count, strideA, strideB, strideC, s); break;
    case 8: gemm16_launch<64, 64, 32, 32, 2, true>(M, N, K, A, lda, B, ldb, C, ldc, count, strideA, strideB, strideC, s); break;
    case 9: gemm16_launch<128, 64, 32, 32, 2, true>(M, N, K, A, lda, B, ldb, C, ldc, count, strideA, strideB, strideC, s); break;
    case 10: gemm16_launch<64, 128, 32, 32, 2, false>(M, N, K, A, lda, B, ldb, C, ldc, count, strideA, strideB, strideC, s); break;
    case 11: gemm_launch<64, 64, 32, 32, 3, 16>(M, N, K, A, lda, B, ldb, C, ldc, count, strideA, strideB, strideC, s); break;
    case 12: gemm_launch<64, 64, 32, 32, 2, 16>(M, N, K, A, lda, B, ldb, C, ldc, count, strideA, strideB, strideC, s); break;
    case 13: gemm16_launch<64, 64, 32, 32, 3, false, 16>(M, N, K, A, lda, B, ldb, C, ldc, count, strideA, strideB, strideC, s); break;
    default: gemm_launch<64, 64, 32, 32, 2>(M, N, K, A, lda, B, ldb, C, ldc, count, strideA, strideB, strideC, s); break;
  }
  lc.n++;
}

// multiprocessors of the current device (148 on B200), cached per device
int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cached[dev] = n > 0 ? n : 148;
  }
  return cached[dev];
}

void launch_dense_diag(const DenseView& V, int count, const double* pert, int32_t* status, int k,
                       int nb, cudaStream_t s, LaunchCounter& lc) {
  if (nb == 128) k_dense_diag<128><<<count, 256, 0, s>>>(V, pert, status, k);
  else k_dense_diag_rows<<<count, 64, 0, s>>>(V, pert, status, k);
  lc.n++;
}

void launch_dense_trsm(const DenseView& V, int count, int k, int nb, cudaStream_t s,
                       LaunchCounter& lc) {
  const int nrb = (V.rows - k - nb) / 64;          // 64-row blocks of L21
  const int ncb = (V.cols - k - nb) / 64;          // 64-column blocks of U12
  if (nrb + ncb <= 0) return;
  if (nb == 128) {
    const int smem = 128 * 129 * 8;
    ensure_smem_limit((const void*)k_dense_trsm<128>, smem);
    k_dense_trsm<128><<<dim3(nrb + ncb, count), 256, smem, s>>>(V, k, nrb);
  } else {
    // 128 rows per CTA (4 warps sharing the staged diagonal block), or 32 when that leaves
    // fewer than two CTAs per SM (one instance, short panels)
    constexpr int smem4 = (64 * 68 + 4 * 64 * 36 + 64) * 8, smem1 = (64 * 68 + 64 * 36 + 64) * 8;
    ensure_smem_limit((const void*)k_dense_trsm_mma<64, 4>, smem4);
    ensure_smem_limit((const void*)k_dense_trsm_mma<64, 1>, smem1);
    const int nrt = (V.rows - k - nb + 127) / 128, nct = (V.cols - k - nb + 127) / 128;
    if ((int64_t)(nrt + nct) * count >= 2 * sm_count()) {
      k_dense_trsm_mma<64, 4><<<dim3(nrt + nct, count), 128, smem4, s>>>(V, k, nrt);
    } else {
      const int nr1 = (V.rows - k - nb + 31) / 32, nc1 = (V.cols - k - nb + 31) / 32;
      k_dense_trsm_mma<64, 1><<<dim3(nr1 + nc1, count), 32, smem1, s>>>(V, k, nr1);
    }
  }
  lc.n++;
}

void launch_dense_update(const DenseView& V, int count, int k, int nb, int variant, cudaStream_t s,
                         LaunchCounter& lc) {
  const int m = V.rows - k - nb, n = V.cols - k - nb;
  // pivots at and past nvalid are identity padding: their zero L and U parts add nothing
  const int kv = std::min(nb, V.nvalid - k);
  if (m <= 0 || n <= 0 || kv <= 0) return;
  double* D = V.base;
  const int64_t ld = V.ld;
  launch_gemm_sub(m, n, kv, D + (k + nb) + (int64_t)k * ld, (int)ld, D + k + (int64_t)(k + nb) * ld,
                  (int)ld, D + (k + nb) + (int64_t)(k + nb) * ld, (int)ld, count, V.stride, V.stride,
                  V.stride, s, lc, variant);
}

// Right-looking LU of the first npiv pivots of a batch of dense blocks, in groups of `depth`
// panels: inside a group each panel first takes the updates of the group's earlier panels on
// its own column block and row block (two thin DMMA products), then is factored (diagonal block,
// L21, U12); the rest of the block takes the whole group's update in one product with
// K = depth * nb.  Every entry still receives its updates pivot by pivot in increasing order,
// while the trailing block is read and written once per group instead of once per panel.
// mark(phase, launches_before) is called after each panel (2), each trailing update (3) and each
// pair of thin in-group updates (6).
void launch_dense_factor(const DenseView& V, int count, const double* pert, int32_t* status,
                         int npiv, int nb, int depth, int variant, cudaStream_t s,
                         LaunchCounter& lc, const std::function<void(int, int64_t)>& mark) {
  double* D = V.base;
  const int64_t ld = V.ld;
  for (int k0 = 0; k0 < npiv; k0 += depth * nb) {
    const int dd = std::min(depth, (npiv - k0) / nb);
    for (int j = 0; j < dd; ++j) {
      const int c = k0 + j * nb;
      if (c >= V.nvalid) break;                  // identity padding from here on
      int64_t c0 = lc.n;
      if (j > 0) {
        // column block rows [c, rows) x [c, c + nb) and row block [c, c + nb) x [c + nb, cols)
        // minus the products of the group's factored panels (K = c - k0)
        launch_gemm_sub(V.rows - c, nb, c - k0, D + c + (int64_t)k0 * ld, (int)ld,
                        D + k0 + (int64_t)c * ld, (int)ld, D + c + (int64_t)c * ld, (int)ld,
                        count, V.stride, V.stride, V.stride, s, lc, 12);
        if (V.cols - c - nb > 0)
          launch_gemm_sub(nb, V.cols - c - nb, c - k0, D + c + (int64_t)k0 * ld, (int)ld,
                          D + k0 + (int64_t)(c + nb) * ld, (int)ld, D + c + (int64_t)(c + nb) * ld,
                          (int)ld, count, V.stride, V.stride, V.stride, s, lc, 12);
        mark(6, c0);
        c0 = lc.n;
      }
      launch_dense_diag(V, count, pert, status, c, nb, s, lc);
      launch_dense_trsm(V, count, c, nb, s, lc);
      mark(2, c0);
    }
    const int64_t c0 = lc.n;
    launch_dense_update(V, count, k0, dd * nb, variant, s, lc);
    mark(3, c0);
  }
}


// ---- fronts ----
__global__ void k_front_pad(double* F, int64_t fstride, int ld, int w, int wp) {
  double* f = F + (int64_t)blockIdx.y * fstride;
  for (int kk = w + threadIdx.x; kk < wp; kk += blockDim.x) f[kk + (int64_t)kk * ld] = 1.0;
}

__global__ void k_front_writeback(const int32_t* __restrict__ slot, const int32_t* __restrict__ idx,
                                  int64_t cnt, double* vals, int64_t blob, const double* F,
                                  int64_t fstride) {
  const int64_t b = blockIdx.y;
  double* V = vals + b * blob;
  const double* f = F + b * fstride;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < cnt;
       e += (int64_t)gridDim.x * blockDim.x)
    V[slot[e]] = f[idx[e]];
}

// The front's lower-right block holds -L(R,S) U(S,J): added to its targets.  Fronts and single
// columns of one level can share targets (their common ancestors), hence the atomics.
__global__ void k_front_schur(const int32_t* __restrict__ slot, const int32_t* __restrict__ idx,
                              int64_t cnt, double* vals, int64_t blob, const double* F,
                              int64_t fstride) {
  const int64_t b = blockIdx.y;
  double* V = vals + b * blob;
  const double* f = F + b * fstride;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < cnt;
       e += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(V + slot[e], f[idx[e]]);
}

void launch_front(const PlanDev& P, const FrontDev& f, double* vals, int count, double* F,
                  int64_t fstride, const double* pert, int32_t* status, int nb, int depth,
                  int variant, cudaStream_t s, LaunchCounter& lc) {
  auto grid = [](int64_t n) {
    int64_t g = (n + 255) / 256;
    return (unsigned)(g < 1 ? 1 : (g > 2048 ? 2048 : g));
  };
  // 1. assemble [A(S,S) A(S,J); A(R,S) 0] (padded pivots: identity)
  cudaMemset2DAsync(F, sizeof(double) * fstride, 0, sizeof(double) * f.size, count, s);
  if (f.wp > f.w) {
    k_front_pad<<<dim3(1, count), 64, 0, s>>>(F, fstride, f.ld, f.w, f.wp);
    lc.n++;
  }
  k_gather<<<dim3(grid(f.g_cnt), count), 256, 0, s>>>(P.fg_slot + f.g_off, P.fg_idx + f.g_off,
                                                      f.g_cnt, vals, P.blob, F, fstride);
  lc.n++;
  // 2. its first w pivots with the dense kernels
  DenseView V{F, fstride, f.ld, f.ld, f.wp + f.qp, P.fhasl + f.h_off, f.w};
  launch_dense_factor(V, count, pert, status, f.wp, nb, depth, variant, s, lc,
                      [](int, int64_t) {});
  // 3. factored S columns and U(S, J) back to their slots; Schur complement to the targets
  k_front_writeback<<<dim3(grid(f.g_cnt), count), 256, 0, s>>>(
      P.fg_slot + f.g_off, P.fg_idx + f.g_off, f.g_cnt, vals, P.blob, F, fstride);
  if (f.c_cnt > 0)
    k_front_schur<<<dim3(grid(f.c_cnt), count), 256, 0, s>>>(
        P.fc_slot + f.c_off, P.fc_idx + f.c_off, f.c_cnt, vals, P.blob, F, fstride);
  lc.n += f.c_cnt > 0 ? 2 : 1;
}

// Identity on the padded pivots [w, wp) of every front f0 + blockIdx.x of a level.
__global__ void k_front_pad_level(PlanDev P, double* F, int64_t fstride, int f0) {
  const FrontGeom g = P.fgeom[f0 + blockIdx.x];
  double* f = F + (int64_t)blockIdx.y * fstride + g.foff;
  for (int kk = g.w + threadIdx.x; kk < g.wp; kk += blockDim.x) f[kk + (int64_t)kk * g.ld] = 1.0;
}

bool front_level_batched(const FrontLevel& L, int count, int nb) {
  return nb == 64 && L.nf > 0 && (int64_t)L.nf * count <= 65535;
}

void launch_front_level(const PlanDev& P, const FrontLevel& L, double* vals, int count, double* F,
                        int64_t fstride, const double* pert, int32_t* status, cudaStream_t s,
                        LaunchCounter& lc) {
  auto grid = [](int64_t n) {
    int64_t g = (n + 255) / 256;
    return (unsigned)(g < 1 ? 1 : (g > 2048 ? 2048 : g));
  };
  const int nf = L.nf, nfc = nf * count;
  // 1. assemble every front [A(S,S) A(S,J); A(R,S) 0] of the level (padded pivots: identity)
  cudaMemset2DAsync(F, sizeof(double) * fstride, 0, sizeof(double) * L.area, count, s);
  k_front_pad_level<<<dim3(nf, count), 64, 0, s>>>(P, F, fstride, L.f0);
  k_gather<<<dim3(grid(L.g1 - L.g0), count), 256, 0, s>>>(P.fg_slot + L.g0, P.fg_aidx + L.g0,
                                                          L.g1 - L.g0, vals, P.blob, F, fstride);
  lc.n += 2;
  // 2. their pivots, 64 at a time: diagonal blocks, L21 / U12, trailing update (the same kernels'
  //    bodies as the trailing block's, every front of the level in one launch per stage)
  constexpr int smem4 = (64 * 68 + 4 * 64 * 36 + 64) * 8, smem1 = (64 * 68 + 64 * 36 + 64) * 8;
  ensure_smem_limit((const void*)k_front_trsm<4>, smem4);
  ensure_smem_limit((const void*)k_front_trsm<1>, smem1);
  using G = Gemm<64, 64, 32, 32, 2, 16>;
  ensure_smem_limit((const void*)k_gemm_sub<64, 64, 32, 32, 2, 16, true>, G::SMEM);
  for (size_t i = 0; i < L.mmax.size(); ++i) {
    const int k = 64 * (int)i;
    k_front_diag<<<dim3(count, nf), 64, 0, s>>>(P, F, fstride, L.f0, pert, status, k);
    lc.n++;
    if (L.tiles1[i] > 0) {      // some front has rows below or columns right of this panel
      if ((int64_t)L.tiles4[i] * nfc >= 2 * sm_count())
        k_front_trsm<4><<<dim3(L.tiles4[i], nfc), 128, smem4, s>>>(P, F, fstride, L.f0, count, k);
      else
        k_front_trsm<1><<<dim3(L.tiles1[i], nfc), 32, smem1, s>>>(P, F, fstride, L.f0, count, k);
      lc.n++;
    }
    if (L.mmax[i] > 0 && L.nmax[i] > 0) {
      const FrontGemm fg{P.fgeom, F, fstride, L.f0, count, k};
      dim3 gg((L.mmax[i] + 63) / 64, (L.nmax[i] + 63) / 64, nfc);
      k_gemm_sub<64, 64, 32, 32, 2, 16, true><<<gg, G::THREADS, G::SMEM, s>>>(
          0, 0, 0, nullptr, 0, nullptr, 0, nullptr, 0, 0, 0, 0, fg);
      lc.n++;
    }
  }
  // 3. factored columns and U(S, J) back to their slots; Schur complements to the targets
  k_front_writeback<<<dim3(grid(L.g1 - L.g0), count), 256, 0, s>>>(
      P.fg_slot + L.g0, P.fg_aidx + L.g0, L.g1 - L.g0, vals, P.blob, F, fstride);
  lc.n++;
  if (L.c1 > L.c0) {
    k_front_schur<<<dim3(grid(L.c1 - L.c0), count), 256, 0, s>>>(
        P.fc_slot + L.c0, P.fc_aidx + L.c0, L.c1 - L.c0, vals, P.blob, F, fstride);
    lc.n++;
  }
}

void launch_hub_update(const PlanDev& P, double* vals, int count, double* gbuf, int variant,
                       cudaStream_t s, LaunchCounter& lc) {
  if (P.hubs_p == 0) return;
  const int64_t gl = (int64_t)P.ntp * P.hubs_p;      // G_L: ntp x Hp, G_U: Hp x ntp
  const int64_t gstride = 2 * gl;
  auto grid = [](int64_t n) {
    int64_t g = (n + 255) / 256;
    return (int)(g < 1 ? 1 : (g > 1024 ? 1024 : g));
  };
  k_gather<<<dim3(grid(P.ngl), count), 256, 0, s>>>(P.gl_src, P.gl_dst, P.ngl, vals, P.blob, gbuf,
                                                     gstride);
  k_gather<<<dim3(grid(P.ngu), count), 256, 0, s>>>(P.gu_src, P.gu_dst, P.ngu, vals, P.blob,
                                                     gbuf + gl, gstride);
  lc.n += 2;
  launch_gemm_sub((int)P.ntp, (int)P.ntp, (int)P.hubs_p, gbuf, (int)P.ntp, gbuf + gl, (int)P.hubs_p,
                  vals + P.dbase, (int)P.ntp, count, gstride, gstride, P.blob, s, lc, variant);
}

bool dense_assembly(const PlanDev& P) {
  return P.ntp > 0 && P.asm_ptr != nullptr && (size_t)P.ntp * 8 <= 200 * 1024;
}

template <bool DET>
void dense_pull_launch(const PlanDev& P, double* vals, int count, const uint8_t* asm_flag,
                       cudaStream_t s, LaunchCounter& lc) {
  const size_t smem = (size_t)P.ntp * 8;
  // heavy columns' extra chunks only when the column grid is a few waves (one or a few
  // matrices); with many instances the grid's depth already evens out the columns
  const int split = !DET && P.npullx > 0 && P.pull_mend != nullptr &&
                    (int64_t)P.ntp * count < 32 * (int64_t)sm_count();
  if (dense_assembly(P)) {
    ensure_smem_limit((const void*)k_dense_pull<true, true, DET>, smem);
    k_dense_pull<true, true, DET><<<dim3(P.ntp, count), 256, smem, s>>>(P, vals, asm_flag, split);
    lc.n++;
  } else {
    if (P.npull == 0 || P.nt == 0) return;
    if (smem <= 200 * 1024) {
      ensure_smem_limit((const void*)k_dense_pull<true, false, DET>, smem);
      k_dense_pull<true, false, DET><<<dim3(P.nt, count), 256, smem, s>>>(P, vals, nullptr, split);
    } else {
      k_dense_pull<false, false, DET><<<dim3(P.nt, count), 256, 0, s>>>(P, vals, nullptr, split);
    }
    lc.n++;
  }
  if (split) {
    k_dense_pull_extra<<<dim3((unsigned)P.npullx, count), 256, 0, s>>>(P, vals);
    lc.n++;
  }
}

void launch_dense_pull(const PlanDev& P, double* vals, int count, const uint8_t* asm_flag,
                       bool det, cudaStream_t s, LaunchCounter& lc) {
  if (det) dense_pull_launch<true>(P, vals, count, asm_flag, s, lc);
  else dense_pull_launch<false>(P, vals, count, asm_flag, s, lc);
}

}  // namespace glu
