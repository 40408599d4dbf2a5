// Device body of the residual check r = b - op(A) x on the user's ORIGINAL matrix, shared by
// the kernel behind glu_residual / glu_refine (kernels.cu) and the one behind
// glu_residual_noalloc (noalloc.cu), so both entry points run the same arithmetic.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "plan.h"

namespace glu {

// Rows chunk * blockDim.x + threadIdx.x, stepping by nchunks * blockDim.x, of vector v
// (= instance * nrhs + rhs): r = b - op(A) x is written to R (if not null), and the infinity
// norms ||r||, ||x||, ||b||, ||A|| of the vector are folded into norms[4 v .. 4 v + 4) with
// atomicMax on their bit patterns (non-negative doubles order like their bits).  A NaN residual
// counts as infinite.  The whole warp must call this (it reduces with shuffles).
__device__ __forceinline__ void residual_rows(const PlanDev& P, int nrhs,
                                              const double* __restrict__ a,
                                              const double* __restrict__ X,
                                              const double* __restrict__ Bm,
                                              double* __restrict__ R, unsigned long long* norms,
                                              int transpose, int64_t v, int64_t chunk,
                                              int64_t nchunks) {
  const int64_t inst = v / nrhs;
  const double* av = a + inst * P.nnz_g;
  const double* xv = X + v * P.n;
  const double* bv = Bm + v * P.n;
  const int64_t* ptr = transpose ? P.o_col_ptr : P.o_row_ptr;
  const int64_t* ent = transpose ? P.o_col_e : P.o_row_e;
  const uint32_t* other = transpose ? P.g_row : P.g_col;
  double mr = 0.0, mx = 0.0, mb = 0.0, ma = 0.0;
  for (int64_t i = chunk * blockDim.x + threadIdx.x; i < P.n; i += nchunks * blockDim.x) {
    double s = 0.0, arow = 0.0;
    for (int64_t q = ptr[i]; q < ptr[i + 1]; ++q) {
      const int64_t e = ent[q];
      s += av[e] * xv[other[e]];
      arow += fabs(av[e]);
    }
    const double r = bv[i] - s;
    if (R) R[v * P.n + i] = r;
    mr = fmax(mr, fabs(r));
    if (!(r == r)) mr = __longlong_as_double(0x7ff0000000000000LL);   // NaN -> inf
    mx = fmax(mx, fabs(xv[i]));
    mb = fmax(mb, fabs(bv[i]));
    ma = fmax(ma, arow);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mb = fmax(mb, __shfl_xor_sync(0xffffffffu, mb, o));
    ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, o));
  }
  if ((threadIdx.x % 32) == 0) {
    unsigned long long* nv = norms + 4 * v;
    atomicMax(nv + 0, (unsigned long long)__double_as_longlong(mr));
    atomicMax(nv + 1, (unsigned long long)__double_as_longlong(mx));
    atomicMax(nv + 2, (unsigned long long)__double_as_longlong(mb));
    atomicMax(nv + 3, (unsigned long long)__double_as_longlong(ma));
  }
}

// ||r|| / (||A|| ||x|| + ||b||) from the four norms of one vector (||r|| when the denominator
// is zero).
__device__ __forceinline__ double residual_ratio(const unsigned long long* nv) {
  const double r = __longlong_as_double((long long)nv[0]);
  const double x = __longlong_as_double((long long)nv[1]);
  const double b = __longlong_as_double((long long)nv[2]);
  const double A = __longlong_as_double((long long)nv[3]);
  const double den = A * x + b;
  return den > 0.0 ? r / den : r;
}

}  // namespace glu
