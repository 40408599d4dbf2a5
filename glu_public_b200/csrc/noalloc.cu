// Allocation-free residual check (glu_residual_noalloc).
//
// Who needs it: a circuit simulator's Newton or transient loop often runs with every byte of
// device memory already handed to its own pool, or inside a real-time section where a
// cudaMalloc (which can synchronize the whole device) is not allowed.  Such a caller still wants
// to test each solve against the residual bound between iterations.  glu_residual needs a small
// per-vector scratch buffer and allocates it lazily; this variant keeps that scratch in a
// fixed-size array in the library's static device memory instead, so it never allocates.
//
// The scratch is the array g_norm_scratch below: 4 norms (as non-negative double bit patterns)
// for each of at most GLU_NOALLOC_MAX_VECTORS (instance, right-hand side) vectors, 2 MiB.
// Every GPU that loads the library keeps these 2 MiB until the process exits.  All calls share
// the one array; each call clears the part it uses before its kernel runs, so calls that run
// one after another are independent, but calls whose work overlaps on the GPU (different
// streams, no ordering between them) race on the array and must not be issued.
//
// Host code must not pass g_norm_scratch itself to a kernel: in host code that name is only a
// stand-in for the device array.  The device address is looked up once per device with
// cudaGetSymbolAddress, with that device current, the first time the entry point runs there.
// That first call therefore does set-up work and should come before any stream capture.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "glu_b200.h"
#include "internal.h"
#include "plan.h"

// Opaque handle layout needed here: the plan/batch structs are defined in api.cu; the accessor
// below (defined there) returns what this file needs without exposing the structs.
namespace glu {
int batch_residual_view(glu_batch_t b, const PlanDev** P, int* count, int* device, int* has_pattern);
}

namespace {

constexpr int kWarp = 32;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned long long g_norm_scratch[4 * GLU_NOALLOC_MAX_VECTORS];

std::mutex g_mu;
unsigned long long* g_scratch_addr[kMaxDevices] = {};

// Same computation as the residual kernel behind glu_residual: r = b - op(A) x on the original
// matrix, with the infinity norms of r, x, b and A per vector accumulated in `norms`.
__global__ void k_residual_noalloc(glu::PlanDev P, int nrhs, const double* __restrict__ a,
                                   const double* __restrict__ X, const double* __restrict__ Bm,
                                   unsigned long long* norms, int transpose) {
  const int64_t v = blockIdx.y;
  const int64_t inst = v / nrhs;
  const double* av = a + inst * P.nnz_g;
  const double* xv = X + v * P.n;
  const double* bv = Bm + v * P.n;
  const int64_t* ptr = transpose ? P.o_col_ptr : P.o_row_ptr;
  const int64_t* ent = transpose ? P.o_col_e : P.o_row_e;
  const uint32_t* other = transpose ? P.g_row : P.g_col;
  double mr = 0.0, mx = 0.0, mb = 0.0, ma = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < P.n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0, arow = 0.0;
    for (int64_t q = ptr[i]; q < ptr[i + 1]; ++q) {
      const int64_t e = ent[q];
      s += av[e] * xv[other[e]];
      arow += fabs(av[e]);
    }
    const double r = bv[i] - s;
    mr = fmax(mr, fabs(r));
    if (!(r == r)) mr = __longlong_as_double(0x7ff0000000000000LL);
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
  if ((threadIdx.x % kWarp) == 0) {
    unsigned long long* nv = norms + 4 * v;
    atomicMax(nv + 0, (unsigned long long)__double_as_longlong(mr));
    atomicMax(nv + 1, (unsigned long long)__double_as_longlong(mx));
    atomicMax(nv + 2, (unsigned long long)__double_as_longlong(mb));
    atomicMax(nv + 3, (unsigned long long)__double_as_longlong(ma));
  }
}

__global__ void k_resid_finish_noalloc(int64_t nv, const unsigned long long* norms, double* out) {
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const double r = __longlong_as_double((long long)norms[4 * v + 0]);
  const double x = __longlong_as_double((long long)norms[4 * v + 1]);
  const double b = __longlong_as_double((long long)norms[4 * v + 2]);
  const double A = __longlong_as_double((long long)norms[4 * v + 3]);
  const double den = A * x + b;
  out[v] = den > 0.0 ? r / den : r;
}

// Device address of g_norm_scratch on `device` (which must be current), looked up once.
int scratch_address(int device, unsigned long long** out) {
  if (device < 0 || device >= kMaxDevices)
    return glu::set_error(GLU_ARGUMENT_ERROR, "device ordinal %d out of range", device);
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_norm_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return glu::set_error(GLU_CUDA_ERROR, "cudaGetSymbolAddress of the residual scratch: %s",
                            cudaGetErrorString(e));
    }
    g_scratch_addr[device] = static_cast<unsigned long long*>(p);
  }
  *out = g_scratch_addr[device];
  return GLU_OK;
}

}  // namespace

extern "C" int glu_residual_noalloc(glu_batch_t b, int32_t nrhs, const double* a_dev,
                                    const double* B_dev, const double* X_dev, int transpose,
                                    double* resid_dev, void* stream) {
  if (!b || !a_dev || !B_dev || !X_dev || !resid_dev || nrhs <= 0)
    return glu::set_error(GLU_ARGUMENT_ERROR, "bad argument");
  const glu::PlanDev* P = nullptr;
  int count = 0, device = 0, has_pattern = 0;
  int st = glu::batch_residual_view(b, &P, &count, &device, &has_pattern);
  if (st) return st;
  if (!has_pattern) return glu::set_error(GLU_NOT_READY, "no original pattern");
  const int64_t nv = (int64_t)count * nrhs;
  if (nv > GLU_NOALLOC_MAX_VECTORS || nv > 65535)
    return glu::set_error(GLU_BUDGET_EXCEEDED,
                          "glu_residual_noalloc handles at most %d (instance, rhs) vectors; "
                          "this call has %lld",
                          GLU_NOALLOC_MAX_VECTORS < 65535 ? GLU_NOALLOC_MAX_VECTORS : 65535,
                          (long long)nv);
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != device) cudaSetDevice(device);
  unsigned long long* norms = nullptr;
  st = scratch_address(device, &norms);
  if (st == GLU_OK) {
    cudaStream_t s = (cudaStream_t)stream;
    // the norms are maxima of non-negative values: they must start at zero on every call
    cudaMemsetAsync(norms, 0, sizeof(unsigned long long) * 4 * nv, s);
    int64_t g = (P->n + 255) / 256;
    if (g > 64) g = 64;
    if (g < 1) g = 1;
    k_residual_noalloc<<<dim3((unsigned)g, (unsigned)nv), 256, 0, s>>>(*P, nrhs, a_dev, X_dev,
                                                                      B_dev, norms, transpose);
    k_resid_finish_noalloc<<<(unsigned)((nv + 127) / 128), 128, 0, s>>>(nv, norms, resid_dev);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
      st = glu::set_error(GLU_CUDA_ERROR, "residual (no-alloc) launch: %s", cudaGetErrorString(e));
  }
  if (prev >= 0 && prev != device) cudaSetDevice(prev);
  return st;
}
