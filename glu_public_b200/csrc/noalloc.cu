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
// That first call therefore does set-up work and should come before any stream capture.  The
// address is kept for the life of the process: cudaDeviceReset while the library is loaded is not
// supported (the module would be loaded again, possibly elsewhere, and the kept address would be
// stale).
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "glu_b200.h"
#include "internal.h"
#include "plan.h"
#include "residual.cuh"

// Opaque handle layout needed here: the plan/batch structs are defined in api.cu; the accessor
// below (defined there) returns what this file needs without exposing the structs.
namespace glu {
int batch_residual_view(glu_batch_t b, const PlanDev** P, int* count, int* device, int* has_pattern);
}

namespace {

constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned long long g_norm_scratch[4 * GLU_NOALLOC_MAX_VECTORS];

std::mutex g_mu;
unsigned long long* g_scratch_addr[kMaxDevices] = {};

// The residual kernel of glu_residual with its vectors folded into gridDim.x (block x covers
// rows chunk x % nchunks of vector x / nchunks), so every count up to
// GLU_NOALLOC_MAX_VECTORS fits in one launch; same device body (residual.cuh).
__global__ void k_residual_noalloc(glu::PlanDev P, int nrhs, const double* __restrict__ a,
                                   const double* __restrict__ X, const double* __restrict__ Bm,
                                   unsigned long long* norms, int transpose, int nchunks) {
  glu::residual_rows(P, nrhs, a, X, Bm, nullptr, norms, transpose, blockIdx.x / nchunks,
                     blockIdx.x % nchunks, nchunks);
}

__global__ void k_resid_finish_noalloc(int64_t nv, const unsigned long long* norms, double* out) {
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (v < nv) out[v] = glu::residual_ratio(norms + 4 * v);
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
  if (nv > GLU_NOALLOC_MAX_VECTORS)
    return glu::set_error(GLU_BUDGET_EXCEEDED,
                          "glu_residual_noalloc handles at most %d (instance, rhs) vectors; "
                          "this call has %lld",
                          GLU_NOALLOC_MAX_VECTORS, (long long)nv);
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != device) cudaSetDevice(device);
  cudaGetLastError();             // report this call's launch errors, not an earlier call's
  unsigned long long* norms = nullptr;
  st = scratch_address(device, &norms);
  if (st == GLU_OK) {
    cudaStream_t s = (cudaStream_t)stream;
    // the norms are maxima of non-negative values: they must start at zero on every call
    cudaMemsetAsync(norms, 0, sizeof(unsigned long long) * 4 * nv, s);
    // row chunks per vector: at most 64, and at most 64 * 65,536 blocks in all
    int64_t g = (P->n + 255) / 256;
    if (g > 64) g = 64;
    if (g < 1) g = 1;
    k_residual_noalloc<<<(unsigned)(g * nv), 256, 0, s>>>(*P, nrhs, a_dev, X_dev, B_dev, norms,
                                                          transpose, (int)g);
    k_resid_finish_noalloc<<<(unsigned)((nv + 127) / 128), 128, 0, s>>>(nv, norms, resid_dev);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
      st = glu::set_error(GLU_CUDA_ERROR, "residual (no-alloc) launch: %s", cudaGetErrorString(e));
  }
  if (prev >= 0 && prev != device) cudaSetDevice(prev);
  return st;
}
