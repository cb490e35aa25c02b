// Allocation-free bounding box: the device form of BoundBox::getBounds (with
// its sequential 1e-5 drift, evaluated in closed form) for callers that must
// not allocate device memory themselves: code embedded in a host application
// or framework that owns all device memory through its own pool (a cudaMalloc
// behind its back breaks its budget and fragments its pool), and latency-bound
// loops that cannot afford cudaMalloc/cudaFree, which synchronize the device.
// Such a caller passes device pointers for the bodies and for the six output
// doubles.  The only other device memory used is a 128-byte file-scope array,
// which every GPU that loads this library holds until the process exits.
//
// Set-up: the first call in each CUDA context looks up the device address of
// that array (cudaGetSymbolAddress) with the context current; make that first
// call before any stream capture.  The address belongs to the context that
// loaded this library's module, so it is remembered per context (by the
// driver's unique context id), not per device ordinal: after cudaDeviceReset,
// or when a host framework makes its own context current, the next call looks
// the address up again.  All calls share the one array, and each call starts
// by clearing it, so calls whose work overlaps on the GPU (different streams,
// or different host threads on the same device) race and must be ordered by
// the caller.
//
// This entry point has no counterpart in the reference.  It runs the same
// two-pass algorithm as the context-based exafmm_get_bounds: an unrounded
// estimate per body, then the exact drift only for bodies whose estimate lies
// within the estimate's error bound of the extreme.
#include <cuda.h>

#include <mutex>
#include <stdexcept>
#include <string>

#include "../../include/exafmm_b200.h"
#include "common.cuh"
#include "drift.cuh"

namespace exafmm_b200 {
namespace {

// [0..5] exact min/max encodings, [6..11] estimate encodings, [12] max |x|.
constexpr int kBoundsScratchWords = 16;
static __device__ __align__(256) unsigned long long g_bounds_scratch[kBoundsScratchWords];

constexpr long long kNoAllocMaxBodies = (1LL << 31) - 1;

std::mutex g_mutex;
// Scratch address per CUDA context, keyed by the driver's context id (unique
// for the life of the process, unlike a context handle, which a new context
// may reuse).  Up to kCtxSlots contexts are remembered; more are looked up on
// every call.
constexpr int kCtxSlots = 64;
struct CtxSlot {
  unsigned long long id;
  unsigned long long *ptr;
};
CtxSlot g_slots[kCtxSlots] = {};
int g_nslots = 0;

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

template <typename F>
F driver_entry(const char *name) {
  void *p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPointByVersion(name, &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !p)
    throw std::runtime_error(std::string("driver entry point not found: ") + name);
  return (F)p;
}

__device__ __forceinline__ unsigned long long enc(double d) {
  unsigned long long u = (unsigned long long)__double_as_longlong(d);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double dec(unsigned long long u) {
  unsigned long long v = (u >> 63) ? (u ^ 0x8000000000000000ull) : ~u;
  return __longlong_as_double((long long)v);
}

__global__ void k_na_clear(unsigned long long *s) {
  const int t = threadIdx.x;
  if (t < kBoundsScratchWords) s[t] = (t < 3 || (t >= 6 && t < 9)) ? ~0ull : 0ull;
}

__global__ void k_na_estimate(const double4 *x, long long n, unsigned long long *s) {
  unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0, 0, 0}, amax = 0;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
    const double4 b = x[j];
    const double v[3] = {b.x, b.y, b.z};
    const double kc = (double)((j == 0) ? n : n - 1 - j) * 1e-5;
    for (int d = 0; d < 3; d++) {
      const unsigned long long a = enc(v[d] - kc), c = enc(v[d] + kc), m = enc(fabs(v[d]));
      lo[d] = a < lo[d] ? a : lo[d];
      hi[d] = c > hi[d] ? c : hi[d];
      amax = m > amax ? m : amax;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    for (int d = 0; d < 3; d++) {
      const unsigned long long a = __shfl_xor_sync(0xffffffffu, lo[d], o);
      const unsigned long long c = __shfl_xor_sync(0xffffffffu, hi[d], o);
      lo[d] = a < lo[d] ? a : lo[d];
      hi[d] = c > hi[d] ? c : hi[d];
    }
    const unsigned long long m = __shfl_xor_sync(0xffffffffu, amax, o);
    amax = m > amax ? m : amax;
  }
  if ((threadIdx.x & 31) == 0) {
    for (int d = 0; d < 3; d++) {
      atomicMin(&s[6 + d], lo[d]);
      atomicMax(&s[9 + d], hi[d]);
    }
    atomicMax(&s[12], amax);
  }
}

__global__ void k_na_exact(const double4 *x, long long n, unsigned long long *s) {
  const double span = dec(s[12]) + (double)n * 1e-5;
  const double B = (double)n * ldexp(1.0, ilogb(span > 1e-300 ? span : 1e-300) - 52) + 1e-300;
  double elo[3], ehi[3];
  for (int d = 0; d < 3; d++) {
    elo[d] = dec(s[6 + d]) + 2.0 * B;
    ehi[d] = dec(s[9 + d]) - 2.0 * B;
  }
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
    const double4 b = x[j];
    const double v[3] = {b.x, b.y, b.z};
    const long long k = (j == 0) ? n : n - 1 - j;
    const double kc = (double)k * 1e-5;
    for (int d = 0; d < 3; d++) {
      if (v[d] - kc <= elo[d]) atomicMin(&s[d], enc(drift_down(v[d], k)));
      if (v[d] + kc >= ehi[d]) atomicMax(&s[3 + d], enc(drift_up(v[d], k)));
    }
  }
}

__global__ void k_na_final(const unsigned long long *s, long long n, double *out) {
  const int t = threadIdx.x;
  if (t < 6) out[t] = (n > 0) ? dec(s[t]) : 0.0;
}

// Device address of the scratch array in the current context, looked up once
// per context.
unsigned long long *scratch_for_current_context() {
  std::lock_guard<std::mutex> lock(g_mutex);
  static CtxGetCurrentFn get_current = driver_entry<CtxGetCurrentFn>("cuCtxGetCurrent");
  static CtxGetIdFn get_id = driver_entry<CtxGetIdFn>("cuCtxGetId");
  auto current_id = [&](unsigned long long *id) {
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS) throw std::runtime_error("cuCtxGetCurrent failed");
    if (!ctx) return false;
    if (get_id(ctx, id) != CUDA_SUCCESS) throw std::runtime_error("cuCtxGetId failed");
    return true;
  };
  unsigned long long id = 0;
  const bool have = current_id(&id);
  if (have)
    for (int k = 0; k < g_nslots; k++)
      if (g_slots[k].id == id) return g_slots[k].ptr;
  // Unknown context, or none current yet: the lookup runs in (and, when none
  // was current, first makes current) the runtime's context for this device.
  unsigned long long *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress((void **)&p, g_bounds_scratch);
  if (e != cudaSuccess || !p)
    throw std::runtime_error(std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
  if ((have || current_id(&id)) && g_nslots < kCtxSlots) g_slots[g_nslots++] = CtxSlot{id, p};
  return p;
}

}  // namespace
}  // namespace exafmm_b200

using namespace exafmm_b200;

extern "C" {

// Status: 0 done (results are ready once `stream` reaches this point),
// 2 n outside [0, 2^31 - 1], 3 null pointer, 4 CUDA error raised by this call
// (context or symbol lookup, or one of its launches), 5 a CUDA error was
// already pending on this thread when the call began (left pending for its
// owner; nothing is launched).
int exafmm_get_bounds_noalloc(const double *d_xyzq, long long n, double *d_bounds6, void *stream) {
  if (n < 0 || n > kNoAllocMaxBodies) return 2;
  if (!d_bounds6 || (n > 0 && !d_xyzq)) return 3;
  if (cudaPeekAtLastError() != cudaSuccess) return 5;
  try {
    cudaStream_t st = (cudaStream_t)stream;
    unsigned long long *s = scratch_for_current_context();
    k_na_clear<<<1, 32, 0, st>>>(s);  // the array keeps the previous call's contents
    EXA_CHECK_LAUNCH();
    if (n > 0) {
      long long g = (n + 255) / 256;
      const int grid = (int)(g > kNumSMs * 16 ? kNumSMs * 16 : g);
      k_na_estimate<<<grid, 256, 0, st>>>((const double4 *)d_xyzq, n, s);
      EXA_CHECK_LAUNCH();
      k_na_exact<<<grid, 256, 0, st>>>((const double4 *)d_xyzq, n, s);
      EXA_CHECK_LAUNCH();
    }
    k_na_final<<<1, 32, 0, st>>>(s, n, d_bounds6);
    EXA_CHECK_LAUNCH();
    return 0;
  } catch (const std::exception &) {
    return 4;
  }
}

}  // extern "C"
