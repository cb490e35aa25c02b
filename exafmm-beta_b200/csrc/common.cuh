// Shared device/host helpers for the B200 Laplace FMM engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

namespace exafmm_b200 {

// Deepest octree level the 63-bit octant keys can hold (3 bits per level).
constexpr int kMaxLevels = 21;
// Largest expansion order the device kernels are built for.
constexpr int kMaxP = 20;
// Persistent-grid sizing: 148 SMs on B200.
constexpr int kNumSMs = 148;

struct Error {
  int code;
  std::string msg;
};

// Throws a C++ exception carrying the CUDA error text; the C-ABI layer turns it
// into a status code and a last-error string.
void throw_cuda(cudaError_t e, const char *what, const char *file, int line);
void throw_msg(const char *msg);

#define EXA_CUDA(call)                                                       \
  do {                                                                       \
    cudaError_t _e = (call);                                                 \
    if (_e != cudaSuccess) ::exafmm_b200::throw_cuda(_e, #call, __FILE__, __LINE__); \
  } while (0)

// Process-wide count of kernel launches issued by this library.
void note_launch();
long long launch_count();

// Follows every kernel launch (exactly one per launch, so the count is exact).
#define EXA_CHECK_LAUNCH()                \
  do {                                    \
    ::exafmm_b200::note_launch();         \
    EXA_CUDA(cudaGetLastError());         \
  } while (0)

// ---- complex arithmetic on double2 / float2 (x = re, y = im) ----
template <typename T> struct cplx_t;
template <> struct cplx_t<double> { using type = double2; };
template <> struct cplx_t<float> { using type = float2; };

__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

__host__ __device__ __forceinline__ int tri(int n) { return n * (n + 1) / 2; }

// Error flags raised by device code and read once per solve on the host.
enum DeviceError : int {
  kErrNone = 0,
  kErrTreeTooDeep = 1,       // a node at the deepest key level still holds > ncrit bodies
  kErrQueueOverflow = 2,     // traversal pair queue exceeded its capacity
  kErrListOverflow = 4,      // an interaction list exceeded its capacity
  kErrCellOverflow = 8,      // more cells than the cell buffers hold
  kErrMmaTimeout = 16,       // a tensor-core product did not signal completion in time
};

inline int div_up(long long a, long long b) { return int((a + b - 1) / b); }

}  // namespace exafmm_b200
