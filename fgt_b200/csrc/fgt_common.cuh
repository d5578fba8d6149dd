// Common definitions of the B200 point fast Gauss transform library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/fgt_b200.h"

#define FGT_MAXDIM 3

// Status codes (mirrored in include/fgt_b200.h as FGT_* macros).
namespace fgt {

struct Error {
  int code;
  const char* what;
};

}  // namespace fgt

#define FGT_CUDA(call)                                                         \
  do {                                                                         \
    cudaError_t _e = (call);                                                   \
    if (_e != cudaSuccess) {                                                   \
      fgt_set_error_message(cudaGetErrorString(_e), __FILE__, __LINE__);       \
      throw fgt::Error{FGT_ERR_CUDA, cudaGetErrorString(_e)};                  \
    }                                                                          \
  } while (0)

#define FGT_LAUNCH_CHECK() FGT_CUDA(cudaGetLastError())

#define FGT_REQUIRE(cond, code, msg)                                           \
  do {                                                                         \
    if (!(cond)) {                                                             \
      fgt_set_error_message(msg, __FILE__, __LINE__);                          \
      throw fgt::Error{code, msg};                                             \
    }                                                                          \
  } while (0)

extern "C" void fgt_set_error_message(const char* msg, const char* file, int line);

// Device bounds checks of the FGT_CHECK build (the stand-in for a memory
// checker): FGT_DCHECK(cond, site) is true when cond holds; otherwise it
// records `site` in the module's check word (first failure wins) and is
// false, so the caller skips the access.  Never traps.  The host reads and
// clears every module's word at the end of a call (check_sites) and fails the
// call with FGT_ERR_CHECK.  In the normal build the macro is the constant
// true and costs nothing.
namespace fgt {
using CheckReader = unsigned (*)(cudaStream_t);
void register_check_reader(CheckReader r);
// First failed check site of any module since the last call (0 = none);
// clears the words.  Synchronises the stream.
unsigned check_sites(cudaStream_t s);
}  // namespace fgt
#ifdef FGT_CHECK
namespace fgt {
namespace {
__device__ unsigned int g_check_site;
unsigned read_check_site(cudaStream_t s) {
  unsigned v = 0, z = 0;
  if (cudaMemcpyFromSymbolAsync(&v, g_check_site, sizeof(v), 0, cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0xffffffffu;
  }
  if (v && cudaMemcpyToSymbolAsync(g_check_site, &z, sizeof(z), 0, cudaMemcpyHostToDevice, s) !=
               cudaSuccess)
    (void)cudaGetLastError();
  return v;
}
struct CheckRegistrar {
  CheckRegistrar() { register_check_reader(read_check_site); }
};
CheckRegistrar check_registrar;
}  // namespace
}  // namespace fgt
#define FGT_DCHECK(cond, site) \
  ((cond) || (atomicCAS(&fgt::g_check_site, 0u, (unsigned)(site)), false))
#else
#define FGT_DCHECK(cond, site) (true)
#endif

namespace fgt {

constexpr int kSMs = 148;

static inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }
static inline int grid_for(long long n, int block, int per_sm = 16) {
  long long g = (n + block - 1) / block;
  long long cap = (long long)kSMs * per_sm;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

// Device helpers -----------------------------------------------------------

__device__ __forceinline__ float fgt_ex2(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

template <typename T>
struct Real;
template <>
struct Real<float> {
  // exp(-u) for u >= 0 via the hardware base-2 exponential.
  static __device__ __forceinline__ float expm(float u) { return fgt_ex2(-u * 1.4426950408889634f); }
  static __device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
  static __device__ __forceinline__ float rsqrt_(float x) { return rsqrtf(x); }
  // a / b for b in [1, 2] (2 ulp)
  static __device__ __forceinline__ float div12(float a, float b) { return __fdividef(a, b); }
};
template <>
struct Real<double> {
  static __device__ __forceinline__ double expm(double u) { return exp(-u); }
  static __device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
  static __device__ __forceinline__ double rsqrt_(double x) { return 1.0 / sqrt(x); }
  static __device__ __forceinline__ double div12(double a, double b) { return a / b; }
};

// Morton-style path keys: the digit of level l (child index, bit k set iff
// coordinate k lies on the + side) occupies bits [dim*(D-1-l), dim*(D-l)).
__device__ __forceinline__ uint64_t key_prefix(uint64_t key, int dim, int D, int l) {
  int sh = dim * (D - l);
  return sh >= 64 ? 0ull : (key >> sh);
}

}  // namespace fgt
