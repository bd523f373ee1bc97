// Shared device helpers: complex arithmetic on float2 / double2, error reporting.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

namespace dcaacc {

// Raised inside the library and turned into a dcaacc_status at the C boundary.
struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

// Error-path tests: makes the nth device or pinned-host buffer allocation from now on fail as if
// memory were exhausted (0 turns it off).  Process-wide; defined in api.cpp.
void setAllocationFailure(long nth);
// Called before each buffer allocation: throws Error(DCAACC_OOM) on the chosen one.
void allocationHook();

#define DCAACC_CUDA_CHECK(expr)                                                               \
  do {                                                                                        \
    cudaError_t _e = (expr);                                                                  \
    if (_e != cudaSuccess)                                                                    \
      throw ::dcaacc::Error(_e == cudaErrorMemoryAllocation ? 3 : 4,                          \
                            std::string(#expr) + ": " + cudaGetErrorString(_e));              \
  } while (0)

#define DCAACC_LAUNCH_CHECK()                                                                 \
  do {                                                                                        \
    cudaError_t _e = cudaPeekAtLastError();                                                   \
    if (_e != cudaSuccess)                                                                    \
      throw ::dcaacc::Error(4, std::string("kernel launch failed: ") + cudaGetErrorString(_e)); \
  } while (0)

// ---- complex helpers ----------------------------------------------------------------------------
template <typename Real>
struct Cplx;
template <>
struct Cplx<double> {
  using type = double2;
};
template <>
struct Cplx<float> {
  using type = float2;
};
template <typename Real>
using cplx_t = typename Cplx<Real>::type;

__host__ __device__ inline double2 mk(double r, double i) {
  return make_double2(r, i);
}
__host__ __device__ inline float2 mk(float r, float i) {
  return make_float2(r, i);
}

template <typename C>
__host__ __device__ inline C cadd(C a, C b) {
  return mk(a.x + b.x, a.y + b.y);
}
template <typename C>
__host__ __device__ inline C csub(C a, C b) {
  return mk(a.x - b.x, a.y - b.y);
}
template <typename C>
__host__ __device__ inline C cmul(C a, C b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C>
__host__ __device__ inline C cmulc(C a, C b) {
  return mk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C, typename R>
__host__ __device__ inline C cscale(C a, R s) {
  return mk(a.x * s, a.y * s);
}
// acc += a * b
template <typename C>
__host__ __device__ inline void cfma(C& acc, C a, C b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// acc += a * conj(b)
template <typename C>
__host__ __device__ inline void cfmac(C& acc, C a, C b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.y, b.x, acc.y);
  acc.y = fma(-a.x, b.y, acc.y);
}

__device__ inline float2 to_f2(double2 a) {
  return make_float2(static_cast<float>(a.x), static_cast<float>(a.y));
}

inline int ceil_div(long a, long b) {
  return static_cast<int>((a + b - 1) / b);
}

}  // namespace dcaacc
