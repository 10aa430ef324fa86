// Shared device helpers for the amaterasu_b200 engine: complex arithmetic on
// float2/double2, compile-time loops, error plumbing for the C-ABI.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <atomic>
#include <utility>
#include <type_traits>

#include "../../include/ama.h"

namespace ama {

template <typename T> struct Cx;
template <> struct Cx<float> { using type = float2; };
template <> struct Cx<double> { using type = double2; };
template <typename T> using cx_t = typename Cx<T>::type;

template <typename C> __host__ __device__ __forceinline__ C mk(double re, double im) {
  C c; c.x = (decltype(c.x))re; c.y = (decltype(c.y))im; return c;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  C r; r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; return r;
}
template <typename C, typename T> __device__ __forceinline__ C cscale(C a, T s) { a.x *= s; a.y *= s; return a; }

// Compile-time loop: f(std::integral_constant<int, I>) for I = 0..N-1.
template <int... Is, class F>
__device__ __forceinline__ void static_for_impl(std::integer_sequence<int, Is...>, F&& f) {
  (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, class F> __device__ __forceinline__ void static_for(F&& f) {
  if constexpr (N > 0) static_for_impl(std::make_integer_sequence<int, N>{}, f);
}

// Thread-local last-error message for the C-ABI.
void set_error(const std::string& msg);

// Generation of the library's allocations. Every allocation, growth or free of device or
// pinned memory that a kernel or copy may reference (scratch, engine tables, engine option
// changes that swap kernels) bumps it; a cached CUDA graph holds raw pointers and launch
// shapes, so it is replayed only while the generation it was captured in is current.
uint64_t memory_epoch();
void bump_memory_epoch();

// Library state that holds device memory is kept per CUDA device: a process that drives
// several GPUs must never hand one device's buffer to a kernel on another.
constexpr int kMaxDevices = 64;
inline int current_device() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDevices) return -1;
  return d;
}
template <typename T> struct PerDevice {
  T slot[kMaxDevices];
  // The current device's instance, or nullptr when the device id is unusable.
  T* here() {
    const int d = current_device();
    return d < 0 ? nullptr : &slot[d];
  }
};

}  // namespace ama

#define AMA_CUDA_TRY(expr)                                                              \
  do {                                                                                  \
    cudaError_t _e = (expr);                                                            \
    if (_e != cudaSuccess) {                                                            \
      ama::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));               \
      return AMA_ERR_CUDA;                                                              \
    }                                                                                   \
  } while (0)

#define AMA_CHECK_LAUNCH()                                                              \
  do {                                                                                  \
    cudaError_t _e = cudaGetLastError();                                                \
    if (_e != cudaSuccess) {                                                            \
      ama::set_error(std::string("kernel launch: ") + cudaGetErrorString(_e));          \
      return AMA_ERR_CUDA;                                                              \
    }                                                                                   \
  } while (0)

#define AMA_REQUIRE(cond, code, msg)                                                    \
  do {                                                                                  \
    if (!(cond)) { ama::set_error(msg); return (code); }                                \
  } while (0)
