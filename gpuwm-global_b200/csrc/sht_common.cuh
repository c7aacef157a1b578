// Shared definitions for the b200sht CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "b200sht.h"

namespace sht {

// ---------------------------------------------------------------- errors
void set_error(const std::string& msg);
void clear_error();

struct Error {
  int code;
  std::string msg;
};

#define SHT_CUDA_OR_THROW(expr)                                                    \
  do {                                                                             \
    cudaError_t e_ = (expr);                                                       \
    if (e_ != cudaSuccess)                                                         \
      throw ::sht::Error{SHT_ERR_CUDA, std::string(#expr) + ": " +                 \
                                           cudaGetErrorString(e_)};               \
  } while (0)

#define SHT_REQUIRE(cond, msg)                                                     \
  do {                                                                             \
    if (!(cond)) throw ::sht::Error{SHT_ERR_ARG, (msg)};                           \
  } while (0)

// ------------------------------------------------------------ constants
constexpr double kPi = 3.14159265358979323846;

// Device error word bits (set by kernels whose bounded waits expire).
constexpr unsigned kErrMbarTimeout = 1u;
constexpr unsigned kErrBadTile = 2u;

inline int64_t div_up(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Host -> device copy of bookkeeping (tile lists, descriptors, operator
// matrices) that has landed on the device when it returns.  cudaMemcpy from
// pageable memory may return while its DMA is still queued on the legacy
// stream, and kernels launched on non-blocking streams (the host-streamed
// calls, CUDA graphs, other libraries' streams) are not ordered after it, so
// a first launch could read the buffer before it is written.  Not for use
// during stream capture.
inline void upload_now(void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return;
  SHT_CUDA_OR_THROW(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
  SHT_CUDA_OR_THROW(cudaDeviceSynchronize());
}
inline int64_t round_up(int64_t a, int64_t b) { return div_up(a, b) * b; }

// Number of degrees n in [m, T] with (n - m) % 2 == q.
__host__ __device__ inline int parity_count(int T, int m, int q) {
  int span = T - m - q;
  return span < 0 ? 0 : span / 2 + 1;
}

// ----------------------------------------------------- complex helpers
template <typename T> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };

template <typename T>
__device__ __forceinline__ typename Vec2<T>::type mk2(T a, T b) {
  typename Vec2<T>::type v;
  v.x = a;
  v.y = b;
  return v;
}

}  // namespace sht
