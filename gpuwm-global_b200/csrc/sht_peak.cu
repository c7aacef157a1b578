// sht_measure_fp32_peak: the FP32 FFMA rate of the current device, measured.
//
// The plain FP32 Legendre contraction is bound by the FFMA pipes, so its
// roofline needs an FFMA peak, measured on the same GPU and clocks as the
// contraction: a grid of two 512-thread CTAs per SM runs long chains of
// independent fmaf() on registers (eight chains per thread, sixteen steps per
// loop trip, no memory traffic), timed with CUDA events on the caller's
// stream after one warm-up launch.  No clock, power or other device setting
// is touched.
#include "sht_plan.h"

namespace {

constexpr int kChains = 8;
constexpr int kUnroll = 16;
constexpr int kThreads = 512;

__global__ void __launch_bounds__(kThreads) ffma_loop_kernel(float* sink, int trips, float b,
                                                            float c) {
  float acc[kChains];
#pragma unroll
  for (int j = 0; j < kChains; ++j) acc[j] = (float)(threadIdx.x + j) * 1e-3f;
#pragma unroll 1
  for (int t = 0; t < trips; ++t) {
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
#pragma unroll
      for (int j = 0; j < kChains; ++j) acc[j] = fmaf(acc[j], b, c);
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < kChains; ++j) s += acc[j];
  // b and c keep every chain bounded (each converges to c / (1 - b)); the
  // store is never taken for them but keeps the chains live.
  if (sink != nullptr && s == 1234.5f) sink[blockIdx.x * kThreads + threadIdx.x] = s;
}

}  // namespace

int sht_measure_fp32_peak(void* stream, double* tflops) {
  try {
    sht::clear_error();
    SHT_REQUIRE(tflops != nullptr, "tflops must not be NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0, sms = 0;
    SHT_CUDA_OR_THROW(cudaGetDevice(&dev));
    SHT_CUDA_OR_THROW(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int grid = 2 * sms;
    const int trips = 20000;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    SHT_CUDA_OR_THROW(cudaEventCreate(&e0));
    SHT_CUDA_OR_THROW(cudaEventCreate(&e1));
    float ms = 0.f;
    cudaError_t err = cudaSuccess;
    // Warm-up, then the timed launch.
    ffma_loop_kernel<<<grid, kThreads, 0, s>>>(nullptr, trips / 10, 0.999f, 1e-4f);
    err = cudaGetLastError();
    if (err == cudaSuccess) err = cudaEventRecord(e0, s);
    if (err == cudaSuccess) {
      ffma_loop_kernel<<<grid, kThreads, 0, s>>>(nullptr, trips, 0.999f, 1e-4f);
      err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaEventRecord(e1, s);
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    SHT_CUDA_OR_THROW(err);
    SHT_REQUIRE(ms > 0.f, "FFMA loop timed at zero");
    const double flops = 2.0 * kChains * kUnroll * (double)trips * grid * kThreads;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return SHT_OK;
  } catch (const sht::Error& e) {
    sht::set_error(e.msg);
    return e.code;
  }
}
