// probes.cu -- hardware-rate measurements used to put the force kernels'
// counters in context (no counterpart in the reference): the FMA rate of the
// device with scalar FP32 chains, packed f32x2 chains and FP64 chains.
// Internal: exported for the benchmark's compute roofline, not part of the
// public header.
//
//   int qgb_fma_rate(int32_t kind, int32_t reps, double* tflops)
//   FMA rate of the current device in TFLOP/s (2 flop per FMA), from 16
//   independent FMA chains per thread over 16 blocks of 256 threads per SM:
//   kind 0 scalar FP32, 1 packed f32x2, 2 FP64; best of reps launches after
//   one warm-up.
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/qlat_b200.h"

namespace qgb
{
void set_last_error(const std::string& msg);
void add_launches(int64_t n);
}  // namespace qgb

namespace
{

constexpr int PROBE_CHAINS = 16;  // independent FMA chains per thread

__global__ void __launch_bounds__(256) k_fma_scalar(float* out, int iters, float a, float b)
{
  float x[PROBE_CHAINS];
#pragma unroll
  for (int j = 0; j < PROBE_CHAINS; ++j) x[j] = threadIdx.x * 1e-3f + j;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < PROBE_CHAINS; ++j) x[j] = fmaf(x[j], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < PROBE_CHAINS; ++j) s += x[j];
  out[(long)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) k_fma_packed(float* out, int iters, float a, float b)
{
  float2 x[PROBE_CHAINS / 2];
  const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
#pragma unroll
  for (int j = 0; j < PROBE_CHAINS / 2; ++j)
    x[j] = make_float2(threadIdx.x * 1e-3f + 2 * j, threadIdx.x * 1e-3f + 2 * j + 1);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < PROBE_CHAINS / 2; ++j) x[j] = __ffma2_rn(x[j], a2, b2);
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < PROBE_CHAINS / 2; ++j) s += x[j].x + x[j].y;
  out[(long)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) k_fma_double(double* out, int iters, double a, double b)
{
  double x[PROBE_CHAINS];
#pragma unroll
  for (int j = 0; j < PROBE_CHAINS; ++j) x[j] = threadIdx.x * 1e-3 + j;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < PROBE_CHAINS; ++j) x[j] = fma(x[j], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < PROBE_CHAINS; ++j) s += x[j];
  out[(long)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

int pfail(int code, const std::string& m)
{
  qgb::set_last_error(m);
  return code;
}

}  // namespace

extern "C" {

int qgb_fma_rate(int32_t kind, int32_t reps, double* tflops);

int qgb_fma_rate(int32_t kind, int32_t reps, double* tflops)
{
  if (!tflops || reps < 1 || kind < 0 || kind > 2) return pfail(QGB_ERR_INVALID_ARG, "qgb_fma_rate: bad argument");
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                 cudaSuccess)
    return pfail(QGB_ERR_NO_DEVICE, "qgb_fma_rate: no CUDA device");
  const int blocks = sms * 16, threads = 256, iters = 4096;
  void* out = nullptr;
  if (cudaMalloc(&out, sizeof(double) * (size_t)blocks * threads) != cudaSuccess)
    return pfail(QGB_ERR_ALLOC, "qgb_fma_rate: cudaMalloc failed");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int r = 0; r <= reps; ++r) {  // the first launch warms up
    cudaEventRecord(e0);
    if (kind == 1) k_fma_packed<<<blocks, threads>>>((float*)out, iters, 0.999f, 1e-3f);
    else if (kind == 2) k_fma_double<<<blocks, threads>>>((double*)out, iters, 0.999, 1e-3);
    else k_fma_scalar<<<blocks, threads>>>((float*)out, iters, 0.999f, 1e-3f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && ms < best) best = ms;
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  qgb::add_launches(reps + 1);
  if (err != cudaSuccess) return pfail(QGB_ERR_CUDA, std::string("qgb_fma_rate: ") + cudaGetErrorString(err));
  const double fmas = (double)blocks * threads * iters * PROBE_CHAINS;
  *tflops = 2.0 * fmas / (best * 1e-3) / 1e12;
  return QGB_OK;
}

}  // extern "C"
