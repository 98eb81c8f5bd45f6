// Measurement helpers for the benchmark: the FP64 peak of this GPU, measured
// with a throughput kernel (no vendor figure for FP64 is assumed); and a
// batched evaluation of the controllers' pow (kpp_ratelaws.cuh's kpp_pow_cr)
// beside the CUDA math library's, for their tests.
//
//   kind 0: fused multiply-add (DFMA), 2 flops per instruction
//   kind 1: separate multiply and add (DMUL + DADD), 1 flop per instruction;
//           this is the instruction mix of the Rosenbrock kernels, which are
//           built without FMA contraction
#include <cuda_runtime.h>

#include <cstdio>

#include "kpp_ratelaws.cuh"

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) fp64_fma_kernel(double* out, int iters, double b, double c) {
  double acc[kChains];
#pragma unroll
  for (int i = 0; i < kChains; i++) acc[i] = threadIdx.x * 1e-3 + i;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < kChains; i++) acc[i] = __fma_rn(acc[i], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < kChains; i++) s += acc[i];
  if (s == 12345.678) out[0] = s;  // keeps the chains alive
}

__global__ void __launch_bounds__(256) fp64_muladd_kernel(double* out, int iters, double b, double c) {
  double acc[kChains];
#pragma unroll
  for (int i = 0; i < kChains; i++) acc[i] = threadIdx.x * 1e-3 + i;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < kChains; i++) acc[i] = __dadd_rn(__dmul_rn(acc[i], b), c);
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < kChains; i++) s += acc[i];
  if (s == 12345.678) out[0] = s;
}

__global__ void __launch_bounds__(256) pow_kernel(long long n, const double* x, const double* y,
                                                  double* out, int which) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = which == 0 ? kpp_pow_cr(x[i], y[i]) : pow(x[i], y[i]);
}

}  // namespace

extern "C" {

// out[i] = x[i]^y[i] for i < n (device arrays, asynchronous on `stream`):
// which 0, kpp_pow_cr (the integrators' controllers); 1, the CUDA math
// library's pow.  0 on success, -1 on a bad argument or launch error.
int kpp_b200_pow_batch(long long n, const double* x, const double* y, double* out, int which,
                       void* stream) {
  if (n < 0 || (which != 0 && which != 1) || (n > 0 && (!x || !y || !out))) return -1;
  if (n == 0) return 0;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long blocks = (n + 255) / 256;
  pow_kernel<<<(int)(blocks < sms * 8LL ? blocks : sms * 8LL), 256, 0, (cudaStream_t)stream>>>(
      n, x, y, out, which);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// Measured FP64 throughput in TFLOP/s (best of `reps` launches); < 0 on error.
double kpp_b200_fp64_peak_tflops(int kind, int reps) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1.0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  double* out = nullptr;
  if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) return -1.0;
  const int threads = 256, blocks = sms * 8, iters = 1 << 14;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double best = -1.0;
  for (int r = 0; r < reps + 1; r++) {
    cudaEventRecord(e0);
    if (kind == 0) fp64_fma_kernel<<<blocks, threads>>>(out, iters, 0.999999, 1e-6);
    else fp64_muladd_kernel<<<blocks, threads>>>(out, iters, 0.999999, 1e-6);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    double ops_per_iter = kind == 0 ? 2.0 * kChains : 2.0 * kChains;
    double tflops = (double)blocks * threads * iters * ops_per_iter / (ms * 1e-3) / 1e12;
    if (r > 0 && tflops > best) best = tflops;  // first launch is warm-up
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess) return -1.0;
  return best;
}

}  // extern "C"
