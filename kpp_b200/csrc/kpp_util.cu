// Measurement helpers for the benchmark: the FP64 peak of this GPU, measured
// with a throughput kernel (no vendor figure for FP64 is assumed); the device
// self-test of kpp_div.cuh's division through a reciprocal; and a batched
// evaluation of the controllers' pow (kpp_ratelaws.cuh's kpp_pow_cr) beside
// the CUDA math library's, for their tests.
//
//   kind 0: fused multiply-add (DFMA), 2 flops per instruction
//   kind 1: separate multiply and add (DMUL + DADD), 1 flop per instruction;
//           this is the instruction mix of the Rosenbrock kernels, which are
//           built without FMA contraction
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "kpp_div.cuh"
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

// Operands for the division self-test: a counter-based hash per sample
// (splitmix64's finaliser) for the sign, significand and exponent.
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33;
  return x;
}

__device__ __forceinline__ double operand(uint64_t r, int emin, int emax) {
  const int e = emin + (int)((r >> 52) % (uint64_t)(emax - emin + 1));
  return __longlong_as_double(
      (long long)(((r >> 63) << 63) | ((uint64_t)(e + 1023) << 52) | (r & 0xFFFFFFFFFFFFFULL)));
}

// mode 0: random operands; 1: divisors with a significand of all ones, or
// nearly; 2: divisors next to a power of two; 3: dividends a = RN(q b), so
// that quotients sit next to representable numbers.
__global__ void __launch_bounds__(256) division_check_kernel(uint64_t seed, long long n, int emin,
                                                             int emax, int mode,
                                                             unsigned long long* bad) {
  unsigned long long local = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const uint64_t r1 = mix64(seed * 0x9E3779B97F4A7C15ULL + 2 * (uint64_t)i);
    const uint64_t r2 = mix64(seed * 0x9E3779B97F4A7C15ULL + 2 * (uint64_t)i + 1);
    double a = operand(r1, emin, emax), b = operand(r2, emin, emax);
    const long long bb = __double_as_longlong(b) & ~0xFFFFFFFFFFFFFLL;
    if (mode == 1) b = __longlong_as_double(bb | (0xFFFFFFFFFFFFFLL - (long long)(r2 & 0xFF)));
    if (mode == 2) b = __longlong_as_double(bb | (long long)(r2 & 0xFF));
    if (mode == 3) a = __dmul_rn(operand(r1 | 1, -20, 20), b);
    const double y = 1.0 / b;
    if (__double_as_longlong(kpp_div_recip(a, b, y)) != __double_as_longlong(a / b)) local++;
  }
  if (local) atomicAdd(bad, local);
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

// Self-test of the division through a reciprocal (kpp_div.cuh): the number of
// n samples (operand exponents in [emin, emax], the given mode) for which it
// differs from the division a / b in any bit; < 0 on error.
long long kpp_b200_check_division(unsigned long long seed, long long n, int emin, int emax,
                                  int mode) {
  if (n < 0 || emin < -1022 || emax > 1023 || emin > emax || mode < 0 || mode > 3) return -1;
  unsigned long long* bad = nullptr;
  if (cudaMalloc(&bad, sizeof *bad) != cudaSuccess) return -1;
  cudaMemset(bad, 0, sizeof *bad);
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  division_check_kernel<<<sms * 8, 256>>>(seed, n, emin, emax, mode, bad);
  unsigned long long h = 0;
  const cudaError_t e = cudaMemcpy(&h, bad, sizeof h, cudaMemcpyDeviceToHost);
  cudaFree(bad);
  return e == cudaSuccess ? (long long)h : -1;
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
