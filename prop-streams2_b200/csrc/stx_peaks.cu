// stx_peaks.cu -- FP64 throughput microbenchmarks of the device (libstx_peaks.so).
//
// The chemistry kernels are bound by FP64 arithmetic, not by HBM, so their
// roofline needs the device's FP64 peaks, which are measured here rather than
// taken from a data sheet:
//   * FP64 FMA: every thread runs 8 independent chains of dependent DFMA;
//   * FP64 tensor core (DMMA): every warp runs 4 independent chains of
//     mma.sync.aligned.m8n8k4 with f64 operands and accumulators, 512 flops each
//     (the only FP64 matrix instruction of sm_100a; tcgen05 has no f64 kind).
// Both run a persistent grid of 8 CTAs of 256 threads per SM for a fixed
// number of iterations and are timed with CUDA events on the caller's stream.
// The results are written back so the compiler keeps the arithmetic.
#include <cstdint>
#include <cuda_runtime.h>

namespace {

__global__ void __launch_bounds__(256) k_peak_dfma(double *out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int q = 0; q < 8; q++) x[q] = a + q * 1e-3 + threadIdx.x * 1e-9;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int q = 0; q < 8; q++) x[q] = fma(x[q], b, a);
  }
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < 8; q++) s += x[q];
  if (s == 12345.678) out[0] = s;           // practically never: keeps the chains live
  if (threadIdx.x == 0 && blockIdx.x == 0) out[1] = s;
}

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(256) k_peak_dmma(double *out, int iters, double a, double b) {
  double c[4][2];
#pragma unroll
  for (int q = 0; q < 4; q++) { c[q][0] = q * 1e-3; c[q][1] = -q * 1e-3; }
  const double av = a + (threadIdx.x & 31) * 1e-9, bv = b - (threadIdx.x & 31) * 1e-9;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int q = 0; q < 4; q++) dmma(c[q][0], c[q][1], av, bv);
  }
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < 4; q++) s += c[q][0] + c[q][1];
  if (s == 12345.678) out[0] = s;
  if (threadIdx.x == 0 && blockIdx.x == 0) out[1] = s;
}

}  // namespace

// which = 0: FP64 FMA, 1: FP64 tensor core (DMMA).  *tflops: the measured rate
// (best of 3 launches after one warm-up), in 1e12 flop/s.  Returns 0, or -2 on a
// CUDA error, -1 on a bad argument.
extern "C" int stx_peak_fp64(int which, void *stream, double *tflops) {
  if (!tflops || (which != 0 && which != 1)) return -1;
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -2;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -2;
  const int blocks = nsm * 8, threads = 256;
  const int iters = which == 0 ? 20000 : 4000;
  double *out = nullptr;
  if (cudaMallocAsync((void **)&out, 2 * sizeof(double), s) != cudaSuccess) return -2;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = -1.f;
  for (int rep = 0; rep < 4; rep++) {
    cudaEventRecord(e0, s);
    if (which == 0) k_peak_dfma<<<blocks, threads, 0, s>>>(out, iters, 1.0000001, 0.9999999);
    else k_peak_dmma<<<blocks, threads, 0, s>>>(out, iters, 1.0000001, 0.9999999);
    cudaEventRecord(e1, s);
    if (cudaEventSynchronize(e1) != cudaSuccess) { best = -1.f; break; }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && (best < 0.f || ms < best)) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(out, s);
  if (cudaGetLastError() != cudaSuccess || best <= 0.f) return -2;
  const double flops = which == 0 ? 2.0 * 8.0 * iters * (double)blocks * threads
                                  : 512.0 * 4.0 * iters * (double)blocks * (threads / 32);
  *tflops = flops / (best * 1e-3) / 1e12;
  return 0;
}
