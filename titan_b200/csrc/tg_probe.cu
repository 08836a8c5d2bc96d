// Measurement and numerics hooks: the FP64 peak of this GPU (the roofline denominator of
// the inversion kernels) and the reciprocal the Gauss-Jordan kernels use for pivots.
//
// tg_fp64_peak times two throughput loops with CUDA events on the context's stream:
//   * DFMA: every thread runs 8 independent fma chains (enough in flight to hide the
//     pipe latency at 8 warps per SM sub-partition);
//   * DMMA: every warp runs 4 independent mma.sync.m8n8k4.f64 chains (512 flops each),
//     the FP64 tensor path of the spectral Green functions.
// Grid: 4 CTAs of 256 threads per SM.  Flops = 2 per fma, 512 per m8n8k4.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "../../include/titan_gpu.h"
#include "tg_internal.cuh"

using namespace tg;

namespace {

constexpr int kProbeThreads = 256;
constexpr int kProbeCtasPerSm = 4;

__global__ void __launch_bounds__(kProbeThreads) dfma_loop(double* out, int iters, double x, double y) {
  double a[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = threadIdx.x * 1e-3 + i;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = fma(a[i], x, y);
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += a[i];
  if (s == 1.2345) out[blockIdx.x] = s;   // never true for the inputs used; keeps the loop
}

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(kProbeThreads) dmma_loop(double* out, int iters, double x) {
  double d[4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i) d[i][0] = d[i][1] = 0.0;
  const double a = x * (threadIdx.x & 3), b = x * (threadIdx.x >> 3);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 4; ++i) dmma(d[i], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 4; ++i) s += d[i][0] + d[i][1];
  if (s == 1.2345) out[blockIdx.x] = s;
}

__global__ void rcp_kernel(const double* s, double* r, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    r[i] = rcp_newton(s[i]);
}

}  // namespace

extern "C" {

int tg_fp64_peak(tg_ctx* ctx, double* tflops_dfma, double* tflops_dmma) {
  (void)ctx;
  if (!tflops_dfma || !tflops_dmma) return TG_ERR_ARG;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return TG_ERR_CUDA;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return TG_ERR_CUDA;
  const int grid = sms * kProbeCtasPerSm;
  double* out = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaMalloc(&out, sizeof(double) * grid);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  float ms_fma = 0.f, ms_mma = 0.f;
  const int it_fma = 1 << 16, it_mma = 1 << 14;
  if (e == cudaSuccess) {
    dfma_loop<<<grid, kProbeThreads, 0, st>>>(out, 256, 1.0000001, 1e-9);   // warm-up
    cudaEventRecord(e0, st);
    dfma_loop<<<grid, kProbeThreads, 0, st>>>(out, it_fma, 1.0000001, 1e-9);
    cudaEventRecord(e1, st);
    e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms_fma, e0, e1);
  }
  if (e == cudaSuccess) {
    dmma_loop<<<grid, kProbeThreads, 0, st>>>(out, 256, 1e-3);
    cudaEventRecord(e0, st);
    dmma_loop<<<grid, kProbeThreads, 0, st>>>(out, it_mma, 1e-3);
    cudaEventRecord(e1, st);
    e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms_mma, e0, e1);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  if (out) cudaFree(out);
  if (e != cudaSuccess) return TG_ERR_CUDA;
  const double threads = (double)grid * kProbeThreads;
  *tflops_dfma = threads * it_fma * 8 * 2.0 / (ms_fma * 1e-3) / 1e12;
  const double warps = threads / 32.0;
  *tflops_dmma = warps * it_mma * 4 * 512.0 / (ms_mma * 1e-3) / 1e12;
  return TG_OK;
}

int tg_rcp_check(int64_t n, const double* s, double* r) {
  if (n < 0 || (n > 0 && (!s || !r))) return TG_ERR_ARG;
  if (n == 0) return TG_OK;
  double *ds = nullptr, *dr = nullptr;
  cudaError_t e = cudaMalloc(&ds, sizeof(double) * n);
  if (e == cudaSuccess) e = cudaMalloc(&dr, sizeof(double) * n);
  if (e == cudaSuccess) e = cudaMemcpy(ds, s, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rcp_kernel<<<(unsigned)std::min<int64_t>((n + 255) / 256, 4096), 256>>>(ds, dr, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(r, dr, sizeof(double) * n, cudaMemcpyDeviceToHost);
  if (ds) cudaFree(ds);
  if (dr) cudaFree(dr);
  return e == cudaSuccess ? TG_OK : TG_ERR_CUDA;
}

}  // extern "C"
