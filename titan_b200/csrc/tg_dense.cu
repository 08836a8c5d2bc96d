// FP64 dense kernels for the RPA Dyson solve chi = (1 + chi_hf U)^-1 chi_hf
// (calculate_chi.F90:85-89): a tiled complex GEMM and a right-looking LU
// with partial pivoting applied to the augmented system [1 + chi_hf U | chi_hf].
#include <cuda_runtime.h>

#include <vector>

#include "../../include/titan_gpu.h"
#include "tg_internal.cuh"

namespace tg {
namespace {

constexpr int GT = 16;

// C = beta*C + A*B, all column-major n x n
__global__ void zgemm_nn_kernel(int n, const double2* __restrict__ A, const double2* __restrict__ B,
                                double2* __restrict__ C, int add_identity) {
  __shared__ double2 As[GT][GT + 1], Bs[GT][GT + 1];
  const int r = blockIdx.y * GT + threadIdx.y;
  const int col = blockIdx.x * GT + threadIdx.x;
  double2 acc = make_double2(0, 0);
  for (int k0 = 0; k0 < n; k0 += GT) {
    const int ka = k0 + threadIdx.x, kb = k0 + threadIdx.y;
    As[threadIdx.y][threadIdx.x] = (r < n && ka < n) ? A[(size_t)ka * n + r] : make_double2(0, 0);
    Bs[threadIdx.y][threadIdx.x] = (kb < n && col < n) ? B[(size_t)col * n + kb] : make_double2(0, 0);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < GT; ++k) acc = cfma(As[threadIdx.y][k], Bs[k][threadIdx.x], acc);
    __syncthreads();
  }
  if (r < n && col < n) {
    if (add_identity && r == col) acc.x += 1.0;
    C[(size_t)col * n + r] = acc;
  }
}

// pivot search in column k (rows k..n-1) by |re| + |im|, first maximum wins
__global__ void pivot_kernel(int n, int k, const double2* __restrict__ M, int* __restrict__ piv, int* status) {
  __shared__ double bv[1024];
  __shared__ int bi[1024];
  double best = -1.0;
  int bidx = k;
  for (int r = k + threadIdx.x; r < n; r += blockDim.x) {
    const double2 v = M[(size_t)k * n + r];
    const double a = fabs(v.x) + fabs(v.y);
    if (a > best) { best = a; bidx = r; }
  }
  bv[threadIdx.x] = best;
  bi[threadIdx.x] = bidx;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      const double o = bv[threadIdx.x + s];
      const int oi = bi[threadIdx.x + s];
      if (o > bv[threadIdx.x] || (o == bv[threadIdx.x] && oi < bi[threadIdx.x])) {
        bv[threadIdx.x] = o;
        bi[threadIdx.x] = oi;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    piv[k] = bi[0];
    if (!(bv[0] > 0.0)) atomicMin(status, k + 1);
  }
}

// swap rows k and piv[k] of the augmented [M | R] (n x (n + n) column-major, two arrays)
__global__ void swap_kernel(int n, int k, const int* __restrict__ piv, double2* M, double2* R) {
  const int p = piv[k];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == k) return;
  if (c < n) {
    double2 t = M[(size_t)c * n + k];
    M[(size_t)c * n + k] = M[(size_t)c * n + p];
    M[(size_t)c * n + p] = t;
    t = R[(size_t)c * n + k];
    R[(size_t)c * n + k] = R[(size_t)c * n + p];
    R[(size_t)c * n + p] = t;
  }
}

// eliminate column k below and above the pivot (Gauss-Jordan on the augmented system)
__global__ void eliminate_kernel(int n, int k, double2* M, double2* R) {
  const int r = blockIdx.y * blockDim.y + threadIdx.y;   // row
  const int c = blockIdx.x * blockDim.x + threadIdx.x;   // column of [M | R], 0 .. 2n-1
  if (r >= n || c >= 2 * n || r == k) return;
  const double2 d = crecip(M[(size_t)k * n + k]);
  const double2 f = cmul(M[(size_t)k * n + r], d);
  if (c < n) {
    if (c <= k) return;   // columns <= k of M are not needed again
    M[(size_t)c * n + r] = cfms(f, M[(size_t)c * n + k], M[(size_t)c * n + r]);
  } else {
    const int cc = c - n;
    R[(size_t)cc * n + r] = cfms(f, R[(size_t)cc * n + k], R[(size_t)cc * n + r]);
  }
}

__global__ void scale_rows_kernel(int n, const double2* __restrict__ M, double2* R) {
  const int r = blockIdx.y * blockDim.y + threadIdx.y;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n || c >= n) return;
  const double2 d = crecip(M[(size_t)r * n + r]);
  R[(size_t)c * n + r] = cmul(R[(size_t)c * n + r], d);
}

}  // namespace

int dyson_device(int n, const double2* chi_hf, const double2* U, double2* work, double2* chi, int* piv, int* status,
                 cudaStream_t s) {
  dim3 b(GT, GT), g((n + GT - 1) / GT, (n + GT - 1) / GT);
  // work = 1 + chi_hf U
  zgemm_nn_kernel<<<g, b, 0, s>>>(n, chi_hf, U, work, 1);
  cudaMemcpyAsync(chi, chi_hf, sizeof(double2) * (size_t)n * n, cudaMemcpyDeviceToDevice, s);
  for (int k = 0; k < n; ++k) {
    pivot_kernel<<<1, 256, 0, s>>>(n, k, work, piv, status);
    swap_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, k, piv, work, chi);
    dim3 eb(32, 8), eg((2 * n + 31) / 32, (n + 7) / 8);
    eliminate_kernel<<<eg, eb, 0, s>>>(n, k, work, chi);
  }
  scale_rows_kernel<<<g, b, 0, s>>>(n, work, chi);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace tg
