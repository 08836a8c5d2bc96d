// Resolvents of large Hermitian H(k) on meshes whose energies share a k list, without an
// eigendecomposition.
//
// Per k, H = Q T Q^H with T real symmetric tridiagonal: the Householder reduction of
// LAPACK's zhetd2 (lower form) with zlarfg's reflectors H_j = I - tau_j v_j v_j^H, which
// make every off-diagonal beta_j real, so Q = H_0 H_1 ... H_{n-2}.  Then for every z
//   G_SS(k, z) = Q_S (z - T)^-1 Q_S^H,
// Q_S being the rows S of Q the caller needs (the d orbitals of a d-only chi, or all rows).
// The reduction runs once per k for all energies; per (k, z) the tridiagonal solve
// (z - T) X = Q_S^H costs O(n |S|) and G_SS = Q_S X is a complex GEMM on the FP64 tensor
// cores (mma.sync m8n8k4 .f64).  z - T is factored without pivoting: its pivots obey
// Im d_{i+1} = Im z + e_i^2 Im d_i / |d_i|^2 >= Im z > 0, so none vanishes for Im z > 0.
// Like Gauss-Jordan, the result is the resolvent of H + dH with |dH| ~ eps |H| (both steps
// are backward stable reductions), without the eigenvector mixing that makes spectral G
// less accurate near the real axis.
#include "tg_internal.cuh"

#include <algorithm>

namespace tg {

namespace {

constexpr int kTriThreads = 256;
constexpr int kTriCols = 32;          // columns of G per solve block
constexpr int kTriStride = kTriCols + 1;   // padded row of the block in shared memory

__device__ __forceinline__ double2 warp_sum2(double2 v) {
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}

// sum over the block, returned to every thread (red: 2 doubles per warp)
__device__ double2 block_sum2(double2 v, double* red) {
  v = warp_sum2(v);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) {
    red[2 * warp] = v.x;
    red[2 * warp + 1] = v.y;
  }
  __syncthreads();
  double2 t = make_double2(0.0, 0.0);
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
    t.x += red[2 * w];
    t.y += red[2 * w + 1];
  }
  return t;
}

// A: [nk][n][n] row-major H(k) table rows, overwritten; rows[ns]: the rows S of Q to form.
// Out: D[k][i] = T(i, i), E[k][i] = T(i + 1, i) (E[k][n - 1] = 0), Q[k][s][c] = Q(rows[s], c).
// One CTA per k; a warp per row for the matrix-vector products and rank-2 updates.
__global__ void __launch_bounds__(kTriThreads) hh_tridiag_kernel(double2* __restrict__ A, int64_t nk, int n,
                                                                 const int* __restrict__ rows, int ns,
                                                                 double* __restrict__ D, double* __restrict__ E,
                                                                 double2* __restrict__ Q) {
  extern __shared__ __align__(16) unsigned char smem[];
  double2* v = reinterpret_cast<double2*>(smem);      // [n] reflector
  double2* w = v + n;                                 // [n] p, then w
  double* red = reinterpret_cast<double*>(w + n);     // [2 * warps]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int64_t k = blockIdx.x; k < nk; k += gridDim.x) {
    double2* Ak = A + k * (int64_t)n * n;
    double2* Qk = Q + k * (int64_t)ns * n;
    for (int64_t e = threadIdx.x; e < (int64_t)ns * n; e += blockDim.x) {
      const int s = (int)(e / n), col = (int)(e % n);
      Qk[e] = make_double2(col == rows[s] ? 1.0 : 0.0, 0.0);
    }
    for (int j = 0; j + 1 < n; ++j) {
      const int m = n - j - 1;
      // x = A(j+1:, j) into v; |x(1:)|^2
      double part = 0.0;
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const double2 x = Ak[(int64_t)(j + 1 + i) * n + j];
        v[i] = x;
        if (i > 0) part += x.x * x.x + x.y * x.y;
      }
      const double xn2 = block_sum2(make_double2(part, 0.0), red).x;   // its barriers publish v
      const double2 alpha = v[0];
      const bool refl = !(xn2 == 0.0 && alpha.y == 0.0);
      // zlarfg: beta = -sign(Re alpha) |(alpha, x)|, tau = (beta - alpha) / beta, v = x / (alpha - beta)
      const double beta = refl ? -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2), alpha.x) : alpha.x;
      if (threadIdx.x == 0) {
        D[k * n + j] = Ak[(int64_t)j * n + j].x;
        E[k * n + j] = beta;
      }
      __syncthreads();   // alpha read by every thread before v changes
      if (!refl) continue;
      const double2 tau = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
      {
        const double dr = alpha.x - beta, di = alpha.y;
        const double inv = 1.0 / (dr * dr + di * di);
        const double2 sc = make_double2(dr * inv, -di * inv);
        for (int i = threadIdx.x; i < m; i += blockDim.x) v[i] = i == 0 ? make_double2(1.0, 0.0) : cmul(v[i], sc);
      }
      __syncthreads();
      // p = tau A22 v into w: a warp per row, lanes along the row
      for (int r = warp; r < m; r += nw) {
        const double2* Ar = Ak + (int64_t)(j + 1 + r) * n + (j + 1);
        double2 acc = make_double2(0.0, 0.0);
        for (int col = lane; col < m; col += 32) acc = cfma(Ar[col], v[col], acc);
        acc = warp_sum2(acc);
        if (lane == 0) w[r] = cmul(tau, acc);
      }
      __syncthreads();
      // w = p - (tau / 2) (p^H v) v
      double2 dp = make_double2(0.0, 0.0);
      for (int i = threadIdx.x; i < m; i += blockDim.x) dp = cfma(cconj(w[i]), v[i], dp);
      dp = block_sum2(dp, red);
      const double2 a2 = cscale(cmul(tau, dp), -0.5);
      for (int i = threadIdx.x; i < m; i += blockDim.x) w[i] = cfma(a2, v[i], w[i]);
      __syncthreads();
      // A22 -= v w^H + w v^H
      for (int r = warp; r < m; r += nw) {
        double2* Ar = Ak + (int64_t)(j + 1 + r) * n + (j + 1);
        const double2 vr = v[r], wr = w[r];
        for (int col = lane; col < m; col += 32)
          Ar[col] = csub(Ar[col], cadd(cmul(vr, cconj(w[col])), cmul(wr, cconj(v[col]))));
      }
      // Q_S <- Q_S H_j on columns j+1..: y = Q_S(:, j+1:) v, Q_S(:, j+1:) -= tau y v^H
      for (int s = warp; s < ns; s += nw) {
        double2* Qs = Qk + (int64_t)s * n + (j + 1);
        double2 acc = make_double2(0.0, 0.0);
        for (int col = lane; col < m; col += 32) acc = cfma(Qs[col], v[col], acc);
        const double2 ty = cmul(tau, warp_sum2(acc));
        for (int col = lane; col < m; col += 32) Qs[col] = csub(Qs[col], cmul(ty, cconj(v[col])));
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      D[k * n + n - 1] = Ak[(int64_t)(n - 1) * n + n - 1].x;
      E[k * n + n - 1] = 0.0;
    }
    __syncthreads();
  }
}

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

struct TriArgs {
  GreenArgs g;
};

__host__ __device__ inline size_t tri_smem(int n) {
  return sizeof(double) * 2 * (size_t)n + sizeof(double2) * 2 * (size_t)n + sizeof(double2) * (size_t)n * kTriStride;
}

constexpr int kTriMB = 5;   // M fragments of a warp in flight

// One CTA per point (k, z) of a k-major pass: the LU of z - T (thread 0), then per block of 32
// columns c of S the solves (z - T) x_c = conj(Q_S(c, :))^T (warp 0, one lane per column) and
// G(S, c) = Q_S x_c (every warp: an 8-column fragment of the block times groups of 8-row
// fragments of Q_S, K = n in steps of 4).  Output MODE_RAW: G column-major per point, entries
// (r, c) of S x S only.
__global__ void __launch_bounds__(kTriThreads) tri_green_kernel(TriArgs ta) {
  extern __shared__ __align__(16) unsigned char smem[];
  const GreenArgs& a = ta.g;
  const int n = a.n, ns = a.tri_ns;
  double* Dk = reinterpret_cast<double*>(smem);         // [n]
  double* Ek = Dk + n;                                  // [n]
  double2* invd = reinterpret_cast<double2*>(Ek + n);   // [n] 1 / pivot
  double2* lm = invd + n;                               // [n] multipliers e_i / d_i
  double2* X = lm + n;                                  // [n][kTriStride]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g8 = lane >> 2, t4 = lane & 3;
  const int64_t nn = (int64_t)n * n;
  const int nmf = (ns + 7) / 8;
  for (int64_t pl = blockIdx.x; pl < a.np; pl += gridDim.x) {
    const int64_t wi = a.p0 + pl;
    const int64_t ik = wi / a.n_e, ie = wi % a.n_e;
    double zx, zy;
    if (a.pts.kind == 0) {
      zx = a.zr;
      zy = a.zi + a.ylist[ie];
    } else {
      zx = a.zr + a.pts.x2[ie];
      zy = a.zi;
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      Dk[i] = a.triD[ik * n + i];
      Ek[i] = a.triE[ik * n + i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      // z - T = L U: d_0 = z - D_0, l_i = -E_i / d_i, d_{i+1} = z - D_{i+1} - E_i^2 / d_i (lm stores +E_i / d_i)
      double2 d = make_double2(zx - Dk[0], zy);
      for (int i = 0; i < n; ++i) {
        const double s2 = d.x * d.x + d.y * d.y;
        if (s2 == 0.0 && a.status) {
          const int64_t pidx = wi + 1;
          atomicMin(a.status, (int)(pidx < 0x7fffffff ? pidx : 0x7fffffff));
        }
        const double inv = s2 > 0.0 ? 1.0 / s2 : 0.0;
        const double2 id = make_double2(d.x * inv, -d.y * inv);
        invd[i] = id;
        if (i + 1 < n) {
          const double2 l = cscale(id, Ek[i]);
          lm[i] = l;
          d = make_double2(zx - Dk[i + 1] - Ek[i] * l.x, zy - Ek[i] * l.y);
        }
      }
    }
    const double2* Qk = a.triQ + ik * (int64_t)ns * n;
    double2* Gp = a.out + pl * nn;
    for (int cb = 0; cb < ns; cb += kTriCols) {
      const int ncols = min(kTriCols, ns - cb);
      // right-hand sides conj(Q_S(c, :)) of the block's columns (zero past the last)
      for (int e = threadIdx.x; e < n * kTriCols; e += blockDim.x) {
        const int t = e / n, i = e % n;
        X[i * kTriStride + t] = t < ncols ? cconj(Qk[(int64_t)(cb + t) * n + i]) : make_double2(0.0, 0.0);
      }
      __syncthreads();
      if (warp == 0 && lane < ncols) {
        double2* x = X + lane;
        double2 y = x[0];
        for (int i = 1; i < n; ++i) {   // L y = b
          y = cfma(lm[i - 1], y, x[i * kTriStride]);
          x[i * kTriStride] = y;
        }
        double2 xi = cmul(y, invd[n - 1]);   // U x = y
        x[(n - 1) * kTriStride] = xi;
        for (int i = n - 2; i >= 0; --i) {
          xi = cmul(cadd(x[i * kTriStride], cscale(xi, Ek[i])), invd[i]);
          x[i * kTriStride] = xi;
        }
      }
      __syncthreads();
      // G(S, cb + t) = Q_S X: warp -> 8-column fragment nf, M fragments mf = half, half + 2, ...
      const int nf = warp & 3, half = warp >> 2;
      for (int mf0 = half; mf0 < nmf; mf0 += 2 * kTriMB) {
        double cr[kTriMB][2], ci[kTriMB][2];
        const double2* qrow[kTriMB];
        bool live[kTriMB];
#pragma unroll
        for (int u = 0; u < kTriMB; ++u) {
          cr[u][0] = cr[u][1] = ci[u][0] = ci[u][1] = 0.0;
          const int mf = mf0 + 2 * u, row = mf * 8 + g8;
          live[u] = mf < nmf && row < ns;
          qrow[u] = Qk + (int64_t)(live[u] ? row : 0) * n;
        }
        for (int k0 = 0; k0 < n; k0 += 4) {
          const int kk = k0 + t4;
          const bool kin = kk < n;
          const double2 b = kin ? X[kk * kTriStride + nf * 8 + g8] : make_double2(0.0, 0.0);
#pragma unroll
          for (int u = 0; u < kTriMB; ++u) {
            const double2 av = live[u] && kin ? qrow[u][kk] : make_double2(0.0, 0.0);
            dmma(cr[u][0], cr[u][1], av.x, b.x);
            dmma(cr[u][0], cr[u][1], -av.y, b.y);
            dmma(ci[u][0], ci[u][1], av.x, b.y);
            dmma(ci[u][0], ci[u][1], av.y, b.x);
          }
        }
#pragma unroll
        for (int u = 0; u < kTriMB; ++u) {
          const int mf = mf0 + 2 * u, row = mf * 8 + g8;
          if (mf >= nmf || row >= ns) continue;
          const int r = a.trirows[row];
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const int t = nf * 8 + 2 * t4 + j;
            if (t < ncols) Gp[(int64_t)a.trirows[cb + t] * n + r] = make_double2(cr[u][j], ci[u][j]);
          }
        }
      }
      __syncthreads();
    }
  }
}

}  // namespace

int tri_supported(int n) {
  if (n < 2) return 0;
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
  return tri_smem(n) <= (size_t)optin;
}

cudaError_t launch_tridiag(double2* H, int64_t nk, int n, const int* rows, int ns, double* D, double* E,
                           double2* Q, int num_sms, cudaStream_t s) {
  if (nk <= 0) return cudaSuccess;
  if (n < 2 || ns <= 0 || ns > n) return cudaErrorInvalidValue;
  const size_t smem = sizeof(double2) * 2 * (size_t)n + sizeof(double) * 2 * (kTriThreads / 32);
  const int64_t grid = std::min<int64_t>(nk, (int64_t)num_sms * 4);
  hh_tridiag_kernel<<<(unsigned)grid, kTriThreads, smem, s>>>(H, nk, n, rows, ns, D, E, Q);
  return cudaGetLastError();
}

cudaError_t launch_green_tri(const GreenArgs& g, int num_sms, cudaStream_t s) {
  if (g.np <= 0) return cudaSuccess;
  if (g.mode != MODE_RAW || g.out2 || !g.triD || !g.triE || !g.triQ || !g.trirows || g.tri_ns <= 0 ||
      g.tri_ns > g.n || g.n_e <= 0)
    return cudaErrorInvalidValue;
  if (!tri_supported(g.n)) return cudaErrorInvalidValue;
  const size_t smem = tri_smem(g.n);
  cudaError_t e = cudaFuncSetAttribute(tri_green_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tri_green_kernel, kTriThreads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm <= 0) return cudaErrorInvalidValue;
  TriArgs ta;
  ta.g = g;
  const int64_t grid = std::min<int64_t>(g.np, (int64_t)num_sms * per_sm);
  tri_green_kernel<<<(unsigned)grid, kTriThreads, smem, s>>>(ta);
  return cudaGetLastError();
}

}  // namespace tg
