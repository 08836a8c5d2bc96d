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
// tri_green_kernel: blocks of COLS columns of G per solve; COLS = 16 lets two CTAs share an
// SM at n = 288, COLS = 96 solves every column of a system up to 96 rows at once
constexpr int kTriColsBig = 96;
constexpr int kTriColsSmall = 16;

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

// not volatile: the scheduler may interleave the MMAs of independent accumulators (a chain on
// one accumulator keeps its order through the data dependence, so results do not change)
__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

struct TriArgs {
  GreenArgs g;
};

template <int COLS>
__host__ __device__ inline size_t tri_smem(int n) {
  return sizeof(double) * 2 * (size_t)n + sizeof(double2) * 2 * (size_t)n + sizeof(double2) * (size_t)n * (COLS + 1);
}

// One CTA per point (k, z) of a k-major pass: the LU of z - T (thread 0), then per block of COLS
// columns c of S the solves (z - T) x_c = conj(Q_S(c, :))^T (one thread per column) and
// G(S, c) = Q_S x_c on the FP64 tensor cores: tiles of MB 8-row fragments of Q_S by one 8-column
// fragment of the block, K = n in steps of 4, tiles dealt to the warps in turn.  With COLS = 16
// two CTAs per SM overlap one's serial LU and solves with the other's GEMM.  Output MODE_RAW: G
// column-major per point, entries (r, c) of S x S only.
template <int COLS, int MB, int MINB>
__global__ void __launch_bounds__(kTriThreads, MINB) tri_green_kernel(TriArgs ta) {
  constexpr int STRIDE = COLS + 1;   // padded row of the block in shared memory
  constexpr int NF = COLS / 8;
  extern __shared__ __align__(16) unsigned char smem[];
  const GreenArgs& a = ta.g;
  const int n = a.n, ns = a.tri_ns;
  double* Dk = reinterpret_cast<double*>(smem);         // [n]
  double* Ek = Dk + n;                                  // [n]
  double2* invd = reinterpret_cast<double2*>(Ek + n);   // [n] 1 / pivot
  double2* lm = invd + n;                               // [n] multipliers e_i / d_i
  double2* X = lm + n;                                  // [n][STRIDE]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  const int g8 = lane >> 2, t4 = lane & 3;
  const int64_t nn = (int64_t)n * n;
  const int nmf = (ns + 7) / 8;
  const int ngroups = (nmf + MB - 1) / MB;
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
        // |d|^2 >= (Im z)^2 keeps the Newton reciprocal in its range; the division covers the rest
        const double inv = s2 > 1e-300 ? rcp_newton(s2) : (s2 > 0.0 ? 1.0 / s2 : 0.0);
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
    for (int cb = 0; cb < ns; cb += COLS) {
      const int ncols = min(COLS, ns - cb);
      // right-hand sides conj(Q_S(c, :)) of the block's columns (zero past the last)
      for (int e = threadIdx.x; e < n * COLS; e += blockDim.x) {
        const int t = e / n, i = e % n;
        X[i * STRIDE + t] = t < ncols ? cconj(Qk[(int64_t)(cb + t) * n + i]) : make_double2(0.0, 0.0);
      }
      __syncthreads();
      if (threadIdx.x < ncols) {
        double2* x = X + threadIdx.x;
        double2 y = x[0];
        for (int i = 1; i < n; ++i) {   // L y = b
          y = cfma(lm[i - 1], y, x[i * STRIDE]);
          x[i * STRIDE] = y;
        }
        double2 xi = cmul(y, invd[n - 1]);   // U x = y
        x[(n - 1) * STRIDE] = xi;
        for (int i = n - 2; i >= 0; --i) {
          xi = cmul(cadd(x[i * STRIDE], cscale(xi, Ek[i])), invd[i]);
          x[i * STRIDE] = xi;
        }
      }
      __syncthreads();
      // G(S, cb + t) = Q_S X: tile (M group mg, column fragment nf) -> warp (tile mod warps)
      const int nfl = (ncols + 7) / 8;
      for (int tile = warp; tile < ngroups * nfl; tile += nwarp) {
        const int nf = tile % nfl, mg = tile / nfl;
        double cr[MB][2], ci[MB][2];
        const double2* qrow[MB];
        bool live[MB];
#pragma unroll
        for (int u = 0; u < MB; ++u) {
          cr[u][0] = cr[u][1] = ci[u][0] = ci[u][1] = 0.0;
          const int row = (mg * MB + u) * 8 + g8;
          live[u] = row < ns;
          qrow[u] = Qk + (int64_t)(live[u] ? row : 0) * n;
        }
        for (int k0 = 0; k0 < n; k0 += 4) {
          const int kk = k0 + t4;
          const bool kin = kk < n;
          const double2 b = kin ? X[kk * STRIDE + nf * 8 + g8] : make_double2(0.0, 0.0);
#pragma unroll
          for (int u = 0; u < MB; ++u) {
            const double2 av = live[u] && kin ? qrow[u][kk] : make_double2(0.0, 0.0);
            dmma(cr[u][0], cr[u][1], av.x, b.x);
            dmma(cr[u][0], cr[u][1], -av.y, b.y);
            dmma(ci[u][0], ci[u][1], av.x, b.y);
            dmma(ci[u][0], ci[u][1], av.y, b.x);
          }
        }
#pragma unroll
        for (int u = 0; u < MB; ++u) {
          const int row = (mg * MB + u) * 8 + g8;
          if (row >= ns) continue;
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

// Systems of at most 96 rows: Q_S stays in shared memory for all the points of its k (each CTA
// walks a contiguous range of the k-major pass), so the GEMM reads both operands from shared
// memory.  Per point: the LU of z - T, then two blocks of 48 columns, each solved one thread per
// column and multiplied on the FP64 tensor cores by a 4 x 2 grid of warps, each holding 3 x 3
// fragments of 8 x 8.
constexpr int kSmallRows = 96;
constexpr int kSmallCols = 48;

__host__ __device__ inline size_t tri_small_smem(int n) {
  return sizeof(double) * 2 * (size_t)n + sizeof(double2) * 2 * (size_t)n +
         sizeof(double2) * (size_t)n * (kSmallCols + 1) + sizeof(double2) * (size_t)kSmallRows * (n + 1);
}

__global__ void __launch_bounds__(kTriThreads, 1) tri_green_small_kernel(TriArgs ta) {
  constexpr int XS = kSmallCols + 1;
  extern __shared__ __align__(16) unsigned char smem[];
  const GreenArgs& a = ta.g;
  const int n = a.n, ns = a.tri_ns, AS = n + 1;
  double* Dk = reinterpret_cast<double*>(smem);         // [n]
  double* Ek = Dk + n;                                  // [n]
  double2* invd = reinterpret_cast<double2*>(Ek + n);   // [n]
  double2* lm = invd + n;                               // [n]
  double2* X = lm + n;                                  // [n][XS]
  double2* As = X + (size_t)n * XS;                     // [ns][AS] = Q_S of the current k
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g8 = lane >> 2, t4 = lane & 3;
  const int wm = warp >> 1, wn = warp & 1;   // 4 x 2 warp grid: M fragments 3 wm.., N fragments 3 wn..
  const int64_t nn = (int64_t)n * n;
  const int64_t per = (a.np + gridDim.x - 1) / gridDim.x;
  const int64_t p_begin = blockIdx.x * per, p_end = min(a.np, p_begin + per);
  int64_t k_loaded = -1;
  for (int64_t pl = p_begin; pl < p_end; ++pl) {
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
    __syncthreads();   // the previous point is done with As, Dk, Ek
    if (ik != k_loaded) {
      const double2* Qk = a.triQ + ik * (int64_t)ns * n;
      for (int e = threadIdx.x; e < ns * n; e += blockDim.x) As[(e / n) * AS + e % n] = Qk[e];
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        Dk[i] = a.triD[ik * n + i];
        Ek[i] = a.triE[ik * n + i];
      }
      k_loaded = ik;
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      double2 d = make_double2(zx - Dk[0], zy);
      for (int i = 0; i < n; ++i) {
        const double s2 = d.x * d.x + d.y * d.y;
        if (s2 == 0.0 && a.status) {
          const int64_t pidx = wi + 1;
          atomicMin(a.status, (int)(pidx < 0x7fffffff ? pidx : 0x7fffffff));
        }
        // |d|^2 >= (Im z)^2 keeps the Newton reciprocal in its range; the division covers the rest
        const double inv = s2 > 1e-300 ? rcp_newton(s2) : (s2 > 0.0 ? 1.0 / s2 : 0.0);
        const double2 id = make_double2(d.x * inv, -d.y * inv);
        invd[i] = id;
        if (i + 1 < n) {
          const double2 l = cscale(id, Ek[i]);
          lm[i] = l;
          d = make_double2(zx - Dk[i + 1] - Ek[i] * l.x, zy - Ek[i] * l.y);
        }
      }
    }
    double2* Gp = a.out + pl * nn;
    for (int cb = 0; cb < ns; cb += kSmallCols) {
      const int ncols = min(kSmallCols, ns - cb);
      for (int e = threadIdx.x; e < n * kSmallCols; e += blockDim.x) {
        const int t = e / n, i = e % n;
        X[i * XS + t] = t < ncols ? cconj(As[(cb + t) * AS + i]) : make_double2(0.0, 0.0);
      }
      __syncthreads();
      if (threadIdx.x < ncols) {
        double2* x = X + threadIdx.x;
        double2 y = x[0];
        for (int i = 1; i < n; ++i) {
          y = cfma(lm[i - 1], y, x[i * XS]);
          x[i * XS] = y;
        }
        double2 xi = cmul(y, invd[n - 1]);
        x[(n - 1) * XS] = xi;
        for (int i = n - 2; i >= 0; --i) {
          xi = cmul(cadd(x[i * XS], cscale(xi, Ek[i])), invd[i]);
          x[i * XS] = xi;
        }
      }
      __syncthreads();
      double cr[3][3][2], ci[3][3][2];
#pragma unroll
      for (int u = 0; u < 3; ++u)
#pragma unroll
        for (int v = 0; v < 3; ++v) cr[u][v][0] = cr[u][v][1] = ci[u][v][0] = ci[u][v][1] = 0.0;
      for (int k0 = 0; k0 < n; k0 += 4) {
        const int kk = k0 + t4;
        const bool kin = kk < n;
        double2 av[3], bv[3];
#pragma unroll
        for (int u = 0; u < 3; ++u) {
          const int row = (3 * wm + u) * 8 + g8;
          av[u] = kin && row < ns ? As[row * AS + kk] : make_double2(0.0, 0.0);
          bv[u] = kin ? X[kk * XS + (3 * wn + u) * 8 + g8] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < 3; ++u)
#pragma unroll
          for (int v = 0; v < 3; ++v) {
            dmma(cr[u][v][0], cr[u][v][1], av[u].x, bv[v].x);
            dmma(cr[u][v][0], cr[u][v][1], -av[u].y, bv[v].y);
            dmma(ci[u][v][0], ci[u][v][1], av[u].x, bv[v].y);
            dmma(ci[u][v][0], ci[u][v][1], av[u].y, bv[v].x);
          }
      }
#pragma unroll
      for (int u = 0; u < 3; ++u) {
        const int row = (3 * wm + u) * 8 + g8;
        if (row >= ns) continue;
        const int r = a.trirows[row];
#pragma unroll
        for (int v = 0; v < 3; ++v)
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const int t = (3 * wn + v) * 8 + 2 * t4 + j;
            if (t < ncols) Gp[(int64_t)a.trirows[cb + t] * n + r] = make_double2(cr[u][v][j], ci[u][v][j]);
          }
      }
      __syncthreads();
    }
  }
}

}  // namespace

int tri_optin() {
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
  return optin;
}

int tri_supported(int n) { return n >= 2 && tri_smem<kTriColsSmall>(n) <= (size_t)tri_optin(); }

cudaError_t launch_tridiag(double2* H, int64_t nk, int n, const int* rows, int ns, double* D, double* E,
                           double2* Q, int num_sms, cudaStream_t s) {
  if (nk <= 0) return cudaSuccess;
  if (n < 2 || ns <= 0 || ns > n) return cudaErrorInvalidValue;
  const size_t smem = sizeof(double2) * 2 * (size_t)n + sizeof(double) * 2 * (kTriThreads / 32);
  const int64_t grid = std::min<int64_t>(nk, (int64_t)num_sms * 4);
  hh_tridiag_kernel<<<(unsigned)grid, kTriThreads, smem, s>>>(H, nk, n, rows, ns, D, E, Q);
  return cudaGetLastError();
}

template <int COLS, int MB, int MINB>
cudaError_t launch_tri_cols(const GreenArgs& g, int num_sms, cudaStream_t s) {
  const size_t smem = tri_smem<COLS>(g.n);
  auto kernel = tri_green_kernel<COLS, MB, MINB>;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTriThreads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm <= 0) return cudaErrorInvalidValue;
  TriArgs ta;
  ta.g = g;
  const int64_t grid = std::min<int64_t>(g.np, (int64_t)num_sms * per_sm);
  kernel<<<(unsigned)grid, kTriThreads, smem, s>>>(ta);
  return cudaGetLastError();
}

cudaError_t launch_green_tri(const GreenArgs& g, int num_sms, cudaStream_t s) {
  if (g.np <= 0) return cudaSuccess;
  if (g.mode != MODE_RAW || g.out2 || !g.triD || !g.triE || !g.triQ || !g.trirows || g.tri_ns <= 0 ||
      g.tri_ns > g.n || g.n_e <= 0)
    return cudaErrorInvalidValue;
  if (!tri_supported(g.n)) return cudaErrorInvalidValue;
  // up to 96 rows: Q_S resident in shared memory per k
  if (g.n <= kSmallRows && g.tri_ns <= kSmallRows && tri_small_smem(g.n) <= (size_t)tri_optin()) {
    const size_t smem = tri_small_smem(g.n);
    cudaError_t e = cudaFuncSetAttribute(tri_green_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    TriArgs ta;
    ta.g = g;
    const int64_t grid = std::min<int64_t>(g.np, (int64_t)num_sms);
    tri_green_small_kernel<<<(unsigned)grid, kTriThreads, smem, s>>>(ta);
    return cudaGetLastError();
  }
  // every column in one block where the rows of chi are few and the block fits
  if (g.tri_ns <= kTriColsBig && tri_smem<kTriColsBig>(g.n) <= (size_t)tri_optin())
    return launch_tri_cols<kTriColsBig, 6, 1>(g, num_sms, s);
  return launch_tri_cols<kTriColsSmall, 5, 2>(g, num_sms, s);
}

}  // namespace tg
