// One-warp-per-matrix fused H(k) + complex Gauss-Jordan inversion, FP64.
//
// For dimensions whose whole matrix fits one warp's registers (n = 36: a
// 4-column x 8-row lane grid, 9 x 5 complex per lane), a warp owns one
// (k, z) matrix and needs no barrier: every broadcast of an elimination step
// is a warp shuffle.
//   * Lane (tr, tc) keeps rows r = tr + TR*rr and columns tc + TC*cc.  The
//     register slots of the pivot column (k / TC) and of the pivot row (p / TR)
//     are runtime values but warp-uniform, so they are reached through
//     branches over compile-time slots instead of indexed (local-memory) access.
//   * Pivot: the lanes of lane column k % TC compare |Re|+|Im| over their
//     unused rows (zgetrf's izamax choice, first index on ties), an xor-shuffle
//     reduction over the lane rows finds the row p, one shuffle broadcasts it.
//   * Multipliers f_r = a_rk (- 1 on the pivot row) are shuffled from the pivot
//     column's lanes; the pivot row is shuffled from lane row p % TR inside a
//     warp-uniform branch on p / TR, so its register slot is a constant there.
//   * a <- a - f (a_p / a_pk) with column k overwritten by (r == p) - f / a_pk:
//     the in-place Gauss-Jordan inverse with implicit row pivoting
//     (G[r][s] = X[piv[r]][pinv[s]], applied by the output stage).
// Outputs: the operand layouts of the chi0 contraction (modes A/B, imaginary
// and real axis), raw G, and the expectation-value sums.
#include "tg_internal.cuh"

namespace tg {

namespace {

constexpr int kWarps = 8;   // matrices (warps) per CTA

__device__ __forceinline__ double2 shfl2(double2 v, int src) {
  v.x = __shfl_sync(0xffffffffu, v.x, src);
  v.y = __shfl_sync(0xffffffffu, v.y, src);
  return v;
}

struct W1Smem {
  size_t stage, phase, piv, pinv, acc, per_warp;
};

__host__ __device__ inline size_t a16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline W1Smem w1_smem(int n, int n_neigh) {
  W1Smem L;
  size_t o = 0;
  L.stage = o; o = a16(o + sizeof(double2) * (size_t)n * n);
  L.phase = o; o = a16(o + sizeof(double2) * (size_t)(n_neigh > 0 ? n_neigh : 1));
  L.piv = o;   o = a16(o + sizeof(int) * (size_t)n);
  L.pinv = o;  o = a16(o + sizeof(int) * (size_t)n);
  L.acc = o;   o = a16(o + sizeof(double2) * 2 * (size_t)n);
  L.per_warp = o;
  return L;
}

// Rank-1 update a <- a - f (a_p / a_pk) of one elimination step, pivot-row slot
// R (compile time), every column slot; column k is rewritten afterwards.
template <int R, int RB, int CB>
__device__ __forceinline__ void w1_update(double2 (&A)[RB][CB], const double2 (&f)[RB], int prr, int src, double2 d) {
  if constexpr (R < RB) {
    if (prr == R) {
#pragma unroll
      for (int cc = 0; cc < CB; ++cc) {
        const double2 pv = cmul(shfl2(A[R][cc], src), d);   // scaled pivot-row element of column slot cc
#pragma unroll
        for (int rr = 0; rr < RB; ++rr) A[rr][cc] = cfms(f[rr], pv, A[rr][cc]);
      }
      return;
    }
    w1_update<R + 1, RB, CB>(A, f, prr, src, d);
  }
}

// column slot G (compile time) of the register tile: copy out, or overwrite
// with the inverse's column (r == p) - f_r / a_pk
template <int G, int RB, int CB>
__device__ __forceinline__ void w1_get_col(const double2 (&A)[RB][CB], int g, double2 (&col)[RB]) {
  if constexpr (G < CB) {
    if (g == G) {
#pragma unroll
      for (int rr = 0; rr < RB; ++rr) col[rr] = A[rr][G];
      return;
    }
    w1_get_col<G + 1, RB, CB>(A, g, col);
  }
}

template <int G, int RB, int CB, int TR>
__device__ __forceinline__ void w1_set_col(double2 (&A)[RB][CB], int g, const double2 (&f)[RB], double2 d, int tr,
                                           int p) {
  if constexpr (G < CB) {
    if (g == G) {
#pragma unroll
      for (int rr = 0; rr < RB; ++rr)
        A[rr][G] = cfms(f[rr], d, make_double2(tr + TR * rr == p ? 1.0 : 0.0, 0.0));
      return;
    }
    w1_set_col<G + 1, RB, CB, TR>(A, g, f, d, tr, p);
  }
}

// OUT: 0 = operand / raw outputs, 1 = MODE_EXPECT
template <int N, int TC, int OUT>
__global__ void __launch_bounds__(32 * kWarps, 1) green_w1_kernel(GreenArgs a) {
  constexpr int TR = 32 / TC;
  constexpr int RB = (N + TR - 1) / TR;
  constexpr int CB = (N + TC - 1) / TC;
  extern __shared__ __align__(16) unsigned char smem[];
  const W1Smem L = w1_smem(N, a.n_neigh);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tr = lane / TC, tc = lane % TC;
  unsigned char* base = smem + (size_t)warp * L.per_warp;
  double2* X = reinterpret_cast<double2*>(base + L.stage);
  double2* phase = reinterpret_cast<double2*>(base + L.phase);
  int* piv = reinterpret_cast<int*>(base + L.piv);
  int* pinv = reinterpret_cast<int*>(base + L.pinv);
  double2* eacc = reinterpret_cast<double2*>(base + L.acc);

  if (OUT == 1)
    for (int e = lane; e < 2 * N; e += 32) eacc[e] = make_double2(0, 0);
  __syncwarp();

  const int64_t nw = (int64_t)gridDim.x * kWarps;
  for (int64_t pl = (int64_t)blockIdx.x * kWarps + warp; pl < a.np; pl += nw) {
    // ---- point data (lane 0), broadcast by shuffles ------------------------------
    int64_t ktab = -1;
    if (a.htab) ktab = (a.p0 + pl) / a.n_e;
    double zr = 0, zi = 0, kx = 0, ky = 0, kz = 0, w = 0;
    if (lane == 0) {
      if (a.htab) {
        const int64_t wi = a.p0 + pl;
        const int64_t ik = wi / a.n_e, ie = wi % a.n_e;
        if (a.pts.kind == 0) {
          zr = a.zr;
          zi = a.zi + a.ylist[ie];
          w = a.pts.w[ie * a.nk_tab + ik];
        } else {
          zr = a.zr + a.pts.x2[ie];
          zi = a.zi;
          w = a.pts.p2[ie] * a.pts.w[ik];
        }
      } else {
        const int64_t p = a.p0 + pl;
        if (a.pts.kind == 0) {
          zr = a.zr;
          zi = a.zi + a.pts.y[p];
          kx = a.pts.kp[3 * p]; ky = a.pts.kp[3 * p + 1]; kz = a.pts.kp[3 * p + 2];
          w = a.pts.w[p];
        } else if (a.pts.kind == 1) {
          const int64_t nep = p / a.pts.nk, ik = p % a.pts.nk;
          zr = a.zr + a.pts.x2[nep];
          zi = a.zi;
          kx = a.pts.kp[3 * ik]; ky = a.pts.kp[3 * ik + 1]; kz = a.pts.kp[3 * ik + 2];
          w = a.pts.p2[nep] * a.pts.w[ik];
        } else {
          zr = a.pts.z[p].x;
          zi = a.pts.z[p].y;
          kx = a.pts.kp[3 * p]; ky = a.pts.kp[3 * p + 1]; kz = a.pts.kp[3 * p + 2];
          w = 1.0;
        }
      }
      kx += a.q[0]; ky += a.q[1]; kz += a.q[2];
    }
    zr = __shfl_sync(0xffffffffu, zr, 0);
    zi = __shfl_sync(0xffffffffu, zi, 0);
    w = __shfl_sync(0xffffffffu, w, 0);
    // energy split: the spectral kernel writes the points with Im z >= y_split (zi is the
    // same expression there, warp-uniform here, and this kernel has no block barrier)
    if (a.y_side < 0 && a.htab && a.pts.kind == 0 && zi >= a.y_split) continue;
    if (ktab < 0) {
      kx = __shfl_sync(0xffffffffu, kx, 0);
      ky = __shfl_sync(0xffffffffu, ky, 0);
      kz = __shfl_sync(0xffffffffu, kz, 0);
      for (int nb = lane; nb < a.n_neigh; nb += 32) {
        const double th = kx * a.R[3 * nb] + ky * a.R[3 * nb + 1] + kz * a.R[3 * nb + 2];
        double s, c;
        sincos(th, &s, &c);
        phase[nb] = make_double2(c, s);
      }
      __syncwarp();
    }

    // ---- A = z 1 - H(k) into registers -------------------------------------------
    double2 A[RB][CB];
#pragma unroll
    for (int rr = 0; rr < RB; ++rr) {
      const int r = tr + TR * rr;
#pragma unroll
      for (int cc = 0; cc < CB; ++cc) {
        const int c = tc + TC * cc;
        double2 v = make_double2(r == c ? 1.0 : 0.0, 0.0);   // inert padding
        if (r < N && c < N) {
          double2 h;
          if (ktab >= 0) {
            h = a.htab[ktab * (N * N) + r * N + c];
          } else {
            h = a.h0[(size_t)c * N + r];
            if (a.row_spin[r] == a.row_spin[c]) {
              const int orr = a.row_orb[r], oc = a.row_orb[c];
              const int pb = a.row_atom[r] * a.n_atoms + a.row_atom[c];
              for (int b = a.pair_start[pb]; b < a.pair_start[pb + 1]; ++b)
                h = cfma(phase[a.pair_neigh[b]], a.pair_t[(size_t)b * a.nmax * a.nmax + oc * a.nmax + orr], h);
            }
          }
          v = make_double2(-h.x, -h.y);
          if (r == c) { v.x += zr; v.y += zi; }
        }
        A[rr][cc] = v;
      }
    }

    // ---- Gauss-Jordan, implicit partial pivoting ---------------------------------
    unsigned used = 0u;
    bool singular = false;
#pragma unroll 1
    for (int k = 0; k < N; ++k) {
      const int tck = k % TC, g = k / TC;
      const bool own_col = tc == tck;
      double2 col[RB];
      w1_get_col<0, RB, CB>(A, g, col);   // pivot column slot (lanes of lane column tck)
      double best = -1.0;
      int brow = 0x7fffffff;
      double2 bval = make_double2(0, 0);
      if (own_col) {
#pragma unroll
        for (int rr = 0; rr < RB; ++rr) {
          const int r = tr + TR * rr;
          const double v = fabs(col[rr].x) + fabs(col[rr].y);
          if (r < N && !((used >> rr) & 1u) && (v > best || (v == best && r < brow))) {
            best = v;
            brow = r;
            bval = col[rr];
          }
        }
      }
#pragma unroll
      for (int m = TC; m < 32; m <<= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, m);
        const int orow = __shfl_xor_sync(0xffffffffu, brow, m);
        const double2 oval = shfl2(bval, lane ^ m);
        if (ob > best || (ob == best && orow < brow)) {
          best = ob;
          brow = orow;
          bval = oval;
        }
      }
      best = __shfl_sync(0xffffffffu, best, tck);
      const int p = __shfl_sync(0xffffffffu, brow, tck);
      const double2 apk = shfl2(bval, tck);
      if (!(best > 0.0)) singular = true;
      const double2 d = crecip_fast(apk);
      const int ptr = p % TR, prr = p / TR;
      double2 f[RB];
#pragma unroll
      for (int rr = 0; rr < RB; ++rr) {
        f[rr] = shfl2(col[rr], tr * TC + tck);
        if (tr + TR * rr == p) f[rr].x -= 1.0;
      }
      if (lane == 0) piv[k] = p;
      if (tr == ptr) used |= 1u << prr;
      w1_update<0, RB, CB>(A, f, prr, ptr * TC + tc, d);
      if (own_col) w1_set_col<0, RB, CB, TR>(A, g, f, d, tr, p);
    }
    if (lane == 0 && singular && a.status) {
      const int64_t pidx = a.p0 + pl + 1;
      atomicMin(a.status, (int)(pidx < 0x7fffffff ? pidx : 0x7fffffff));
    }
    // ---- stage X and the permutation in shared memory ----------------------------
#pragma unroll
    for (int rr = 0; rr < RB; ++rr)
#pragma unroll
      for (int cc = 0; cc < CB; ++cc) {
        const int r = tr + TR * rr, c = tc + TC * cc;
        if (r < N && c < N) X[r * N + c] = A[rr][cc];
      }
    __syncwarp();
    for (int k = lane; k < N; k += 32) pinv[piv[k]] = k;
    __syncwarp();

    // ---- output stage ---------------------------------------------------------------
    const int NN = N * N;
    if (OUT == 0) {
      const int nout = a.out2 ? 2 : 1;
      for (int slot = 0; slot < nout; ++slot) {
        const int mode = slot == 0 ? a.mode : a.mode2;
        double2* dst = (slot == 0 ? a.out : a.out2) + pl * (int64_t)NN;
        for (int o = lane; o < NN; o += 32) {
          double2 v;
          if (mode == MODE_RAW) {
            const int r = o % N, c = o / N;
            v = X[piv[r] * N + pinv[c]];
          } else {
            const int rc = a.outmap[o];
            const int r = rc / N, c = rc % N;
            if (mode == MODE_A_IMAG) {
              v = cscale(X[piv[r] * N + pinv[c]], w);
            } else if (mode == MODE_B_IMAG) {
              v = X[piv[c] * N + pinv[r]];
            } else if (mode == MODE_A_REAL) {
              v = cscale(csub(X[piv[r] * N + pinv[c]], cconj(X[piv[c] * N + pinv[r]])), w);
            } else {
              v = cconj(X[piv[r] * N + pinv[c]]);
            }
          }
          dst[o] = v;
        }
      }
    } else {
      for (int o = lane; o < N / 2; o += 32) {
        const int ru = a.gg_desc[2 * o], rd = a.gg_desc[2 * o + 1];
        eacc[4 * o + 0] = cadd(eacc[4 * o + 0], cscale(X[piv[ru] * N + pinv[ru]], w));
        eacc[4 * o + 1] = cadd(eacc[4 * o + 1], cscale(X[piv[rd] * N + pinv[rd]], w));
        eacc[4 * o + 2] = cadd(eacc[4 * o + 2], cscale(X[piv[ru] * N + pinv[rd]], w));
        eacc[4 * o + 3] = cadd(eacc[4 * o + 3], cscale(X[piv[rd] * N + pinv[ru]], w));
      }
    }
    __syncwarp();
  }

  if (OUT == 1) {
    __syncwarp();
    double2* dst = a.acc + ((size_t)blockIdx.x * kWarps + warp) * (2 * N);
    for (int e = lane; e < 2 * N; e += 32) dst[e] = eacc[e];
  }
}

template <int N, int TC, int OUT>
cudaError_t launch_w1(const GreenArgs& a, int num_sms, cudaStream_t s, int* grid_used) {
  const W1Smem L = w1_smem(N, a.n_neigh);
  int dev = 0;
  cudaGetDevice(&dev);
  int max_smem = 0;
  cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const size_t smem = L.per_warp * kWarps;
  if (smem > (size_t)max_smem) return cudaErrorInvalidValue;
  auto kern = green_w1_kernel<N, TC, OUT>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  int per_sm = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * kWarps, smem);
  if (err != cudaSuccess) return err;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  per_sm = 1;   // per-CTA partial slots: kWarps per SM
  int64_t grid = (int64_t)num_sms * per_sm;
  const int64_t need = (a.np + kWarps - 1) / kWarps;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  if (grid_used) *grid_used = (int)grid * kWarps;
  kern<<<(unsigned)grid, 32 * kWarps, smem, s>>>(a);
  return cudaGetLastError();
}

}  // namespace

int green_w1_supported(int n, int mode) {
  const bool mok = mode == MODE_RAW || mode == MODE_A_IMAG || mode == MODE_B_IMAG || mode == MODE_A_REAL ||
                   mode == MODE_B_REAL || mode == MODE_EXPECT;
  return n == 36 && mok;
}

cudaError_t launch_green_w1(const GreenArgs& a, int num_sms, cudaStream_t s, int* grid_used) {
  if (a.np <= 0) {
    if (grid_used) *grid_used = 0;
    return cudaSuccess;
  }
  if (a.n == 36) {
    if (a.mode == MODE_EXPECT) return launch_w1<36, 4, 1>(a, num_sms, s, grid_used);
    return launch_w1<36, 4, 0>(a, num_sms, s, grid_used);
  }
  return cudaErrorInvalidValue;
}

}  // namespace tg
