// Fused H(k) Fourier sum + batched complex Gauss-Jordan inversion, FP64.
//
// One CTA holds MPB matrices; each matrix is spread over TS x TS threads that
// own an RB x RB register block (RB = n / TS).  Per (k, z) point:
//   1. phases exp(i k.R) of every neighbour cell (calchk, mod_hamiltonian.F90:196-204)
//   2. A = z 1 - h0 - sum_blocks phase * t0i, built straight into registers
//      (green, mod_greenfunction.F90:38-54)
//   3. in-place Gauss-Jordan with partial pivoting (largest |Re|+|Im| among the
//      rows not yet used -- the izamax choice of zgetrf), rows never swapped:
//      the pivot row is broadcast through shared memory, the result is the
//      inverse with rows/columns permuted, G[r][s] = X[piv[r]][pinv[s]]
//      (replaces invers = zgetrf + zgetri, mod_tools.F90:796-829)
//   4. an output stage selected by `mode`: raw G, the chi0 contraction operands
//      in pair-block layout, or on-chip accumulation of the occupation /
//      Jacobian reductions.
// The kernel is persistent: a grid of (#SMs x resident CTAs) walks over the
// point range in steps of MPB matrices.
#include "tg_internal.cuh"

#include <algorithm>

namespace tg {

namespace {

struct SmemLayout {
  size_t xs, prow, fcol, phase, candv, candr, piv, pinv, zw, accum, total;
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline SmemLayout smem_layout(int n, int ts, int mpb, int n_neigh, int acc_len) {
  SmemLayout L;
  size_t o = 0;
  L.xs = o;    o = align16(o + sizeof(double2) * size_t(mpb) * n * n);
  L.prow = o;  o = align16(o + sizeof(double2) * 2 * size_t(mpb) * n);
  L.fcol = o;  o = align16(o + sizeof(double2) * 2 * size_t(mpb) * n);
  L.phase = o; o = align16(o + sizeof(double2) * size_t(mpb) * (n_neigh > 0 ? n_neigh : 1));
  L.candv = o; o = align16(o + sizeof(double) * 2 * size_t(mpb) * ts);
  L.candr = o; o = align16(o + sizeof(int) * 2 * size_t(mpb) * ts);
  L.piv = o;   o = align16(o + sizeof(int) * size_t(mpb) * n);
  L.pinv = o;  o = align16(o + sizeof(int) * size_t(mpb) * n);
  L.zw = o;    o = align16(o + sizeof(double) * 8 * size_t(mpb));   // z(2), k(3), w, valid, point
  L.accum = o; o = align16(o + sizeof(double2) * size_t(acc_len));
  L.total = o;
  return L;
}

// entry of the inverse through the implicit-pivot permutation
__device__ __forceinline__ double2 ginv(const double2* X, const int* piv, const int* pinv, int n, int r, int c) {
  return X[piv[r] * n + pinv[c]];
}

// <= 256 threads: two warps per SM sub-partition leave 255 registers per thread
constexpr int kMaxThreads = 256;

template <int N, int TS>
__global__ void __launch_bounds__(kMaxThreads, 1) green_gj_kernel(GreenArgs a, int mpb) {
  constexpr int RB = N / TS;
  constexpr int CB = RB;
  constexpr int TPM = TS * TS;
  static_assert(RB * TS == N, "N must be a multiple of TS");
  static_assert(RB <= 32, "row block too large");

  extern __shared__ __align__(16) unsigned char smem[];
  const SmemLayout L = smem_layout(N, TS, mpb, a.n_neigh, a.acc_len);
  double2* Xs = reinterpret_cast<double2*>(smem + L.xs);
  double2* prow = reinterpret_cast<double2*>(smem + L.prow);
  double2* fcol = reinterpret_cast<double2*>(smem + L.fcol);
  double2* phase = reinterpret_cast<double2*>(smem + L.phase);
  double* candv = reinterpret_cast<double*>(smem + L.candv);
  int* candr = reinterpret_cast<int*>(smem + L.candr);
  int* piv = reinterpret_cast<int*>(smem + L.piv);
  int* pinv = reinterpret_cast<int*>(smem + L.pinv);
  double* zw = reinterpret_cast<double*>(smem + L.zw);
  double2* accum = reinterpret_cast<double2*>(smem + L.accum);

  const int tid = threadIdx.x;
  const int nthreads = blockDim.x;
  const int m = tid / TPM;             // matrix slot of this thread
  const int lt = tid % TPM;
  const int tr = lt / TS, tc = lt % TS;
  const bool active = m < mpb;

  for (int e = tid; e < a.acc_len; e += nthreads) accum[e] = make_double2(0.0, 0.0);

  // per-thread accumulators of MODE_EXPECT: orbital o = tid < n/2
  double2 ex_uu = make_double2(0, 0), ex_dd = ex_uu, ex_ud = ex_uu, ex_du = ex_uu;

  const int64_t ngroups = (a.np + mpb - 1) / mpb;
  for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
    // ---- point data -------------------------------------------------------
    if (active && lt == 0) {
      const int64_t pl = g * mpb + m;
      double* zp = zw + 8 * m;
      const bool valid = pl < a.np;
      double zr = 1.0, zi = 0.0, kx = 0, ky = 0, kz = 0, w = 0.0;
      if (valid) {
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
        kx += a.q[0]; ky += a.q[1]; kz += a.q[2];
      }
      zp[0] = zr; zp[1] = zi; zp[2] = kx; zp[3] = ky; zp[4] = kz; zp[5] = w;
      zp[6] = valid ? 1.0 : 0.0;
    }
    __syncthreads();
    // ---- phases exp(i k.R) -------------------------------------------------
    for (int e = tid; e < mpb * a.n_neigh; e += nthreads) {
      const int mm = e / a.n_neigh, nb = e % a.n_neigh;
      const double* zp = zw + 8 * mm;
      const double th = zp[2] * a.R[3 * nb] + zp[3] * a.R[3 * nb + 1] + zp[4] * a.R[3 * nb + 2];
      double s, c;
      sincos(th, &s, &c);
      phase[mm * a.n_neigh + nb] = make_double2(c, s);
    }
    __syncthreads();

    // ---- A = z 1 - h0 - H_nl(k) straight into the register block -----------
    double2 A[RB][CB];
    const double* zp = zw + 8 * (active ? m : 0);
    const bool valid = active && zp[6] != 0.0;
    const double2 zc = make_double2(zp[0], zp[1]);
    const double2* ph = phase + (active ? m : 0) * a.n_neigh;
#pragma unroll
    for (int rr = 0; rr < RB; ++rr) {
      const int r = tr * RB + rr;
      const int ar = a.row_atom[r], orr = a.row_orb[r], sr = a.row_spin[r];
#pragma unroll
      for (int cc = 0; cc < CB; ++cc) {
        const int c = tc * CB + cc;
        double2 h = a.h0[(size_t)c * N + r];
        const int ac = a.row_atom[c];
        if (a.row_spin[c] == sr) {
          const int oc = a.row_orb[c];
          const int pb = ar * a.n_atoms + ac;
          const int b0 = a.pair_start[pb], b1 = a.pair_start[pb + 1];
          for (int b = b0; b < b1; ++b) {
            const double2 t = a.pair_t[(size_t)b * a.nmax * a.nmax + oc * a.nmax + orr];
            h = cfma(ph[a.pair_neigh[b]], t, h);
          }
        }
        double2 v = make_double2(-h.x, -h.y);
        if (r == c) v = cadd(v, zc);
        if (!valid) v = make_double2(r == c ? 1.0 : 0.0, 0.0);
        A[rr][cc] = v;
      }
    }

    if (a.mode == MODE_HK) {
      // write H = h0 + H_nl(k) (column-major) and skip the inversion
      if (valid) {
        const int64_t pl = g * mpb + m;
#pragma unroll
        for (int rr = 0; rr < RB; ++rr)
#pragma unroll
          for (int cc = 0; cc < CB; ++cc) {
            const int r = tr * RB + rr, c = tc * CB + cc;
            double2 v = A[rr][cc];
            if (r == c) v = csub(v, zc);
            a.out[pl * N * N + (size_t)c * N + r] = make_double2(-v.x, -v.y);
          }
      }
      __syncthreads();
      continue;
    }

    // ---- Gauss-Jordan with implicit partial pivoting -----------------------
    // All register-block accesses use compile-time indices; the step's column
    // and pivot row are selected with runtime predicates (no local memory).
    unsigned used = 0u;
    bool singular = false;
#pragma unroll 1
    for (int k = 0; k < N; ++k) {
      const int kc = k / CB, kk = k - kc * CB;
      const int buf = k & 1;
      double* cv = candv + (buf * mpb + m) * TS;
      int* cr = candr + (buf * mpb + m) * TS;
      const bool owns_col = active && tc == kc;
      double2 colk[RB];
#pragma unroll
      for (int rr = 0; rr < RB; ++rr) {
        double2 v = A[rr][0];
#pragma unroll
        for (int cc = 1; cc < CB; ++cc)
          if (cc == kk) v = A[rr][cc];
        colk[rr] = v;
      }
      if (owns_col) {
        double best = -1.0;
        int brow = 0;
#pragma unroll
        for (int rr = 0; rr < RB; ++rr) {
          const double v = fabs(colk[rr].x) + fabs(colk[rr].y);
          const bool freerow = !((used >> rr) & 1u);
          if (freerow && v > best) { best = v; brow = tr * RB + rr; }
        }
        cv[tr] = best;
        cr[tr] = brow;
      }
      __syncthreads();
      double best = -1.0;
      int p = 0;
      if (active) {
        for (int t = 0; t < TS; ++t) {
          const double v = cv[t];
          if (v > best) { best = v; p = cr[t]; }
        }
      }
      if (!(best > 0.0)) singular = true;
      const int ptr = p / RB, prr = p - ptr * RB;
      double2* pr = prow + (buf * mpb + m) * N;
      double2* fc = fcol + (buf * mpb + m) * N;
      if (active && tr == ptr) {
#pragma unroll
        for (int cc = 0; cc < CB; ++cc) {
          double2 v = A[0][cc];
#pragma unroll
          for (int rr = 1; rr < RB; ++rr)
            if (rr == prr) v = A[rr][cc];
          pr[tc * CB + cc] = v;
        }
        used |= 1u << prr;
      }
      if (owns_col) {
#pragma unroll
        for (int rr = 0; rr < RB; ++rr) fc[tr * RB + rr] = colk[rr];
      }
      if (active && lt == 0) piv[m * N + k] = p;
      __syncthreads();
      if (active) {
        const double2 d = crecip(pr[k]);
        double2 pvd[CB];
#pragma unroll
        for (int cc = 0; cc < CB; ++cc) {
          const int c = tc * CB + cc;
          pvd[cc] = (c == k) ? d : cmul(pr[c], d);
        }
#pragma unroll
        for (int rr = 0; rr < RB; ++rr) {
          const int r = tr * RB + rr;
          const double2 f = fc[r];
          const bool is_p = (r == p);
#pragma unroll
          for (int cc = 0; cc < CB; ++cc) {
            double2 old = A[rr][cc];
            if (owns_col && cc == kk) old = make_double2(0.0, 0.0);
            const double2 upd = cfms(f, pvd[cc], old);
            A[rr][cc] = is_p ? pvd[cc] : upd;
          }
        }
      }
    }
    if (active && lt == 0 && valid && singular && a.status) {
      const int64_t pidx = a.p0 + g * mpb + m + 1;
      atomicMin(a.status, (int)(pidx < 0x7fffffff ? pidx : 0x7fffffff));
    }
    // ---- stage the (permuted) inverse in shared memory ---------------------
    if (active) {
      double2* X = Xs + (size_t)m * N * N;
#pragma unroll
      for (int rr = 0; rr < RB; ++rr)
#pragma unroll
        for (int cc = 0; cc < CB; ++cc) X[(tr * RB + rr) * N + tc * CB + cc] = A[rr][cc];
    }
    __syncthreads();
    for (int e = tid; e < mpb * N; e += nthreads) {
      const int mm = e / N, k = e % N;
      pinv[mm * N + piv[mm * N + k]] = k;
    }
    __syncthreads();

    // ---- output stage ------------------------------------------------------
    const int NN = N * N;
    if (a.mode == MODE_RAW || a.mode == MODE_A_IMAG || a.mode == MODE_B_IMAG || a.mode == MODE_A_REAL ||
        a.mode == MODE_B_REAL) {
      const int nout = a.out2 ? 2 : 1;
      for (int slot = 0; slot < mpb * nout; ++slot) {
        const int mm = slot % mpb;
        const int mode = slot < mpb ? a.mode : a.mode2;
        double2* outp = slot < mpb ? a.out : a.out2;
        const double* zq = zw + 8 * mm;
        if (zq[6] == 0.0) continue;
        const double w = zq[5];
        const double2* X = Xs + (size_t)mm * NN;
        const int* pv = piv + mm * N;
        const int* pi = pinv + mm * N;
        double2* dst = outp + (g * mpb + mm) * (int64_t)NN;
        for (int o = tid; o < NN; o += nthreads) {
          double2 v;
          if (mode == MODE_RAW) {
            const int r = o % N, c = o / N;
            v = ginv(X, pv, pi, N, r, c);
          } else {
            const int rc = a.outmap[o];
            const int r = rc / N, c = rc % N;
            if (mode == MODE_A_IMAG) {
              v = cscale(ginv(X, pv, pi, N, r, c), w);
            } else if (mode == MODE_B_IMAG) {
              v = ginv(X, pv, pi, N, c, r);
            } else if (mode == MODE_A_REAL) {
              v = cscale(csub(ginv(X, pv, pi, N, r, c), cconj(ginv(X, pv, pi, N, c, r))), w);
            } else {
              v = cconj(ginv(X, pv, pi, N, r, c));
            }
          }
          dst[o] = v;
        }
      }
    } else if (a.mode == MODE_EXPECT) {
      // orbital o = tid: up/down rows from the host table gg_desc[2o], gg_desc[2o+1]
      if (tid < N / 2) {
        const int r_up = a.gg_desc[2 * tid], r_dn = a.gg_desc[2 * tid + 1];
        for (int mm = 0; mm < mpb; ++mm) {
          const double* zq = zw + 8 * mm;
          if (zq[6] == 0.0) continue;
          const double w = zq[5];
          const double2* X = Xs + (size_t)mm * NN;
          const int* pv = piv + mm * N;
          const int* pi = pinv + mm * N;
          ex_uu = cadd(ex_uu, cscale(ginv(X, pv, pi, N, r_up, r_up), w));
          ex_dd = cadd(ex_dd, cscale(ginv(X, pv, pi, N, r_dn, r_dn), w));
          ex_ud = cadd(ex_ud, cscale(ginv(X, pv, pi, N, r_up, r_dn), w));
          ex_du = cadd(ex_du, cscale(ginv(X, pv, pi, N, r_dn, r_up), w));
        }
      }
    } else if (a.mode == MODE_GG) {
      // descriptor per block: [i_up_off, i_dn_off, j_up_off, j_dn_off, row_list, col_list]
      // followed by orbital lists stored as [len, orb_0, orb_1, ...] (local orbital indices).
      const int nblocks = a.acc_len / 16;
      const int* desc = a.gg_desc;
      const int* orbl = a.gg_desc + 6 * nblocks;
      for (int b = tid; b < nblocks; b += nthreads) {
        const int* d = desc + 6 * b;
        const int i_off_up = d[0], i_off_dn = d[1];   // row offsets of site i (up block, down block)
        const int j_off_up = d[2], j_off_dn = d[3];
        const int gs = d[4], hs = d[5];
        const int glen = orbl[gs], hlen = orbl[hs];
        double2 acc16[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) acc16[q] = accum[16 * b + q];
        for (int mm = 0; mm < mpb; ++mm) {
          const double* zq = zw + 8 * mm;
          if (zq[6] == 0.0) continue;
          const double w = zq[5];
          const double2* X = Xs + (size_t)mm * NN;
          const int* pv = piv + mm * N;
          const int* pi = pinv + mm * N;
          for (int gi = 0; gi < glen; ++gi) {
            const int mu = orbl[gs + 1 + gi];
            const int ri[2] = {i_off_up + mu, i_off_dn + mu};
            for (int hi = 0; hi < hlen; ++hi) {
              const int nu = orbl[hs + 1 + hi];
              const int rj[2] = {j_off_up + nu, j_off_dn + nu};
              double2 u[2][2], v[2][2];
#pragma unroll
              for (int s1 = 0; s1 < 2; ++s1)
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                  u[s1][t] = cscale(ginv(X, pv, pi, N, ri[s1], rj[t]), w);   // G(i s' mu, j t nu)
                  v[t][s1] = ginv(X, pv, pi, N, rj[t], ri[s1]);              // G(j t' nu, i s mu)
                }
#pragma unroll
              for (int sp = 0; sp < 2; ++sp)
#pragma unroll
                for (int t = 0; t < 2; ++t)
#pragma unroll
                  for (int tp = 0; tp < 2; ++tp)
#pragma unroll
                    for (int s = 0; s < 2; ++s) {
                      const int q = sp + 2 * t + 4 * tp + 8 * s;
                      acc16[q] = cfma(u[sp][t], v[tp][s], acc16[q]);
                    }
            }
          }
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) accum[16 * b + q] = acc16[q];
      }
    } else if (a.mode == MODE_DIAG4) {
      // acc[4*o + a] += w * sum_{s,s'} sigma_a[s,s'] G(i s' mu, i s mu) (trace over spin)
      for (int o = tid; o < N / 2; o += nthreads) {
        const int* d = a.gg_desc + 2 * o;   // up row, down row of orbital o
        const int ru = d[0], rd = d[1];
        double2 s0 = make_double2(0, 0), s1 = s0, s2 = s0, s3 = s0;
        for (int mm = 0; mm < mpb; ++mm) {
          const double* zq = zw + 8 * mm;
          if (zq[6] == 0.0) continue;
          const double w = zq[5];
          const double2* X = Xs + (size_t)mm * NN;
          const int* pv = piv + mm * N;
          const int* pi = pinv + mm * N;
          const double2 guu = cscale(ginv(X, pv, pi, N, ru, ru), w), gdd = cscale(ginv(X, pv, pi, N, rd, rd), w);
          const double2 gud = cscale(ginv(X, pv, pi, N, ru, rd), w), gdu = cscale(ginv(X, pv, pi, N, rd, ru), w);
          s0 = cadd(s0, cadd(guu, gdd));                                   // 1
          s1 = cadd(s1, cadd(gdu, gud));                                   // sigma_x
          s2 = cadd(s2, cmul(make_double2(0, 1), csub(gud, gdu)));         // sigma_y: -i G(d,u) + i G(u,d)
          s3 = cadd(s3, csub(guu, gdd));                                   // sigma_z
        }
        accum[4 * o + 0] = cadd(accum[4 * o + 0], s0);
        accum[4 * o + 1] = cadd(accum[4 * o + 1], s1);
        accum[4 * o + 2] = cadd(accum[4 * o + 2], s2);
        accum[4 * o + 3] = cadd(accum[4 * o + 3], s3);
      }
    } else if (a.mode == MODE_ENTRIES) {
      // acc[e] += w * G(r_e, c_e) for the entry list (r_e, c_e) = gg_desc[2e], gg_desc[2e + 1]
      for (int e = tid; e < a.acc_len; e += nthreads) {
        const int r = a.gg_desc[2 * e], c = a.gg_desc[2 * e + 1];
        double2 sum = make_double2(0, 0);
        for (int mm = 0; mm < mpb; ++mm) {
          const double* zq = zw + 8 * mm;
          if (zq[6] == 0.0) continue;
          sum = cfma(make_double2(zq[5], 0.0), ginv(Xs + (size_t)mm * NN, piv + mm * N, pinv + mm * N, N, r, c), sum);
        }
        accum[e] = cadd(accum[e], sum);
      }
    }
    __syncthreads();
  }

  // ---- per-CTA partial results ----------------------------------------------
  if (a.mode == MODE_EXPECT) {
    if (tid < N / 2) {
      double2* dst = a.acc + (size_t)blockIdx.x * (2 * N);
      dst[4 * tid + 0] = ex_uu;
      dst[4 * tid + 1] = ex_dd;
      dst[4 * tid + 2] = ex_ud;
      dst[4 * tid + 3] = ex_du;
    }
  } else if (a.mode == MODE_GG || a.mode == MODE_DIAG4 || a.mode == MODE_ENTRIES) {
    double2* dst = a.acc + (size_t)blockIdx.x * a.acc_len;
    for (int e = tid; e < a.acc_len; e += nthreads) dst[e] = accum[e];
  }
}

struct Cfg {
  int n, ts, mpb;
};

// thread-grid side and matrices per CTA for each supported dimension
const Cfg kCfgs[] = {
    {4, 2, 64}, {8, 2, 64}, {16, 4, 16}, {18, 3, 28}, {20, 5, 10}, {36, 6, 7},
    {40, 10, 2}, {54, 9, 3}, {72, 12, 1}, {90, 15, 1},
};

const Cfg* find_cfg(int n) {
  for (const Cfg& c : kCfgs)
    if (c.n == n) return &c;
  return nullptr;
}

template <int N, int TS>
cudaError_t launch_t(const GreenArgs& a, int mpb, int num_sms, cudaStream_t s, int* grid_used) {
  int dev = 0;
  cudaGetDevice(&dev);
  int max_smem = 0;
  cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  int acc_len = a.acc_len;
  // shrink the matrix group until the tile fits in shared memory
  while (mpb > 1 && smem_layout(N, TS, mpb, a.n_neigh, acc_len).total > (size_t)max_smem) mpb = (mpb + 1) / 2;
  const size_t smem = smem_layout(N, TS, mpb, a.n_neigh, acc_len).total;
  if (smem > (size_t)max_smem) return cudaErrorInvalidValue;
  auto kern = green_gj_kernel<N, TS>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  const int threads = TS * TS * mpb;
  int per_sm = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  if (err != cudaSuccess) return err;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  if (per_sm > 8) per_sm = 8;   // per-CTA partial buffers are sized for 8 CTAs per SM
  const int64_t ngroups = (a.np + mpb - 1) / mpb;
  int64_t grid = (int64_t)num_sms * per_sm;
  if (grid > ngroups) grid = ngroups;
  if (grid < 1) grid = 1;
  if (grid_used) *grid_used = (int)grid;
  kern<<<(unsigned)grid, threads, smem, s>>>(a, mpb);
  return cudaGetLastError();
}

}  // namespace

int green_supported(int n) { return find_cfg(n) != nullptr; }

int green_acc_ctas(int n, int64_t np, int num_sms) {
  // upper bound of the grid launch_green uses (for sizing per-CTA partial buffers)
  (void)n;
  int64_t g = (int64_t)num_sms * 8;
  if (g > np) g = np;
  return (int)std::max<int64_t>(g, 1);
}

bool green_is_spectral(const GreenArgs& a) {
  return a.eigU && a.eigL && a.n_e > 0 && spectral_supported(a.mode, a.mode2, a.out2 != nullptr);
}

cudaError_t launch_green(const GreenArgs& a, int num_sms, cudaStream_t s, int* grid_used) {
  if (a.triQ) {
    if (grid_used) *grid_used = 0;
    return launch_green_tri(a, num_sms, s);
  }
  if (green_is_spectral(a)) {
    if (grid_used) *grid_used = 0;
    return launch_green_spectral(a, a.eigU, a.eigL, a.outinv, num_sms, s);
  }
  if (a.eout || a.eout2) return cudaErrorInvalidValue;   // only the spectral kernel writes sidecars
  // eigendecompositions without an H(k) table: the pass is k-major, which only the spectral
  // kernel walks without a table
  if (a.eigU && !a.htab) return cudaErrorInvalidValue;
  if (green_w1_supported(a.n, a.mode)) return launch_green_w1(a, num_sms, s, grid_used);
  if (green_warp_supported(a.n, a.mode)) return launch_green_warp(a, num_sms, s, grid_used);
  const Cfg* c = find_cfg(a.n);
  if (!c) {
    if (grid_used) *grid_used = 0;
    if (green_cluster_supported(a.n, a.mode)) return launch_green_cluster(a, num_sms, s);
    return cudaErrorInvalidValue;
  }
  if (a.np <= 0) {
    if (grid_used) *grid_used = 0;
    return cudaSuccess;
  }
  switch (a.n) {
    case 4: return launch_t<4, 2>(a, c->mpb, num_sms, s, grid_used);
    case 8: return launch_t<8, 2>(a, c->mpb, num_sms, s, grid_used);
    case 16: return launch_t<16, 4>(a, c->mpb, num_sms, s, grid_used);
    case 18: return launch_t<18, 3>(a, c->mpb, num_sms, s, grid_used);
    case 20: return launch_t<20, 5>(a, c->mpb, num_sms, s, grid_used);
    case 36: return launch_t<36, 6>(a, c->mpb, num_sms, s, grid_used);
    case 40: return launch_t<40, 10>(a, c->mpb, num_sms, s, grid_used);
    case 54: return launch_t<54, 9>(a, c->mpb, num_sms, s, grid_used);
    case 72: return launch_t<72, 12>(a, c->mpb, num_sms, s, grid_used);
    case 90: return launch_t<90, 15>(a, c->mpb, num_sms, s, grid_used);
  }
  return cudaErrorInvalidValue;
}

}  // namespace tg
