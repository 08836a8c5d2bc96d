// Team-per-matrix fused H(k) + complex Gauss-Jordan inversion, FP64.
//
// A team of W warps (32 W lanes) owns one (k, z) matrix at a time.  Lanes
// form a TR x TC grid (TR * TC = 32 W, TC = 8 or 16 divides 32); lane
// (tr, tc) keeps rows r = tr + TR*rr and columns c = tc + TC*cc in registers
// (cyclic distribution, padded slots are an inert identity).  Per elimination
// step k = tck + TC*kk (slot kk compile-time, lane column tck runtime):
//   * the lanes owning column k pick the largest |Re|+|Im| among the rows not
//     yet used (the zgetrf/izamax choice): shuffles inside each warp, shared
//     memory + one named barrier across the team's warps;
//   * the owners of row p publish the scaled pivot row a_p/a_pk, the owners of
//     column k the multipliers (a_pk - 1 for row p itself, so the update below
//     needs no branch), both in team-private shared memory, double-buffered by
//     step parity: one more barrier (W > 1) or __syncwarp (W = 1) per step;
//   * every lane applies  a <- a - f * pvd  to its register block.
// Rows are never swapped; G[r][s] = X[piv[r]][pinv[s]] is applied when the
// result leaves through the output stage.  Teams are persistent and
// independent; H(k) comes either from a precomputed table (k-major walk,
// so each table row is reused from L2 across energies) or is summed here.
#include "tg_internal.cuh"

namespace tg {

namespace {

template <int N, int W, int TC>
struct Team {
  static constexpr int LANES = 32 * W;
  static constexpr int TR = LANES / TC;
  static constexpr int RB = (N + TR - 1) / TR;
  static constexpr int CB = (N + TC - 1) / TC;
  static constexpr int NR = TR * RB;
  static constexpr int NC = TC * CB;
};

struct TeamSmem {
  size_t stage, bufs, cand, phase, piv, pinv, zw, acc, per_team;
};

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline TeamSmem team_smem(int n, int nr, int nc, int w, int n_neigh) {
  TeamSmem L;
  size_t o = 0;
  L.stage = o; o = al16(o + sizeof(double2) * (size_t)n * n);
  L.bufs = o;  o = al16(o + sizeof(double2) * 2 * (size_t)(nr + nc));
  L.cand = o;  o = al16(o + sizeof(double2) * 2 * 2 * (size_t)w);        // [buf][warp] {value,row}, pivot
  L.phase = o; o = al16(o + sizeof(double2) * (size_t)(n_neigh > 0 ? n_neigh : 1));
  L.piv = o;   o = al16(o + sizeof(int) * (size_t)n);
  L.pinv = o;  o = al16(o + sizeof(int) * (size_t)n);
  L.zw = o;    o = al16(o + sizeof(double) * 8);
  L.acc = o;   o = al16(o + sizeof(double2) * 2 * (size_t)n);           // MODE_EXPECT sums (4 per orbital)
  L.per_team = o;
  return L;
}

__device__ __forceinline__ double2 shfl_d2(double2 v, int src) {
  v.x = __shfl_sync(0xffffffffu, v.x, src);
  v.y = __shfl_sync(0xffffffffu, v.y, src);
  return v;
}

template <int W>
__device__ __forceinline__ void team_sync(int team) {
  if (W == 1) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(team + 1), "r"(32 * W) : "memory");
  }
}

// OUT: 0 = operand / raw outputs, 1 = MODE_EXPECT, 2 = MODE_HK
template <int N, int W, int TC, int OUT>
__global__ void __launch_bounds__(256, 1) green_team_kernel(GreenArgs a) {
  using T = Team<N, W, TC>;
  constexpr int TR = T::TR, RB = T::RB, CB = T::CB, NR = T::NR, NC = T::NC, LANES = T::LANES;
  extern __shared__ __align__(16) unsigned char smem[];
  const TeamSmem L = team_smem(N, NR, NC, W, a.n_neigh);
  const int teams = blockDim.x / LANES;
  const int team = threadIdx.x / LANES;
  const int tl = threadIdx.x % LANES;          // lane within the team
  const int lane = threadIdx.x & 31;
  const int wt = tl >> 5;                      // warp within the team
  unsigned char* base = smem + (size_t)team * L.per_team;
  double2* X = reinterpret_cast<double2*>(base + L.stage);
  double2* bufs = reinterpret_cast<double2*>(base + L.bufs);
  double2* cand = reinterpret_cast<double2*>(base + L.cand);
  double2* phase = reinterpret_cast<double2*>(base + L.phase);
  int* piv = reinterpret_cast<int*>(base + L.piv);
  int* pinv = reinterpret_cast<int*>(base + L.pinv);
  double* zw = reinterpret_cast<double*>(base + L.zw);
  double2* eacc = reinterpret_cast<double2*>(base + L.acc);
  const int tr = tl / TC, tc = tl % TC;

  if (OUT == 1) {
    for (int e = tl; e < 2 * N; e += LANES) eacc[e] = make_double2(0, 0);
  }
  team_sync<W>(team);

  const int64_t nteams = (int64_t)gridDim.x * teams;
  for (int64_t pl = (int64_t)blockIdx.x * teams + team; pl < a.np; pl += nteams) {
    // ---- point data ------------------------------------------------------------
    int64_t ktab = -1;
    if (a.htab) ktab = (a.p0 + pl) / a.n_e;
    if (tl == 0) {
      double zr, zi, kx = 0, ky = 0, kz = 0, w;
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
      zw[0] = zr; zw[1] = zi; zw[2] = kx + a.q[0]; zw[3] = ky + a.q[1]; zw[4] = kz + a.q[2]; zw[5] = w;
    }
    team_sync<W>(team);
    if (ktab < 0) {
      const double kx = zw[2], ky = zw[3], kz = zw[4];
      for (int nb = tl; nb < a.n_neigh; nb += LANES) {
        const double th = kx * a.R[3 * nb] + ky * a.R[3 * nb + 1] + kz * a.R[3 * nb + 2];
        double s, c;
        sincos(th, &s, &c);
        phase[nb] = make_double2(c, s);
      }
      team_sync<W>(team);
    }

    // ---- A = z 1 - H(k) into registers ------------------------------------------
    double2 A[RB][CB];
    {
      const double2 zc = make_double2(zw[0], zw[1]);
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
            if (r == c) v = cadd(v, zc);
          }
          A[rr][cc] = v;
        }
      }
    }

    if (OUT == 2) {
      const double2 zc = make_double2(zw[0], zw[1]);
#pragma unroll
      for (int rr = 0; rr < RB; ++rr)
#pragma unroll
        for (int cc = 0; cc < CB; ++cc) {
          const int r = tr + TR * rr, c = tc + TC * cc;
          if (r < N && c < N) {
            double2 v = A[rr][cc];
            if (r == c) v = csub(v, zc);
            a.out[pl * N * N + (size_t)c * N + r] = make_double2(-v.x, -v.y);
          }
        }
      team_sync<W>(team);
      continue;
    }

    // ---- Gauss-Jordan with implicit partial pivoting -----------------------------
    unsigned used = 0u;     // bit rr: row tr + TR*rr already used as a pivot row
    bool singular = false;
#pragma unroll
    for (int kk = 0; kk < CB; ++kk) {
#pragma unroll 1
      for (int tck = 0; tck < TC; ++tck) {
        const int k = tck + TC * kk;
        if (k >= N) break;
        const int buf = k & 1;
        const bool own_col = (tc == tck);
        double best = -1.0;
        int brow = 0x7fffffff;
        double2 bval = make_double2(0, 0);
        if (own_col) {
#pragma unroll
          for (int rr = 0; rr < RB; ++rr) {
            const int r = tr + TR * rr;
            const double v = fabs(A[rr][kk].x) + fabs(A[rr][kk].y);
            if (r < N && !((used >> rr) & 1u) && (v > best || (v == best && r < brow))) {
              best = v;
              brow = r;
              bval = A[rr][kk];
            }
          }
        }
        // reduce over the lanes of lane column tck inside this warp
#pragma unroll
        for (int m = TC; m < 32; m <<= 1) {
          const double ob = __shfl_xor_sync(0xffffffffu, best, m);
          const int orow = __shfl_xor_sync(0xffffffffu, brow, m);
          const double2 oval = shfl_d2(bval, lane ^ m);
          if (ob > best || (ob == best && orow < brow)) {
            best = ob;
            brow = orow;
            bval = oval;
          }
        }
        int p;
        double2 apk = make_double2(0, 0);
        if (W == 1) {
          best = __shfl_sync(0xffffffffu, best, tck);
          p = __shfl_sync(0xffffffffu, brow, tck);
          apk = shfl_d2(bval, tck);
        } else {
          double2* cb = cand + buf * 2 * W;
          if (lane == tck) {
            cb[2 * wt] = make_double2(best, __longlong_as_double((long long)brow));
            cb[2 * wt + 1] = bval;
          }
          team_sync<W>(team);
          best = -1.0;
          p = 0x7fffffff;
#pragma unroll
          for (int ww = 0; ww < W; ++ww) {
            const double2 e = cb[2 * ww];
            const int row = (int)__double_as_longlong(e.y);
            if (e.x > best || (e.x == best && row < p)) {
              best = e.x;
              p = row;
              apk = cb[2 * ww + 1];
            }
          }
        }
        if (!(best > 0.0)) singular = true;
        const double2 d = crecip_fast(apk);
        const int ptr = p % TR, prr = p / TR;
        double2* pvd = bufs + buf * (NR + NC);
        double2* fcol = pvd + NC;
        if (tr == ptr) {
#pragma unroll
          for (int cc = 0; cc < CB; ++cc) {
            double2 v = A[0][cc];
#pragma unroll
            for (int rr = 1; rr < RB; ++rr)
              if (rr == prr) v = A[rr][cc];
            pvd[tc + TC * cc] = (cc == kk && own_col) ? d : cmul(v, d);
          }
          used |= 1u << prr;
        }
        if (own_col) {
#pragma unroll
          for (int rr = 0; rr < RB; ++rr) {
            const int r = tr + TR * rr;
            double2 f = A[rr][kk];
            if (r == p) f.x -= 1.0;
            fcol[r] = f;
          }
        }
        if (tl == 0) piv[k] = p;
        team_sync<W>(team);
        double2 pv[CB];
#pragma unroll
        for (int cc = 0; cc < CB; ++cc) pv[cc] = pvd[tc + TC * cc];
#pragma unroll
        for (int rr = 0; rr < RB; ++rr) {
          const int r = tr + TR * rr;
          const double2 f = fcol[r];
          if (own_col) A[rr][kk] = make_double2(r == p ? 1.0 : 0.0, 0.0);
#pragma unroll
          for (int cc = 0; cc < CB; ++cc) A[rr][cc] = cfms(f, pv[cc], A[rr][cc]);
        }
      }
    }
    if (tl == 0 && singular && a.status) {
      const int64_t pidx = a.p0 + pl + 1;
      atomicMin(a.status, (int)(pidx < 0x7fffffff ? pidx : 0x7fffffff));
    }
    // ---- stage X and the permutation in shared memory --------------------------
#pragma unroll
    for (int rr = 0; rr < RB; ++rr)
#pragma unroll
      for (int cc = 0; cc < CB; ++cc) {
        const int r = tr + TR * rr, c = tc + TC * cc;
        if (r < N && c < N) X[r * N + c] = A[rr][cc];
      }
    team_sync<W>(team);
    for (int k = tl; k < N; k += LANES) pinv[piv[k]] = k;
    team_sync<W>(team);

    // ---- output stage -----------------------------------------------------------
    const int NN = N * N;
    const double w = zw[5];
    if (OUT == 0) {
      const int nout = a.out2 ? 2 : 1;
      for (int slot = 0; slot < nout; ++slot) {
        const int mode = slot == 0 ? a.mode : a.mode2;
        double2* dst = (slot == 0 ? a.out : a.out2) + pl * (int64_t)NN;
        for (int o = tl; o < NN; o += LANES) {
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
    } else if (OUT == 1) {
      for (int o = tl; o < N / 2; o += LANES) {
        const int ru = a.gg_desc[2 * o], rd = a.gg_desc[2 * o + 1];
        eacc[4 * o + 0] = cadd(eacc[4 * o + 0], cscale(X[piv[ru] * N + pinv[ru]], w));
        eacc[4 * o + 1] = cadd(eacc[4 * o + 1], cscale(X[piv[rd] * N + pinv[rd]], w));
        eacc[4 * o + 2] = cadd(eacc[4 * o + 2], cscale(X[piv[ru] * N + pinv[rd]], w));
        eacc[4 * o + 3] = cadd(eacc[4 * o + 3], cscale(X[piv[rd] * N + pinv[ru]], w));
      }
    }
    team_sync<W>(team);
  }

  if (OUT == 1) {
    team_sync<W>(team);
    double2* dst = a.acc + ((size_t)blockIdx.x * teams + team) * (2 * N);
    for (int e = tl; e < 2 * N; e += LANES) dst[e] = eacc[e];
  }
}

template <int N, int W, int TC, int OUT>
cudaError_t launch_t3(const GreenArgs& a, int num_sms, cudaStream_t s, int* grid_used) {
  using T = Team<N, W, TC>;
  const TeamSmem L = team_smem(N, T::NR, T::NC, W, a.n_neigh);
  int dev = 0;
  cudaGetDevice(&dev);
  int max_smem = 0;
  cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  int teams = 256 / T::LANES;
  while (teams > 1 && L.per_team * teams > (size_t)max_smem) --teams;
  const size_t smem = L.per_team * teams;
  if (smem > (size_t)max_smem) return cudaErrorInvalidValue;
  auto kern = green_team_kernel<N, W, TC, OUT>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  const int threads = teams * T::LANES;
  int per_sm = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  if (err != cudaSuccess) return err;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  if (per_sm * teams > 8) per_sm = (8 + teams - 1) / teams;   // partial buffers: <= 8 teams per SM
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)num_sms * per_sm;
  const int64_t need = (a.np + teams - 1) / teams;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  if (grid_used) *grid_used = (int)grid * teams;   // partial slots (one per team)
  kern<<<(unsigned)grid, threads, smem, s>>>(a);
  return cudaGetLastError();
}

template <int N, int W, int TC>
cudaError_t launch_t(const GreenArgs& a, int num_sms, cudaStream_t s, int* grid_used) {
  if (a.mode == MODE_EXPECT) return launch_t3<N, W, TC, 1>(a, num_sms, s, grid_used);
  if (a.mode == MODE_HK) return launch_t3<N, W, TC, 2>(a, num_sms, s, grid_used);
  return launch_t3<N, W, TC, 0>(a, num_sms, s, grid_used);
}

}  // namespace

// Team-per-matrix path: raw / operand / expectation / H(k) modes.
int green_warp_supported(int n, int mode) {
  const bool nok = (n == 4 || n == 8 || n == 16 || n == 18 || n == 20 || n == 36 || n == 40 || n == 54 ||
                    n == 72 || n == 90);
  const bool mok = mode == MODE_RAW || mode == MODE_A_IMAG || mode == MODE_B_IMAG || mode == MODE_A_REAL ||
                   mode == MODE_B_REAL || mode == MODE_EXPECT || mode == MODE_HK;
  return nok && mok;
}

cudaError_t launch_green_warp(const GreenArgs& a, int num_sms, cudaStream_t s, int* grid_used) {
  if (a.np <= 0) {
    if (grid_used) *grid_used = 0;
    return cudaSuccess;
  }
  switch (a.n) {
    case 4: return launch_t<4, 1, 8>(a, num_sms, s, grid_used);
    case 8: return launch_t<8, 1, 8>(a, num_sms, s, grid_used);
    case 16: return launch_t<16, 1, 8>(a, num_sms, s, grid_used);
    case 18: return launch_t<18, 1, 8>(a, num_sms, s, grid_used);
    case 20: return launch_t<20, 1, 8>(a, num_sms, s, grid_used);
    case 36: return launch_t<36, 2, 8>(a, num_sms, s, grid_used);
    case 40: return launch_t<40, 2, 8>(a, num_sms, s, grid_used);
    case 54: return launch_t<54, 4, 16>(a, num_sms, s, grid_used);
    case 72: return launch_t<72, 8, 16>(a, num_sms, s, grid_used);
    case 90: return launch_t<90, 8, 16>(a, num_sms, s, grid_used);
  }
  return cudaErrorInvalidValue;
}

}  // namespace tg
