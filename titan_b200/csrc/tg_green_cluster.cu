// Batched G(k, z) = (z - h0 - H(k))^-1 for any dimension up to 288: one thread-block
// cluster per matrix, panel-blocked Gauss-Jordan with partial pivoting.
//
// The matrix of one (k, z) point is too large for one SM at the reference's larger
// systems (a 288 x 288 complex matrix is 1.33 MB), so a cluster of CS <= 9 CTAs shares it:
//   * columns are grouped in panels of kPB = 8; panel P lives in CTA P % CS (local panel
//     P / CS), so each CTA holds up to kNLC = 32 columns (four panels) of every row, kept in
//     shared memory as [slot][row] (147 KB at dimH = 288, 9 CTAs); thread t works on row t.
//     (A row segment of 32 complex entries in registers would leave 9-warp CTAs, 168
//     registers per thread, spilling; the update runs over register halves of 16 slots);
//   * panel P, phase 1 (its owner CTA alone): eight Gauss-Jordan steps restricted to the
//     panel's columns.  Step j picks the pivot row r_j of column 8 P + j (largest
//     |Re| + |Im| among the rows not yet used, first index on ties -- the izamax choice of
//     zgetrf), records the column before the step (the multipliers f_j) and 1 / a_rj, and
//     eliminates inside the panel.  The multipliers and pivots go to a per-cluster buffer in
//     global memory (L2-resident, read back with ld.global.cg), then one cluster barrier
//     publishes the panel;
//   * phase 2 (every CTA, on its other columns): the pivot rows' current segments are
//     staged in shared memory, 32 threads turn them into the scaled pivot rows of the eight
//     steps (prow_j = (row r_j - sum_{k<j} f_k[r_j] prow_k) / a_rj), and every row applies
//     the rank-8 update row_i -= sum_j f_j[i] prow_j (pivot row r_j: prow_j - sum_{k>j} ...);
//     the result equals eight rank-1 Gauss-Jordan steps, with one cluster barrier per panel
//     instead of one per step;
//   * rows are never swapped: the result X holds G[step(t)][piv(j)] at (t, j), where step(t)
//     is the step whose pivot row was t; the output stage permutes the rows in shared memory
//     and writes G column-major per point (MODE_RAW), one column per coalesced store run.
// The kernel is persistent: the grid holds as many clusters as fit, each walking the point
// range.  This replaces invers = zgetrf + zgetri (mod_tools.F90:796-829) inside green
// (mod_greenfunction.F90:19-75) for dimensions the single-SM kernels do not cover; H(k)
// comes from a tabulated row (calchk + hamilt_local) or is summed in the kernel.
#include "tg_internal.cuh"

#include <cooperative_groups.h>

#include <algorithm>

namespace tg {

namespace {

namespace cg = cooperative_groups;

constexpr int kPB = 8;           // columns per panel
constexpr int kNLC = 32;         // local columns per CTA (four panels; registers per row segment)
constexpr int kMaxN = 288;       // one row per thread
constexpr int kMaxCS = 9;        // cluster size (9 > 8: non-portable, enabled at launch)
constexpr int kMaxWarps = kMaxN / 32;

struct ClSmem {
  size_t candrow, prow, pr, pinv, piv, phase, fs, blk, total;
};

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline ClSmem cl_smem(int n, int n_neigh) {
  ClSmem L;
  size_t o = 0;
  L.candrow = o; o = al16(o + sizeof(double2) * 2 * kMaxWarps * (kPB + 1));
  L.prow = o;    o = al16(o + sizeof(double2) * kPB * kNLC);
  L.pr = o;      o = al16(o + sizeof(int) * kPB);
  L.pinv = o;    o = al16(o + sizeof(double2) * kPB);
  L.piv = o;     o = al16(o + sizeof(int) * (size_t)n);
  L.phase = o;   o = al16(o + sizeof(double2) * (size_t)(n_neigh > 0 ? n_neigh : 1));
  L.fs = o;      o = al16(o + sizeof(double2) * (size_t)kPB * n);
  L.blk = o;     o = al16(o + sizeof(double2) * (size_t)kNLC * n);
  L.total = o;
  return L;
}

// per-cluster workspace in global memory: F[2][kPB][n] multipliers, INV[2][kPB], R[2][kPB]
__host__ __device__ inline size_t ws_cluster_bytes(int n) {
  return sizeof(double2) * (2 * kPB * (size_t)n + 2 * kPB) + sizeof(int) * 2 * kPB;
}

struct ClState {
  int n, t;
  bool used;           // this thread's row has been a pivot row
  int my_step;         // step at which it became one
};

__device__ __forceinline__ double2 ldcg2(const double2* p) { return __ldcg(p); }

// Phase 1 of the panel in slots s0 .. s0 + 7 of the CTA's block (its owner CTA only): nb
// Gauss-Jordan steps on the panel's columns; the multipliers f_j (the column before step j)
// go to F[j][row], 1 / a_rj and r_j to INV[j], R[j].  One CTA barrier per step: every warp
// reduces its best candidate row by shuffles and its winning lane posts that row's panel
// entries (cand rows, two buffers by step parity); after the barrier every thread picks the
// CTA-wide winner (largest |Re| + |Im|, smallest row on ties), scales the winner's posted
// entries itself and updates its own row.
__device__ __forceinline__ void factor_panel(ClState& st, double2* blk, int s0, double2* candrow, double2* F,
                                             double2* INV, int* R, int nb, int* status, int64_t point) {
  const int t = st.t, n = st.n;
  const int warp = t >> 5, lane = t & 31, nw = (blockDim.x + 31) >> 5;
  double2* row = blk + (size_t)s0 * n + t;   // row[s * n] = this thread's entry in slot s0 + s
  double2 x[kPB];
#pragma unroll
  for (int s = 0; s < kPB; ++s) x[s] = t < n ? row[(size_t)s * n] : make_double2(0, 0);
#pragma unroll
  for (int j = 0; j < kPB; ++j) {
    if (j < nb) {
      const double2 v = x[j];
      if (t < n) F[(size_t)j * n + t] = v;
      double best = (t < n && !st.used) ? fabs(v.x) + fabs(v.y) : -1.0;
      int bi = t;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      const int pb = j & 1;
      double2* cw = candrow + (size_t)(pb * kMaxWarps + warp) * (kPB + 1);   // [value, row] + kPB entries
      if (t == bi) {
        cw[0] = make_double2(best, (double)bi);
#pragma unroll
        for (int s = 0; s < kPB; ++s) cw[1 + s] = x[s];
      }
      __syncthreads();
      int wbest = 0;
      double vb = -2.0;
      int rb = 0x7fffffff;
      for (int w = 0; w < nw; ++w) {
        const double2 h = candrow[(size_t)(pb * kMaxWarps + w) * (kPB + 1)];
        const int hr = (int)h.y;
        if (h.x > vb || (h.x == vb && hr < rb)) {
          vb = h.x;
          rb = hr;
          wbest = w;
        }
      }
      const double2* pr = candrow + (size_t)(pb * kMaxWarps + wbest) * (kPB + 1) + 1;
      const double2 pv = pr[j];
      if (pv.x == 0.0 && pv.y == 0.0 && t == 0) atomicMin(status, (int)(point + 1));
      const double2 inv = crecip_fast(pv);
      if (t == 0) {
        INV[j] = inv;
        R[j] = rb;
      }
      if (t == rb) {
#pragma unroll
        for (int s = 0; s < kPB; ++s) x[s] = cmul(x[s], inv);
        x[j] = inv;
        st.used = true;
      } else if (t < n) {
#pragma unroll
        for (int s = 0; s < kPB; ++s) x[s] = cfms(v, cmul(pr[s], inv), x[s]);
        x[j] = cmul(make_double2(-v.x, -v.y), inv);
      }
      // buffer pb is posted again two steps later, after the next step's barrier
    }
  }
  if (t < n) {
#pragma unroll
    for (int s = 0; s < kPB; ++s) row[(size_t)s * n] = x[s];
  }
}

// this thread's 16-slot half h of its row: every panel step k < nb with multipliers Fs[k][row]
// and scaled pivot rows prow[k][slot]; the row that was the pivot row of step myj becomes
// prow[myj] minus the later steps; slots of local panel `skip` are left alone
__device__ __forceinline__ void update_half(double2* blk, int h, int t, int n, int nb, int myj, int skip,
                                            const double2* Fs, const double2* prow) {
  constexpr int kH = kNLC / 2;
  double2 a[kH];
#pragma unroll
  for (int s = 0; s < kH; ++s) a[s] = blk[(size_t)(kH * h + s) * n + t];
  int k0 = 0;
  if (myj >= 0) {
#pragma unroll
    for (int s = 0; s < kH; ++s)
      if (((kH * h + s) >> 3) != skip) a[s] = prow[myj * kNLC + kH * h + s];
    k0 = myj + 1;
  }
  for (int k = k0; k < nb; ++k) {
    const double2 f = Fs[k * n + t];
    if (myj < 0 || k > myj) {
#pragma unroll
      for (int s = 0; s < kH; ++s)
        if (((kH * h + s) >> 3) != skip) a[s] = cfms(f, prow[k * kNLC + kH * h + s], a[s]);
    }
  }
#pragma unroll
  for (int s = 0; s < kH; ++s) blk[(size_t)(kH * h + s) * n + t] = a[s];
}

__global__ void __launch_bounds__(kMaxN, 1) green_cluster_kernel(GreenArgs a, int cs, double2* ws) {
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smem[];
  const int n = a.n;
  const ClSmem L = cl_smem(n, a.n_neigh);
  double2* candrow = reinterpret_cast<double2*>(smem + L.candrow);
  double2* prow = reinterpret_cast<double2*>(smem + L.prow);         // [kPB][kNLC]
  int* pr_s = reinterpret_cast<int*>(smem + L.pr);
  double2* pinv_s = reinterpret_cast<double2*>(smem + L.pinv);
  int* piv = reinterpret_cast<int*>(smem + L.piv);
  double2* phase = reinterpret_cast<double2*>(smem + L.phase);
  double2* Fs = reinterpret_cast<double2*>(smem + L.fs);             // [kPB][n]
  double2* blk = reinterpret_cast<double2*>(smem + L.blk);           // [kNLC][n]
  ClState st;
  st.n = n;
  st.t = threadIdx.x;
  const int rank = (int)cl.block_rank();
  const int64_t cid = blockIdx.x / cs, ncl = gridDim.x / cs;
  // this cluster's workspace
  unsigned char* wsb = reinterpret_cast<unsigned char*>(ws) + cid * ws_cluster_bytes(n);
  double2* F = reinterpret_cast<double2*>(wsb);               // [2][kPB][n]
  double2* INV = F + 2 * kPB * (size_t)n;                     // [2][kPB]
  int* R = reinterpret_cast<int*>(INV + 2 * kPB);             // [2][kPB]
  const int npanels = (n + kPB - 1) / kPB;
  const int t = st.t;
  int pcount = 0;   // panels processed by this cluster so far (selects the workspace buffer)

  for (int64_t pl = cid; pl < a.np; pl += ncl) {
    // ---- point data ----------------------------------------------------------------
    const int64_t pg = a.p0 + pl;
    int64_t ktab = -1;
    double zr, zi, kx = 0, ky = 0, kz = 0;
    if (a.htab) {
      const int64_t ik = pg / a.n_e, ie = pg % a.n_e;
      ktab = ik;
      if (a.pts.kind == 0) {
        zr = a.zr;
        zi = a.zi + a.ylist[ie];
      } else {
        zr = a.zr + a.pts.x2[ie];
        zi = a.zi;
      }
    } else if (a.pts.kind == 0) {
      zr = a.zr;
      zi = a.zi + a.pts.y[pg];
      kx = a.pts.kp[3 * pg]; ky = a.pts.kp[3 * pg + 1]; kz = a.pts.kp[3 * pg + 2];
    } else if (a.pts.kind == 1) {
      const int64_t nep = pg / a.pts.nk, ik = pg % a.pts.nk;
      zr = a.zr + a.pts.x2[nep];
      zi = a.zi;
      kx = a.pts.kp[3 * ik]; ky = a.pts.kp[3 * ik + 1]; kz = a.pts.kp[3 * ik + 2];
    } else {
      zr = a.pts.z[pg].x;
      zi = a.pts.z[pg].y;
      kx = a.pts.kp[3 * pg]; ky = a.pts.kp[3 * pg + 1]; kz = a.pts.kp[3 * pg + 2];
    }
    kx += a.q[0]; ky += a.q[1]; kz += a.q[2];
    if (ktab < 0) {
      for (int nb = threadIdx.x; nb < a.n_neigh; nb += blockDim.x) {
        const double th = kx * a.R[3 * nb] + ky * a.R[3 * nb + 1] + kz * a.R[3 * nb + 2];
        double s, c;
        sincos(th, &s, &c);
        phase[nb] = make_double2(c, s);
      }
      __syncthreads();
    }
    // ---- A = z 1 - H(k) into the block: slot ls = 8 lp + c holds column 8 (lp cs + rank) + c
    for (int e = t; e < kNLC * n; e += blockDim.x) {
      const int ls = e / n, r = e - ls * n;
      const int j = ((ls / kPB) * cs + rank) * kPB + (ls % kPB);
      double2 v = make_double2(0, 0);
      if (j < n) {
        double2 h;
        if (ktab >= 0) {
          h = a.htab[ktab * ((int64_t)n * n) + (int64_t)r * n + j];
        } else {
          h = a.h0[(size_t)j * n + r];
          if (a.row_spin[r] == a.row_spin[j]) {
            const int orr = a.row_orb[r], oc = a.row_orb[j];
            const int pb = a.row_atom[r] * a.n_atoms + a.row_atom[j];
            for (int b = a.pair_start[pb]; b < a.pair_start[pb + 1]; ++b)
              h = cfma(phase[a.pair_neigh[b]], a.pair_t[(size_t)b * a.nmax * a.nmax + oc * a.nmax + orr], h);
          }
        }
        v = make_double2((r == j ? zr : 0.0) - h.x, (r == j ? zi : 0.0) - h.y);
      }
      blk[e] = v;
    }
    st.used = false;
    st.my_step = 0;
    __syncthreads();

    for (int P = 0; P < npanels; ++P, ++pcount) {
      const int buf = pcount & 1;
      const int owner = P % cs;
      const int nb = min(kPB, n - P * kPB);
      double2* Fb = F + (size_t)buf * kPB * n;
      const bool own = rank == owner;
      // ---- phase 1: the owner factorises the panel (slots 8 lp .. 8 lp + 7) ---------------
      if (own) {
        factor_panel(st, blk, kPB * (P / cs), candrow, Fb, INV + buf * kPB, R + buf * kPB, nb, a.status, pg);
        __threadfence();
      }
      cl.sync();
      // ---- phase 2: every CTA applies the panel's steps to its other columns ----------
      // the panel's multipliers go to shared memory first: one round of independent L2
      // loads instead of one per use
      if (t < nb) {
        pr_s[t] = __ldcg(R + buf * kPB + t);
        pinv_s[t] = ldcg2(INV + buf * kPB + t);
      }
      if (t < n) {
        double2 fv[kPB];
#pragma unroll
        for (int k = 0; k < kPB; ++k)
          if (k < nb) fv[k] = ldcg2(Fb + (size_t)k * n + t);
#pragma unroll
        for (int k = 0; k < kPB; ++k)
          if (k < nb) Fs[k * n + t] = fv[k];
      }
      __syncthreads();
      int myj = -1;   // the panel step whose pivot row is this thread's row
      for (int j = 0; j < nb; ++j)
        if (pr_s[j] == t) myj = j;
      if (myj >= 0) {
        st.used = true;
        st.my_step = P * kPB + myj;
      }
      if (t < nb) piv[P * kPB + t] = pr_s[t];
      // scaled pivot rows: thread t < 32 runs the eight-step recurrence for slot t, reading
      // the pivot rows' current entries from the block (not written before the barrier below)
      if (t < kNLC) {
        for (int j = 0; j < nb; ++j) {
          const int rj = pr_s[j];
          double2 x = blk[(size_t)t * n + rj];
          for (int k = 0; k < j; ++k) x = cfms(Fs[k * n + rj], prow[k * kNLC + t], x);
          prow[j * kNLC + t] = cmul(x, pinv_s[j]);
        }
      }
      __syncthreads();
      // the owner's panel slots were done in phase 1
      const int skip = own ? P / cs : -1;
      if (t < n) {
        update_half(blk, 0, t, n, nb, myj, skip, Fs, prow);
        update_half(blk, 1, t, n, nb, myj, skip, Fs, prow);
      }
      // prow, pr_s, pinv_s and Fs are rewritten by the next panel after this barrier; the
      // next panel's owner reads its panel slots of the block after it as well
      __syncthreads();
    }
    // ---- output: G[step(t)][piv(j)] = X[t][slot] -> column piv(j), row step(t) ------------
    // rows are permuted in place: every thread reads its 32 entries before any is written
    double2 keep[kNLC / 2];
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
      if (t < n) {
#pragma unroll
        for (int s = 0; s < kNLC / 2; ++s) keep[s] = blk[(size_t)(kNLC / 2 * hh + s) * n + t];
      }
      __syncthreads();
      if (t < n) {
#pragma unroll
        for (int s = 0; s < kNLC / 2; ++s) blk[(size_t)(kNLC / 2 * hh + s) * n + st.my_step] = keep[s];
      }
      __syncthreads();
    }
    double2* out = a.out + pl * ((int64_t)n * n);
    for (int ls = 0; ls < kNLC; ++ls) {
      const int j = ((ls / kPB) * cs + rank) * kPB + (ls % kPB);
      if (j >= n) continue;
      const int col = piv[j];
      for (int r = t; r < n; r += blockDim.x) out[(int64_t)col * n + r] = blk[(size_t)ls * n + r];
    }
    // the next point rewrites the block and piv: this CTA is done with them
    __syncthreads();
  }
}

}  // namespace

int green_cluster_supported(int n, int mode) { return n >= 1 && n <= kMaxN && mode == MODE_RAW; }

int green_cluster_size(int n) {
  const int npanels = (n + kPB - 1) / kPB;
  return std::min(kMaxCS, std::max(1, (npanels + kNLC / kPB - 1) / (kNLC / kPB)));
}

size_t green_cluster_ws_bytes(int n, int num_sms) { return ws_cluster_bytes(n) * (size_t)std::max(num_sms, 1); }

cudaError_t launch_green_cluster(const GreenArgs& a, int num_sms, cudaStream_t s) {
  if (!green_cluster_supported(a.n, a.mode) || a.out2) return cudaErrorInvalidValue;
  if (a.np <= 0) return cudaSuccess;
  const int cs = green_cluster_size(a.n);
  if (((a.n + kPB - 1) / kPB + cs - 1) / cs * kPB > kNLC) return cudaErrorInvalidValue;
  const int threads = (a.n + 31) / 32 * 32;
  const size_t smem = cl_smem(a.n, a.n_neigh).total;
  cudaError_t e = cudaFuncSetAttribute(green_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (cs > 8) {
    e = cudaFuncSetAttribute(green_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
  }
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3(cs * num_sms, 1, 1);
  int max_clusters = 0;
  e = cudaOccupancyMaxActiveClusters(&max_clusters, green_cluster_kernel, &cfg);
  if (e != cudaSuccess) return e;
  if (max_clusters < 1) return cudaErrorInvalidConfiguration;
  // the workspace holds num_sms clusters (more than can be resident)
  const int64_t ncl = std::min<int64_t>(std::min(max_clusters, num_sms), a.np);
  if (!a.ws || a.ws_bytes < ws_cluster_bytes(a.n) * (size_t)ncl) return cudaErrorInvalidValue;
  cfg.gridDim = dim3((unsigned)(ncl * cs), 1, 1);
  return cudaLaunchKernelEx(&cfg, green_cluster_kernel, a, cs, reinterpret_cast<double2*>(a.ws));
}

}  // namespace tg
