// Batched G(k, z) = (z - h0 - H(k))^-1 for any dimension up to 288: one thread-block
// cluster per matrix, Gauss-Jordan with partial pivoting across distributed shared memory.
//
// The matrix of one (k, z) point is too large for one SM at the reference's larger
// systems (a 288 x 288 complex matrix is 1.33 MB), so a cluster of CS <= 8 CTAs shares it:
//   * column j lives in CTA j % CS (local column j / CS), row t in thread t of every CTA,
//     so each thread holds one row segment of up to kNLC = 32 complex entries in
//     registers (288 rows x 9 CTAs x 32 columns at dimH = 288; 9 warps per CTA leave 168
//     registers per thread, so the segment is 128 of them);
//   * step p (pivot column p, owned by CTA p % CS): the owner has already published the
//     column's values and its pivot row r (largest |Re| + |Im| among the rows not yet
//     used, first index on ties -- the izamax choice of zgetrf) into every CTA's shared
//     memory; thread r scales its row segment by 1 / a_rp, every other row subtracts its
//     multiple of the scaled segment, and column p becomes (-a_tp / a_rp, 1 / a_rp on row r);
//   * lookahead: the owner of column p + 1 updates that column first, searches its pivot
//     and writes it into the other CTAs (st through the cluster window) before updating its
//     remaining columns; one cluster barrier per step publishes it (two buffers);
//   * a CTA's columns become pivot columns in local order, so the next one is always kept
//     in register slot 0 by rotating the segment after each (no dynamic register index);
//   * rows are never swapped: the result X holds G[step(t)][piv(j)] at (t, j), where
//     step(t) is the step whose pivot row was t (the same implicit permutation as the
//     single-SM kernels); the output stage unpermutes through shared memory and writes
//     G column-major per point (MODE_RAW), one column per coalesced store run.
// The kernel is persistent: the grid holds as many clusters as fit, each walking the
// point range.  This replaces invers = zgetrf + zgetri (mod_tools.F90:796-829) inside
// green (mod_greenfunction.F90:19-75) for dimensions the single-SM kernels do not cover;
// H(k) comes from a tabulated row (calchk + hamilt_local) or is summed in the kernel.
#include "tg_internal.cuh"

#include <cooperative_groups.h>

#include <algorithm>

namespace tg {

namespace {

namespace cg = cooperative_groups;

constexpr int kNLC = 32;       // local columns per CTA (registers per row segment)
constexpr int kMaxN = 288;     // one row per thread
constexpr int kMaxCS = 9;      // cluster size (9 > 8: non-portable, enabled at launch)
constexpr int kMaxWarps = kMaxN / 32;

struct ClSmem {
  size_t fcol, pidx, prow, candv, candr, piv, phase, stage, total;
};

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline ClSmem cl_smem(int n, int n_neigh) {
  ClSmem L;
  size_t o = 0;
  L.fcol = o;  o = al16(o + sizeof(double2) * 2 * (size_t)n);
  L.pidx = o;  o = al16(o + sizeof(int) * 4);
  L.prow = o;  o = al16(o + sizeof(double2) * kNLC);
  L.candv = o; o = al16(o + sizeof(double) * kMaxWarps);
  L.candr = o; o = al16(o + sizeof(int) * kMaxWarps);
  L.piv = o;   o = al16(o + sizeof(int) * (size_t)n);
  L.phase = o; o = al16(o + sizeof(double2) * (size_t)(n_neigh > 0 ? n_neigh : 1));
  L.stage = o; o = al16(o + sizeof(double2) * (size_t)kNLC * n);
  L.total = o;
  return L;
}

struct ClState {
  double2* fcol;       // [2][n] pivot column of the step (this CTA's copy)
  int* pidx;           // [2] pivot row of the step
  double2* prow;       // [kNLC] this CTA's part of the scaled pivot row
  double* candv;
  int* candr;
  int* piv;            // [n] step -> pivot row
  int n, cs, rank, t;
  int rot;             // left rotations of the row segment so far (see gj_step)
  bool used;           // this thread's row has been a pivot row
  int my_step;         // step at which it became one
};

// |Re| + |Im| argmax over the CTA's unused rows (first index on ties); all threads call it
__device__ __forceinline__ int cta_argmax(const ClState& st, double2 v) {
  double best = (st.t < st.n && !st.used) ? fabs(v.x) + fabs(v.y) : -1.0;
  int bi = st.t;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, off);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
    if (ob > best || (ob == best && oi < bi)) {
      best = ob;
      bi = oi;
    }
  }
  const int warp = st.t >> 5, lane = st.t & 31;
  if (lane == 0) {
    st.candv[warp] = best;
    st.candr[warp] = bi;
  }
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  double b2 = -2.0;
  int i2 = 0x7fffffff;
  for (int w = 0; w < nw; ++w) {
    const double cv = st.candv[w];
    const int cr = st.candr[w];
    if (cv > b2 || (cv == b2 && cr < i2)) {
      b2 = cv;
      i2 = cr;
    }
  }
  return i2;
}

// publish column values (one per thread) and the pivot row into buffer `buf` of every CTA
__device__ __forceinline__ void publish(const ClState& st, cg::cluster_group& cl, int buf, double2 v, int r) {
  for (int d = 0; d < st.cs; ++d) {
    double2* rf = cl.map_shared_rank(st.fcol, d);
    if (st.t < st.n) rf[buf * st.n + st.t] = v;
    if (st.t == 0) {
      int* rp = cl.map_shared_rank(st.pidx, d);
      rp[buf] = r;
    }
  }
}

// one elimination step p.  The CTA's next own pivot column is always A[0]: after its
// column has been the pivot column, the owner rotates its row segment left by one
// (st.rot counts the rotations, physical slot i holds local column (i + rot) % kNLC).
__device__ __forceinline__ void gj_step(ClState& st, cg::cluster_group& cl, double2 (&A)[kNLC], int p, int* status,
                                        int64_t point) {
  const int buf = p & 1;
  const int r = st.pidx[buf];
  const double2 fi = st.t < st.n ? st.fcol[buf * st.n + st.t] : make_double2(0, 0);
  const double2 pv = st.fcol[buf * st.n + r];
  if (pv.x == 0.0 && pv.y == 0.0 && st.rank == 0 && st.t == 0) atomicMin(status, (int)(point + 1));
  const double2 inv = crecip_fast(pv);
  const int q = p % st.cs;
  const bool own_p = q == st.rank;
  if (st.t == 0) st.piv[p] = r;
  if (st.t == r) {
#pragma unroll
    for (int lc = 0; lc < kNLC; ++lc) {
      const double2 v = cmul(A[lc], inv);
      st.prow[lc] = v;
      A[lc] = v;
    }
    if (own_p) A[0] = inv;
    st.used = true;
    st.my_step = p;
  }
  __syncthreads();
  const bool upd = st.t < st.n && st.t != r;
  // lookahead: the owner of column p + 1 updates it first (slot 0, or slot 1 when the
  // same CTA also owns column p, i.e. a one-CTA cluster), searches its pivot and
  // publishes it before updating its other columns
  const bool own_next = p + 1 < st.n && (p + 1) % st.cs == st.rank;
  const bool one = st.cs == 1;
  if (own_next) {
    double2 v = one ? A[1] : A[0];
    if (upd) v = cfms(fi, one ? st.prow[1] : st.prow[0], v);
    if (one) A[1] = v; else A[0] = v;
    const int rn = cta_argmax(st, v);
    publish(st, cl, buf ^ 1, v, rn);
  }
  if (upd) {
    const bool skip0 = own_next && !one, skip1 = own_next && one;
#pragma unroll
    for (int lc = 0; lc < kNLC; ++lc) {
      if ((lc == 0 && skip0) || (lc == 1 && skip1)) continue;
      A[lc] = cfms(fi, st.prow[lc], A[lc]);
    }
    if (own_p) A[0] = cmul(make_double2(-fi.x, -fi.y), inv);
  }
  if (own_p) {
    const double2 a0 = A[0];
#pragma unroll
    for (int lc = 0; lc + 1 < kNLC; ++lc) A[lc] = A[lc + 1];
    A[kNLC - 1] = a0;
    ++st.rot;
  }
  cl.sync();
}

__global__ void __launch_bounds__(kMaxN, 1) green_cluster_kernel(GreenArgs a, int cs) {
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smem[];
  const int n = a.n;
  const ClSmem L = cl_smem(n, a.n_neigh);
  ClState st;
  st.fcol = reinterpret_cast<double2*>(smem + L.fcol);
  st.pidx = reinterpret_cast<int*>(smem + L.pidx);
  st.prow = reinterpret_cast<double2*>(smem + L.prow);
  st.candv = reinterpret_cast<double*>(smem + L.candv);
  st.candr = reinterpret_cast<int*>(smem + L.candr);
  st.piv = reinterpret_cast<int*>(smem + L.piv);
  double2* phase = reinterpret_cast<double2*>(smem + L.phase);
  double2* stage = reinterpret_cast<double2*>(smem + L.stage);
  st.n = n;
  st.cs = cs;
  st.rank = (int)cl.block_rank();
  st.t = threadIdx.x;
  const int64_t cid = blockIdx.x / cs, ncl = gridDim.x / cs;

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
    // ---- A = z 1 - H(k): row t, columns j = lc * cs + rank ------------------------------
    // built through the stage buffer ([lc][row]) so that no address lives beside the row
    // segment in registers
    const int t = st.t;
    for (int e = t; e < kNLC * n; e += blockDim.x) {
      const int lc = e / n, r = e - lc * n;
      const int j = lc * cs + st.rank;
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
      stage[e] = v;
    }
    __syncthreads();
    double2 A[kNLC];
#pragma unroll
    for (int lc = 0; lc < kNLC; ++lc) A[lc] = t < n ? stage[lc * n + t] : make_double2(0, 0);
    st.used = false;
    st.my_step = 0;
    st.rot = 0;
    // ---- pivot of column 0 (CTA 0, local column 0), published before the first step ----
    if (st.rank == 0) {
      const int r0 = cta_argmax(st, A[0]);
      publish(st, cl, 0, A[0], r0);
    }
    cl.sync();
    for (int p = 0; p < n; ++p) gj_step(st, cl, A, p, a.status, pg);
    // ---- output: G[step(t)][piv(j)] = A[t][lc] -> column piv(j), row step(t) ---------------
#pragma unroll
    for (int i = 0; i < kNLC; ++i)
      if (t < n) stage[((i + st.rot) % kNLC) * n + st.my_step] = A[i];
    __syncthreads();
    double2* out = a.out + pl * ((int64_t)n * n);
    for (int lc = 0; lc < kNLC; ++lc) {
      const int j = lc * cs + st.rank;
      if (j >= n) break;
      const int col = st.piv[j];
      for (int r = t; r < n; r += blockDim.x) out[(int64_t)col * n + r] = stage[lc * n + r];
    }
    // the next point rewrites stage, fcol[0] and pidx[0]: every CTA is done with them
    cl.sync();
  }
}

}  // namespace

int green_cluster_supported(int n, int mode) { return n >= 1 && n <= kMaxN && mode == MODE_RAW; }

int green_cluster_size(int n) { return std::min(kMaxCS, std::max(1, (n + kNLC - 1) / kNLC)); }

cudaError_t launch_green_cluster(const GreenArgs& a, int num_sms, cudaStream_t s) {
  if (!green_cluster_supported(a.n, a.mode) || a.out2) return cudaErrorInvalidValue;
  if (a.np <= 0) return cudaSuccess;
  const int cs = green_cluster_size(a.n);
  if ((a.n + cs - 1) / cs > kNLC) return cudaErrorInvalidValue;
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
  const int64_t ncl = std::min<int64_t>(max_clusters, a.np);
  cfg.gridDim = dim3((unsigned)(ncl * cs), 1, 1);
  return cudaLaunchKernelEx(&cfg, green_cluster_kernel, a, cs);
}

}  // namespace tg
