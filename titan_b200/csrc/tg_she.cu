// Disturbance-response integrand of eintshe (source/eintshe.F90:2-309).
//
// Per (k, E) point, with V = dtdk(k) = sum_n i (u.R_n) t_n exp(i k.R_n) in the
// spinless orbital space (source/dtdksub.F90:2-28; rows: the neighbour's basis
// site, columns: site i), the integrand on the diagonal site blocks is
//   imaginary axis (eintshe.F90:104-179):
//     df[(s, i, mu, nu), s'] += w [ G1^{ab}(i nu, j g) V(j g, l x) G2^{cd}(l x, i mu)
//                                 + conj(G2^{a'b'}(i mu, l x)) V(j g, l x) conj(G1^{c'd'}(j g, i nu)) ]
//   real axis (eintshe.F90:226-249):
//     df[(s, i, mu, nu), s'] += -i w (G1 - G1^+)^{ab}(i nu, j g) V(j g, l x) (G2^+)^{cd}(l x, i mu)
// where the four spins (a, b, c, d) of each term are fixed by (s, s') through
// the reference's tables.  G1 = G(k + q, E + e), G2 = G(k, E).
//
// Work split: one CTA per point at a time (grid-stride), V built in shared
// memory from per-neighbour phases, then two small products per term:
// Y^b = L[:, spin b] V (n x no) and Z = Y^b R[spin c, :] restricted to the
// output entries, which form n_i x n_i blocks per (sigma, s', site).  Both
// products are register-tiled (2 x 3 and 3 x 3 outputs per thread), so each
// operand read from shared memory feeds two to three complex FMAs;
// shared-memory bandwidth bounds the kernel.  Each CTA owns a slice (4 dimens
// complex) of a per-CTA global array, so successive launches (passes)
// accumulate without atomics; the slices are summed once at the end.  Three
// variants: when every second-stage tile has its own thread (two spd sites at
// 288 threads), the slice entries stay in the owning threads' registers for the
// launch (she_kernel_reg); else, when they fit (dimH up to about 48 for small
// dimens), both Green functions are staged row-major in shared memory and the
// slice is held there; larger cells read the column-major inversion output
// through L1 / L2 and add into the slice in place.
#include "tg_internal.cuh"

#include <algorithm>

namespace tg {

namespace {

struct SheArgs {
  const double2* G1 = nullptr;    // [np][n][n] column-major, G(k + q, E + e)
  const double2* G2 = nullptr;    // [np][n][n] column-major, G(k, E)
  int64_t p0 = 0, np = 0;
  PointSet pts;                   // kind 0 (imaginary list) or 1 (real axis)
  int n = 0, no = 0, dimens = 0, n_neigh = 0, nmax = 0, n_atoms = 0;
  const double* R = nullptr;
  const int* pair_start = nullptr;
  const int* pair_neigh = nullptr;
  const double2* pair_t = nullptr;
  const int* tab = nullptr;       // [4][no]: full row (spin up), full row (spin down), site, orbital in site
  const int* ia = nullptr;        // first row of each site
  const int* norb = nullptr;
  const int* decode = nullptr;    // [dimens] sigma | i << 2 | mu << 12 | nu << 18
  const int* ztiles = nullptr;    // second-stage tiles: sigma | s' << 2 | i << 4 | x0 << 14 | y0 << 20
  int n_ztiles = 0;
  const int* rowoff = nullptr;    // first df row of each site
  int real_axis = 0;
  double ue[3] = {0, 0, 0};
  unsigned char spins[3][16] = {};   // term t, (s * 4 + s') -> a << 3 | b << 2 | c << 1 | d (0 = up)
  double2* partial = nullptr;        // [gridDim][4 dimens], df(row, s') at s' dimens + row
  int64_t n_e = 0, nk_tab = 0;       // k-major order of a tabulated pass (n_e > 0)
  const double* klist = nullptr;
};

// 288 threads: the 288 second-stage tiles of two spd sites (32 blocks of 3 x 3 tiles) and
// the 216 first-stage tiles at dimH 36 each take one round of the CTA
constexpr int kSheThreads = 288;

struct SheSmem {
  int s1, s2, m, y, acc, ph, tab;   // offsets in double2 units (tab: in bytes)
  size_t bytes;
};

// Row strides of the staged Green functions and of Y: odd, so the 16-byte reads of a
// quarter warp on rows a few apart fall into distinct bank groups.
__host__ __device__ inline int she_sst(int n) { return n | 1; }
__host__ __device__ inline int she_yst(int no) { return no | 1; }

// Shared-memory layout.  STAGED: both Green functions (row-major, stride she_sst) and
// the df partial live in shared memory; otherwise they are read from / accumulated in
// global memory (L1 / L2) and only V, Y and the tables are staged.  V^T is read from
// V with swapped indices.
__host__ __device__ inline SheSmem she_layout(int n, int dimens, int n_neigh, bool staged, bool acc_smem = true) {
  const int no = n / 2;
  SheSmem L;
  int o = 0;
  L.s1 = o; o += staged ? n * she_sst(n) : 0;
  L.s2 = o; o += staged ? n * she_sst(n) : 0;
  L.m = o; o += no * no;
  L.y = o; o += 2 * n * she_yst(no);
  L.acc = o; o += staged && acc_smem ? 4 * dimens : 0;
  L.ph = o; o += n_neigh > 0 ? n_neigh : 1;
  L.tab = o * (int)sizeof(double2);
  L.bytes = (size_t)L.tab + sizeof(int) * 4 * (size_t)no;
  return L;
}

// n x n operand of a term, element (r, c).  Shared-memory operands are row-major
// and already transformed; global operands are the column-major inversion output
// with the transform applied on read.
struct RowMajor {
  const double2* p;
  int n;
  __device__ __forceinline__ double2 operator()(int r, int c) const { return p[r * n + c]; }
};
enum GlobKind : int { GK_G = 0, GK_CONJ = 1, GK_ANTI = 2, GK_DAGGER = 3 };
struct ColMajor {
  const double2* g;
  int n, kind;   // G, conj(G), G - G^+, G^+
  __device__ __forceinline__ double2 operator()(int r, int c) const {
    const double2 x = g[(size_t)c * n + r];
    if (kind == GK_G) return x;
    if (kind == GK_CONJ) return make_double2(x.x, -x.y);
    const double2 xt = g[(size_t)r * n + c];
    if (kind == GK_ANTI) return make_double2(x.x - xt.x, x.y + xt.y);
    return make_double2(xt.x, -xt.y);
  }
};

// One sandwich term.  M: no x no row-major (the middle factor as used: V or V^T).
// Z(r, col) = sum_{o1, o2} L(r, row_b(o2)) M(o2, o1) R(row_c(o1), col) for the
// output rows (r, col) of each df entry; acc[s' dimens + row] += f Z, in two stages:
// Y^b = L[:, spin b] M for both spins b (2 n x no), then Z from Y and R.
// First stage, register-tiled: each thread computes a 2 x 3 tile (rows r, columns o1) of
// Y^b, so five L and M values loaded per o2 feed six complex FMAs (2 x 18 x 6 = 216 tiles
// at n = 36: one round of the CTA).
template <class LM>
__device__ void she_y_tiled(const SheArgs& a, LM L, const double2* M, bool mt, double2* Y, const int* tab) {
  const int n = a.n, no = a.no, yst = she_yst(no);
  const int tr = (n + 1) / 2, to = (no + 2) / 3;
  for (int t = threadIdx.x; t < 2 * tr * to; t += blockDim.x) {
    const int b = t / (tr * to), r0 = 2 * ((t / to) % tr), q0 = 3 * (t % to);
    const int* rowb = tab + b * no;
    double2 z[2][3];
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) z[k][l] = make_double2(0.0, 0.0);
    for (int o2 = 0; o2 < no; ++o2) {
      const int cb = rowb[o2];
      double2 lv[2], mv[3];
#pragma unroll
      for (int k = 0; k < 2; ++k) lv[k] = r0 + k < n ? L(r0 + k, cb) : make_double2(0.0, 0.0);
#pragma unroll
      for (int l = 0; l < 3; ++l)
        mv[l] = q0 + l < no ? (mt ? M[(q0 + l) * no + o2] : M[o2 * no + q0 + l]) : make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int l = 0; l < 3; ++l) z[k][l] = cfma(lv[k], mv[l], z[k][l]);
    }
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l)
        if (r0 + k < n && q0 + l < no) Y[(b * n + r0 + k) * yst + q0 + l] = z[k][l];
  }
  __syncthreads();
}

// Second stage, register-tiled: the df entries of one (sigma, s', site i) form an n_i x n_i
// block Z(x, y) = sum_o1 Y^b(ia + sa n_i + x, o1) R(row_c(o1), ia + sd n_i + y) with
// (mu, nu) = (y, x) when rows_are_nu else (x, y); each thread takes 3 x 3 tiles of blocks.
template <class RM>
__device__ void she_z_tiled(const SheArgs& a, const double2* Y, RM R, double2* acc, const int* tab,
                            const unsigned char* spins, double2 f, bool rows_are_nu) {
  const int n = a.n, no = a.no, D = a.dimens, yst = she_yst(no);
  for (int t = threadIdx.x; t < a.n_ztiles; t += blockDim.x) {
    const int code = a.ztiles[t];
    const int sigma = code & 3, sp = (code >> 2) & 3, i = (code >> 4) & 1023;
    const int x0 = (code >> 14) & 63, y0 = (code >> 20) & 63;
    const int sc = spins[sigma * 4 + sp];
    const int sa = (sc >> 3) & 1, b = (sc >> 2) & 1, c = (sc >> 1) & 1, sd = sc & 1;
    const int ni = a.norb[i], ia = a.ia[i];
    const double2* Yb = Y + (b * n + ia + sa * ni) * yst;
    const int* rowc = tab + c * no;
    const int col0 = ia + sd * ni + y0;
    double2 z[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) z[k][l] = make_double2(0.0, 0.0);
    for (int o1 = 0; o1 < no; ++o1) {
      const int rc = rowc[o1];
      double2 yv[3], rv[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) yv[k] = x0 + k < ni ? Yb[(x0 + k) * yst + o1] : make_double2(0.0, 0.0);
#pragma unroll
      for (int l = 0; l < 3; ++l) rv[l] = y0 + l < ni ? R(rc, col0 + l) : make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int l = 0; l < 3; ++l) z[k][l] = cfma(yv[k], rv[l], z[k][l]);
    }
    const int base = sp * D + a.rowoff[i] + sigma;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) {
        if (x0 + k >= ni || y0 + l >= ni) continue;
        const int mu = rows_are_nu ? y0 + l : x0 + k, nu = rows_are_nu ? x0 + k : y0 + l;
        const int o = base + 4 * (mu * ni + nu);
        acc[o] = cfma(f, z[k][l], acc[o]);
      }
  }
}

// Second stage with the df entries in registers: the thread owns tile t (one tile per
// thread) for the whole launch.  Slot (k, l) holds the entry (mu, nu) = (y0 + l, x0 + k).
// A term with rows on nu (rows_are_nu) computes tile (x0, y0) as stored; a term with
// rows on mu computes the mirrored tile (y0, x0), whose element (k', l') is that same
// entry for (k', l') = (l, k), so both terms add into the same slots.
template <class RM>
__device__ void she_z_reg(const SheArgs& a, const double2* Y, RM R, double2 (&racc)[9], const int* tab,
                          const unsigned char* spins, double2 f, bool rows_are_nu) {
  const int n = a.n, no = a.no, yst = she_yst(no);
  const int t = threadIdx.x;
  if (t < a.n_ztiles) {
    const int code = a.ztiles[t];
    const int sigma = code & 3, sp = (code >> 2) & 3, i = (code >> 4) & 1023;
    const int tx = (code >> 14) & 63, ty = (code >> 20) & 63;
    const int x0 = rows_are_nu ? tx : ty, y0 = rows_are_nu ? ty : tx;
    const int sc = spins[sigma * 4 + sp];
    const int sa = (sc >> 3) & 1, b = (sc >> 2) & 1, c = (sc >> 1) & 1, sd = sc & 1;
    const int ni = a.norb[i], ia = a.ia[i];
    const double2* Yb = Y + (b * n + ia + sa * ni) * yst;
    const int* rowc = tab + c * no;
    const int col0 = ia + sd * ni + y0;
    double2 z[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) z[k][l] = make_double2(0.0, 0.0);
    for (int o1 = 0; o1 < no; ++o1) {
      const int rc = rowc[o1];
      double2 yv[3], rv[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) yv[k] = x0 + k < ni ? Yb[(x0 + k) * yst + o1] : make_double2(0.0, 0.0);
#pragma unroll
      for (int l = 0; l < 3; ++l) rv[l] = y0 + l < ni ? R(rc, col0 + l) : make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int l = 0; l < 3; ++l) z[k][l] = cfma(yv[k], rv[l], z[k][l]);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) {
        const int slot = rows_are_nu ? 3 * k + l : 3 * l + k;
        racc[slot] = cfma(f, z[k][l], racc[slot]);   // invalid slots only ever add zeros
      }
  }
}

// df entry of register slot (k, l) of this thread's tile, or -1
__device__ __forceinline__ int she_slot_entry(const SheArgs& a, int slot) {
  const int t = threadIdx.x;
  if (t >= a.n_ztiles) return -1;
  const int code = a.ztiles[t];
  const int sigma = code & 3, sp = (code >> 2) & 3, i = (code >> 4) & 1023;
  const int x0 = (code >> 14) & 63, y0 = (code >> 20) & 63;
  const int k = slot / 3, l = slot % 3, ni = a.norb[i];
  if (x0 + k >= ni || y0 + l >= ni) return -1;
  const int mu = y0 + l, nu = x0 + k;
  return sp * a.dimens + a.rowoff[i] + sigma + 4 * (mu * ni + nu);
}

// the term with the df slice in memory (shared or global), both stages register-tiled
template <class LM, class RM>
__device__ void she_term_reg(const SheArgs& a, LM L, const double2* M, bool mt, RM R, double2* Y,
                             double2 (&racc)[9], const int* tab, const unsigned char* spins, double2 f,
                             bool rows_are_nu) {
  she_y_tiled(a, L, M, mt, Y, tab);
  she_z_reg(a, Y, R, racc, tab, spins, f, rows_are_nu);
  __syncthreads();
}

template <class LM, class RM>
__device__ void she_term(const SheArgs& a, LM L, const double2* M, bool mt, RM R, double2* Y, double2* acc,
                         const int* tab, const unsigned char* spins, double2 f, bool rows_are_nu) {
  she_y_tiled(a, L, M, mt, Y, tab);
  she_z_tiled(a, Y, R, acc, tab, spins, f, rows_are_nu);
  __syncthreads();
}

// STAGED: Green functions in shared memory.  REG (staged only, at most one second-stage
// tile per thread): each thread keeps its tile's df entries in registers for the whole
// launch, and the df slice leaves shared memory (no read-modify-write there, whose
// 16-byte accesses of a quarter warp fell into two bank groups).
template <bool STAGED, bool REG>
__device__ __forceinline__ void she_body(const SheArgs& a) {
  static_assert(STAGED || !REG, "register slices only in the staged kernel");
  extern __shared__ __align__(16) unsigned char smem[];
  const int n = a.n, no = a.no, D = a.dimens;
  const SheSmem L = she_layout(n, D, a.n_neigh, STAGED, !REG);
  double2* base = reinterpret_cast<double2*>(smem);
  double2* S1 = base + L.s1;
  double2* S2 = base + L.s2;
  double2* M = base + L.m;
  double2* Y = base + L.y;
  const int sst = she_sst(n);
  double2* ph = base + L.ph;
  int* tab = reinterpret_cast<int*>(smem + L.tab);
  double2* mine = a.partial + (size_t)blockIdx.x * 4 * D;
  double2* acc = STAGED && !REG ? base + L.acc : mine;
  double2 racc[9];
  if (REG) {
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      const int o = she_slot_entry(a, j);
      racc[j] = o >= 0 ? mine[o] : make_double2(0.0, 0.0);
    }
  } else if (STAGED) {
    for (int e = threadIdx.x; e < 4 * D; e += blockDim.x) acc[e] = mine[e];
  }
  for (int e = threadIdx.x; e < 4 * no; e += blockDim.x) tab[e] = a.tab[e];
  __syncthreads();
  for (int64_t pl = blockIdx.x; pl < a.np; pl += gridDim.x) {
    const int64_t p = a.p0 + pl;
    double kx, ky, kz, w;
    if (a.n_e > 0) {
      const int64_t ik = p / a.n_e, ie = p % a.n_e;
      kx = a.klist[3 * ik];
      ky = a.klist[3 * ik + 1];
      kz = a.klist[3 * ik + 2];
      w = a.pts.kind == 0 ? a.pts.w[ie * a.nk_tab + ik] : a.pts.p2[ie] * a.pts.w[ik];
    } else if (a.pts.kind == 0) {
      kx = a.pts.kp[3 * p];
      ky = a.pts.kp[3 * p + 1];
      kz = a.pts.kp[3 * p + 2];
      w = a.pts.w[p];
    } else {
      const int64_t nep = p / a.pts.nk, ik = p % a.pts.nk;
      kx = a.pts.kp[3 * ik];
      ky = a.pts.kp[3 * ik + 1];
      kz = a.pts.kp[3 * ik + 2];
      w = a.pts.p2[nep] * a.pts.w[ik];
    }
    // i (u.R) exp(i k.R) per neighbour cell
    for (int nb = threadIdx.x; nb < a.n_neigh; nb += blockDim.x) {
      const double* Rn = a.R + 3 * nb;
      const double th = kx * Rn[0] + ky * Rn[1] + kz * Rn[2];
      const double ur = a.ue[0] * Rn[0] + a.ue[1] * Rn[1] + a.ue[2] * Rn[2];
      double sn, cs;
      sincos(th, &sn, &cs);
      ph[nb] = make_double2(-ur * sn, ur * cs);
    }
    const double2* g1 = a.G1 + pl * (int64_t)n * n;
    const double2* g2 = a.G2 + pl * (int64_t)n * n;
    if (STAGED) {
      // Green functions of the point, row-major; real axis: S1 = G1 - G1^+, S2 = G2^+
      if (!a.real_axis) {
        for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
          const int c = e / n, r = e % n;
          S1[r * sst + c] = g1[e];
          S2[r * sst + c] = g2[e];
        }
      } else {
        for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
          const int r = e / n, c = e % n;
          const double2 x = g1[(size_t)c * n + r], xt = g1[(size_t)r * n + c];
          S1[r * sst + c] = make_double2(x.x - xt.x, x.y + xt.y);
          const double2 y = g2[(size_t)r * n + c];
          S2[r * sst + c] = make_double2(y.x, -y.y);
        }
      }
    }
    __syncthreads();
    // V(rr, cc): rr on the neighbour's basis site, cc on site i
    for (int e = threadIdx.x; e < no * no; e += blockDim.x) {
      const int rr = e / no, cc = e % no;
      const int sj = tab[2 * no + rr], si = tab[2 * no + cc];
      const int orr = tab[3 * no + rr], occ = tab[3 * no + cc];
      const int pb = sj * a.n_atoms + si;
      double2 v = make_double2(0, 0);
      for (int b = a.pair_start[pb]; b < a.pair_start[pb + 1]; ++b)
        v = cfma(ph[a.pair_neigh[b]], a.pair_t[(size_t)b * a.nmax * a.nmax + occ * a.nmax + orr], v);
      M[rr * no + cc] = v;
    }
    __syncthreads();
    if (REG) {
      if (!a.real_axis) {
        she_term_reg(a, RowMajor{S1, sst}, M, false, RowMajor{S2, sst}, Y, racc, tab, a.spins[0],
                     make_double2(w, 0.0), true);
        for (int e = threadIdx.x; e < n * sst; e += blockDim.x) {
          S1[e].y = -S1[e].y;
          S2[e].y = -S2[e].y;
        }
        __syncthreads();
        she_term_reg(a, RowMajor{S2, sst}, M, true, RowMajor{S1, sst}, Y, racc, tab, a.spins[1],
                     make_double2(w, 0.0), false);
      } else {
        she_term_reg(a, RowMajor{S1, sst}, M, false, RowMajor{S2, sst}, Y, racc, tab, a.spins[2],
                     make_double2(0.0, -w), true);
      }
    } else if (STAGED) {
      if (!a.real_axis) {
        she_term(a, RowMajor{S1, sst}, M, false, RowMajor{S2, sst}, Y, acc, tab, a.spins[0], make_double2(w, 0.0),
                 true);
        for (int e = threadIdx.x; e < n * sst; e += blockDim.x) {
          S1[e].y = -S1[e].y;
          S2[e].y = -S2[e].y;
        }
        __syncthreads();
        she_term(a, RowMajor{S2, sst}, M, true, RowMajor{S1, sst}, Y, acc, tab, a.spins[1], make_double2(w, 0.0),
                 false);
      } else {
        she_term(a, RowMajor{S1, sst}, M, false, RowMajor{S2, sst}, Y, acc, tab, a.spins[2], make_double2(0.0, -w),
                 true);
      }
    } else {
      if (!a.real_axis) {
        she_term(a, ColMajor{g1, n, GK_G}, M, false, ColMajor{g2, n, GK_G}, Y, acc, tab, a.spins[0], make_double2(w, 0.0),
                 true);
        she_term(a, ColMajor{g2, n, GK_CONJ}, M, true, ColMajor{g1, n, GK_CONJ}, Y, acc, tab, a.spins[1],
                 make_double2(w, 0.0), false);
      } else {
        she_term(a, ColMajor{g1, n, GK_ANTI}, M, false, ColMajor{g2, n, GK_DAGGER}, Y, acc, tab, a.spins[2],
                 make_double2(0.0, -w), true);
      }
    }
  }
  if (REG) {
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      const int o = she_slot_entry(a, j);
      if (o >= 0) mine[o] = racc[j];
    }
  } else if (STAGED) {
    for (int e = threadIdx.x; e < 4 * D; e += blockDim.x) mine[e] = acc[e];
  }
}

template <bool STAGED>
__global__ void __launch_bounds__(kSheThreads) she_kernel(SheArgs a) {
  she_body<STAGED, false>(a);
}

// two CTAs per SM: registers capped at 65 536 / (2 x 288)
__global__ void __launch_bounds__(kSheThreads, 2) she_kernel_reg(SheArgs a) {
  she_body<true, true>(a);
}

// tchi(r, s') = scale sum_c P(r, c) df(c, s'), P column-major (dimens x dimens); P == nullptr: identity
__global__ void she_prefactor_kernel(const double2* __restrict__ P, const double2* __restrict__ df, int D, double scale,
                                     double2* __restrict__ out) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= 4 * D) return;
  const int sp = o / D, r = o % D;
  double2 s = make_double2(0, 0);
  if (P) {
    for (int c = 0; c < D; ++c) s = cfma(P[(size_t)c * D + r], df[(size_t)sp * D + c], s);
  } else {
    s = df[o];
  }
  out[o] = cscale(s, scale);
}

}  // namespace

// Variant choice: the register-slice kernel when every second-stage tile has its own
// thread and its shared memory fits, else the staged kernel when its shared memory fits,
// else the global-operand kernel; 0 bytes when none fits.
enum SheVariant { SHE_GLOBAL = 0, SHE_STAGED = 1, SHE_REG = 2 };

int she_optin() {
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
  return optin;
}

SheVariant she_variant(int n, int dimens, int n_neigh, int n_ztiles, size_t optin) {
  if (n_ztiles <= kSheThreads && she_layout(n, dimens, n_neigh, true, false).bytes <= optin) return SHE_REG;
  if (she_layout(n, dimens, n_neigh, true).bytes <= optin) return SHE_STAGED;
  return SHE_GLOBAL;
}

size_t she_variant_bytes(int n, int dimens, int n_neigh, SheVariant v) {
  return she_layout(n, dimens, n_neigh, v != SHE_GLOBAL, v != SHE_REG).bytes;
}

const void* she_variant_fn(SheVariant v) {
  if (v == SHE_REG) return (const void*)she_kernel_reg;
  if (v == SHE_STAGED) return (const void*)she_kernel<true>;
  return (const void*)she_kernel<false>;
}

size_t she_smem_bytes(int n, int dimens, int n_neigh, int n_ztiles) {
  const int optin = she_optin();
  const size_t b = she_variant_bytes(n, dimens, n_neigh, she_variant(n, dimens, n_neigh, n_ztiles, (size_t)optin));
  return b <= (size_t)optin ? b : 0;
}

int she_grid(int n, int dimens, int n_neigh, int n_ztiles, int num_sms) {
  const int optin = she_optin();
  const SheVariant v = she_variant(n, dimens, n_neigh, n_ztiles, (size_t)optin);
  const size_t smem = she_variant_bytes(n, dimens, n_neigh, v);
  if (smem > (size_t)optin) return 0;
  const void* fn = she_variant_fn(v);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kSheThreads, smem) != cudaSuccess) return 0;
  return num_sms * std::max(per_sm, 1);
}

cudaError_t launch_she(const SheLaunch& l, cudaStream_t s) {
  if (l.grid <= 0) return cudaErrorInvalidValue;
  SheArgs a;
  a.G1 = l.G1;
  a.G2 = l.G2;
  a.p0 = l.p0;
  a.np = l.np;
  a.pts = l.pts;
  a.n = l.g->n;
  a.no = l.g->n / 2;
  a.dimens = l.dimens;
  a.n_neigh = l.g->n_neigh;
  a.nmax = l.g->nmax;
  a.n_atoms = l.g->n_atoms;
  a.R = l.g->R;
  a.pair_start = l.g->pair_start;
  a.pair_neigh = l.g->pair_neigh;
  a.pair_t = l.g->pair_t;
  a.tab = l.tab;
  a.ia = l.ia;
  a.norb = l.norb;
  a.decode = l.decode;
  a.ztiles = l.ztiles;
  a.n_ztiles = l.n_ztiles;
  a.rowoff = l.rowoff;
  a.real_axis = l.real_axis;
  for (int i = 0; i < 3; ++i) a.ue[i] = l.ue[i];
  for (int t = 0; t < 3; ++t)
    for (int i = 0; i < 16; ++i) a.spins[t][i] = l.spins[t][i];
  a.partial = l.partial;
  a.n_e = l.n_e;
  a.nk_tab = l.nk_tab;
  a.klist = l.klist;
  const int optin = she_optin();
  if (optin <= 0) return cudaErrorInvalidValue;
  const SheVariant v = she_variant(a.n, a.dimens, a.n_neigh, a.n_ztiles, (size_t)optin);
  const size_t smem = she_variant_bytes(a.n, a.dimens, a.n_neigh, v);
  if (smem > (size_t)optin) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(she_variant_fn(v), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (v == SHE_REG)
    she_kernel_reg<<<l.grid, kSheThreads, smem, s>>>(a);
  else if (v == SHE_STAGED)
    she_kernel<true><<<l.grid, kSheThreads, smem, s>>>(a);
  else
    she_kernel<false><<<l.grid, kSheThreads, smem, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_she_prefactor(const double2* P, const double2* df, int dimens, double scale, double2* out,
                                 cudaStream_t s) {
  const int total = 4 * dimens;
  she_prefactor_kernel<<<(total + 127) / 128, 128, 0, s>>>(P, df, dimens, scale, out);
  return cudaGetLastError();
}

}  // namespace tg
