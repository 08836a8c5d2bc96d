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
// output entries.  Each CTA owns a slice (4 dimens complex) of a per-CTA
// global array, so successive launches (passes) accumulate without atomics;
// the slices are summed once at the end.  When they fit (dimH up to about 48
// for small dimens), both Green functions are staged row-major in shared memory
// and the slice is held there during the launch; larger cells read the
// column-major inversion output through L1 / L2 and add into the slice in
// place.
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
  int real_axis = 0;
  double ue[3] = {0, 0, 0};
  unsigned char spins[3][16] = {};   // term t, (s * 4 + s') -> a << 3 | b << 2 | c << 1 | d (0 = up)
  double2* partial = nullptr;        // [gridDim][4 dimens], df(row, s') at s' dimens + row
  int64_t n_e = 0, nk_tab = 0;       // k-major order of a tabulated pass (n_e > 0)
  const double* klist = nullptr;
};

struct SheSmem {
  int s1, s2, m, mt, y, acc, ph, tab;   // offsets in double2 units (tab: in bytes)
  size_t bytes;
};

// Shared-memory layout.  STAGED: both Green functions (row-major) live in shared
// memory, and the df partial too unless it is held in registers (acc_smem false);
// otherwise they are read from / accumulated in global memory (L1 / L2) and only
// V, V^T, Y and the tables are staged.
__host__ __device__ inline SheSmem she_layout(int n, int dimens, int n_neigh, bool staged, bool acc_smem = true) {
  const int no = n / 2;
  SheSmem L;
  int o = 0;
  L.s1 = o; o += staged ? n * n : 0;
  L.s2 = o; o += staged ? n * n : 0;
  L.m = o; o += no * no;
  L.mt = o; o += no * no;
  L.y = o; o += 2 * n * no;
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
// output rows (r, col) of each df entry; acc[s' dimens + row] += f Z.
// First stage: Y^b = L[:, spin b] M for both spins b (2 n x no).
template <class LM>
__device__ void she_y(const SheArgs& a, LM L, const double2* M, double2* Y, const int* tab) {
  const int n = a.n, no = a.no;
  for (int e = threadIdx.x; e < 2 * n * no; e += blockDim.x) {
    const int b = e / (n * no), r = (e / no) % n, o1 = e % no;
    const int* rowb = tab + b * no;
    double2 s = make_double2(0, 0);
    for (int o2 = 0; o2 < no; ++o2) s = cfma(L(r, rowb[o2]), M[o2 * no + o1], s);
    Y[e] = s;
  }
  __syncthreads();
}

// Second stage for df entry o = s' dimens + row: Z(r, col) of that entry.
template <class RM>
__device__ __forceinline__ double2 she_z(const SheArgs& a, int o, const double2* Y, RM R, const int* tab,
                                         const unsigned char* spins, bool rows_are_nu) {
  const int n = a.n, no = a.no, D = a.dimens;
  const int sp = o / D, row = o % D;
  const int dec = a.decode[row];
  const int sigma = dec & 3, i = (dec >> 2) & 1023, mu = (dec >> 12) & 63, nu = (dec >> 18) & 63;
  const int code = spins[sigma * 4 + sp];
  const int sa = (code >> 3) & 1, b = (code >> 2) & 1, c = (code >> 1) & 1, sd = code & 1;
  const int x = rows_are_nu ? nu : mu, y = rows_are_nu ? mu : nu;
  const int ni = a.norb[i];
  const int r = a.ia[i] + sa * ni + x, col = a.ia[i] + sd * ni + y;
  const double2* Yr = Y + (b * n + r) * no;
  const int* rowc = tab + c * no;
  double2 s = make_double2(0, 0);
  for (int o1 = 0; o1 < no; ++o1) s = cfma(Yr[o1], R(rowc[o1], col), s);
  return s;
}

// the term with the df slice in memory (shared or global)
template <class LM, class RM>
__device__ void she_term(const SheArgs& a, LM L, const double2* M, RM R, double2* Y, double2* acc, const int* tab,
                         const unsigned char* spins, double2 f, bool rows_are_nu) {
  she_y(a, L, M, Y, tab);
  for (int o = threadIdx.x; o < 4 * a.dimens; o += blockDim.x)
    acc[o] = cfma(f, she_z(a, o, Y, R, tab, spins, rows_are_nu), acc[o]);
  __syncthreads();
}

// the term with the df slice in registers: entry o = threadIdx.x + i blockDim.x in racc[i]
template <int RACC, class LM, class RM>
__device__ void she_term_reg(const SheArgs& a, LM L, const double2* M, RM R, double2* Y, double2 (&racc)[RACC],
                             const int* tab, const unsigned char* spins, double2 f, bool rows_are_nu) {
  she_y(a, L, M, Y, tab);
#pragma unroll
  for (int i = 0; i < RACC; ++i) {
    const int o = threadIdx.x + i * blockDim.x;
    if (o < 4 * a.dimens) racc[i] = cfma(f, she_z(a, o, Y, R, tab, spins, rows_are_nu), racc[i]);
  }
  __syncthreads();
}

// STAGED: Green functions in shared memory; RACC > 0 (staged only): the df slice in
// RACC registers per thread (4 dimens <= RACC x 256), which leaves the shared memory
// to the Green functions, V and Y and fits three CTAs per SM at dimH 36
template <bool STAGED, int RACC>
__device__ __forceinline__ void she_body(const SheArgs& a) {
  static_assert(STAGED || RACC == 0, "register slices only in the staged kernel");
  extern __shared__ __align__(16) unsigned char smem[];
  const int n = a.n, no = a.no, D = a.dimens;
  const SheSmem L = she_layout(n, D, a.n_neigh, STAGED, RACC == 0);
  double2* base = reinterpret_cast<double2*>(smem);
  double2* S1 = base + L.s1;
  double2* S2 = base + L.s2;
  double2* M = base + L.m;
  double2* MT = base + L.mt;
  double2* Y = base + L.y;
  double2* ph = base + L.ph;
  int* tab = reinterpret_cast<int*>(smem + L.tab);
  double2* mine = a.partial + (size_t)blockIdx.x * 4 * D;
  double2* acc = STAGED && RACC == 0 ? base + L.acc : mine;
  double2 racc[RACC > 0 ? RACC : 1];
  if (RACC > 0) {
#pragma unroll
    for (int i = 0; i < (RACC > 0 ? RACC : 1); ++i) {
      const int o = threadIdx.x + i * blockDim.x;
      racc[i] = o < 4 * D ? mine[o] : make_double2(0.0, 0.0);
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
          S1[r * n + c] = g1[e];
          S2[r * n + c] = g2[e];
        }
      } else {
        for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
          const int r = e / n, c = e % n;
          const double2 x = g1[(size_t)c * n + r], xt = g1[(size_t)r * n + c];
          S1[e] = make_double2(x.x - xt.x, x.y + xt.y);
          const double2 y = g2[(size_t)r * n + c];
          S2[e] = make_double2(y.x, -y.y);
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
      MT[cc * no + rr] = v;
    }
    __syncthreads();
    if (STAGED && RACC > 0) {
      if (!a.real_axis) {
        she_term_reg(a, RowMajor{S1, n}, M, RowMajor{S2, n}, Y, racc, tab, a.spins[0], make_double2(w, 0.0), true);
        for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
          S1[e].y = -S1[e].y;
          S2[e].y = -S2[e].y;
        }
        __syncthreads();
        she_term_reg(a, RowMajor{S2, n}, MT, RowMajor{S1, n}, Y, racc, tab, a.spins[1], make_double2(w, 0.0),
                     false);
      } else {
        she_term_reg(a, RowMajor{S1, n}, M, RowMajor{S2, n}, Y, racc, tab, a.spins[2], make_double2(0.0, -w), true);
      }
    } else if (STAGED) {
      if (!a.real_axis) {
        she_term(a, RowMajor{S1, n}, M, RowMajor{S2, n}, Y, acc, tab, a.spins[0], make_double2(w, 0.0), true);
        for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
          S1[e].y = -S1[e].y;
          S2[e].y = -S2[e].y;
        }
        __syncthreads();
        she_term(a, RowMajor{S2, n}, MT, RowMajor{S1, n}, Y, acc, tab, a.spins[1], make_double2(w, 0.0), false);
      } else {
        she_term(a, RowMajor{S1, n}, M, RowMajor{S2, n}, Y, acc, tab, a.spins[2], make_double2(0.0, -w), true);
      }
    } else {
      if (!a.real_axis) {
        she_term(a, ColMajor{g1, n, GK_G}, M, ColMajor{g2, n, GK_G}, Y, acc, tab, a.spins[0], make_double2(w, 0.0),
                 true);
        she_term(a, ColMajor{g2, n, GK_CONJ}, MT, ColMajor{g1, n, GK_CONJ}, Y, acc, tab, a.spins[1],
                 make_double2(w, 0.0), false);
      } else {
        she_term(a, ColMajor{g1, n, GK_ANTI}, M, ColMajor{g2, n, GK_DAGGER}, Y, acc, tab, a.spins[2],
                 make_double2(0.0, -w), true);
      }
    }
  }
  if (RACC > 0) {
#pragma unroll
    for (int i = 0; i < (RACC > 0 ? RACC : 1); ++i) {
      const int o = threadIdx.x + i * blockDim.x;
      if (o < 4 * D) mine[o] = racc[i];
    }
  } else if (STAGED) {
    for (int e = threadIdx.x; e < 4 * D; e += blockDim.x) mine[e] = acc[e];
  }
}

template <bool STAGED>
__global__ void __launch_bounds__(256) she_kernel(SheArgs a) {
  she_body<STAGED, 0>(a);
}

// the register-slice variant: 127 registers, two CTAs per SM (a three-CTA bound spills)
constexpr int kSheRacc = 12;
__global__ void __launch_bounds__(256, 2) she_kernel_reg(SheArgs a) {
  she_body<true, kSheRacc>(a);
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

// Variant choice: the staged kernel with register slices when 4 dimens <= kSheRacc x 256
// and its shared memory fits, else the staged kernel with the slice in shared memory,
// else the global-operand kernel; 0 bytes when none fits.
enum SheVariant { SHE_GLOBAL = 0, SHE_STAGED = 1, SHE_STAGED_REG = 2 };

SheVariant she_variant(int n, int dimens, int n_neigh, size_t optin) {
  if (4 * dimens <= kSheRacc * 256 && she_layout(n, dimens, n_neigh, true, false).bytes <= optin)
    return SHE_STAGED_REG;
  if (she_layout(n, dimens, n_neigh, true).bytes <= optin) return SHE_STAGED;
  return SHE_GLOBAL;
}

size_t she_variant_bytes(int n, int dimens, int n_neigh, SheVariant v) {
  return she_layout(n, dimens, n_neigh, v != SHE_GLOBAL, v != SHE_STAGED_REG).bytes;
}

const void* she_variant_fn(SheVariant v) {
  if (v == SHE_STAGED_REG) return (const void*)she_kernel_reg;
  if (v == SHE_STAGED) return (const void*)she_kernel<true>;
  return (const void*)she_kernel<false>;
}

int she_optin() {
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
  return optin;
}

size_t she_smem_bytes(int n, int dimens, int n_neigh) {
  const int optin = she_optin();
  const size_t b = she_variant_bytes(n, dimens, n_neigh, she_variant(n, dimens, n_neigh, (size_t)optin));
  return b <= (size_t)optin ? b : 0;
}

int she_grid(int n, int dimens, int n_neigh, int num_sms) {
  const int optin = she_optin();
  const SheVariant v = she_variant(n, dimens, n_neigh, (size_t)optin);
  const size_t smem = she_variant_bytes(n, dimens, n_neigh, v);
  if (smem > (size_t)optin) return 0;
  const void* fn = she_variant_fn(v);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, smem) != cudaSuccess) return 0;
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
  const SheVariant v = she_variant(a.n, a.dimens, a.n_neigh, (size_t)optin);
  const size_t smem = she_variant_bytes(a.n, a.dimens, a.n_neigh, v);
  if (smem > (size_t)optin) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(she_variant_fn(v), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (v == SHE_STAGED_REG)
    she_kernel_reg<<<l.grid, 256, smem, s>>>(a);
  else if (v == SHE_STAGED)
    she_kernel<true><<<l.grid, 256, smem, s>>>(a);
  else
    she_kernel<false><<<l.grid, 256, smem, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_she_prefactor(const double2* P, const double2* df, int dimens, double scale, double2* out,
                                 cudaStream_t s) {
  const int total = 4 * dimens;
  she_prefactor_kernel<<<(total + 127) / 128, 128, 0, s>>>(P, df, dimens, scale, out);
  return cudaGetLastError();
}

}  // namespace tg
