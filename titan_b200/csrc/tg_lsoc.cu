// Linear-SOC susceptibility (eintshechilinearsoc, source/eintshechi.F90:182-414).
//
// With G0 = (z - H0)^-1 for the Hamiltonian without the local spin-orbit blocks and
// V the SOC blocks (hamiltklinearsoc, mod_hamiltonian.F90:304-396), the reference's
// greenlinearsoc (mod_greenfunction.F90:141-202) forms G0 V G0 per point and
//   chi_lsoc = chi(G0 V G0 (k+q, E+e), G0(k, E)) + chi(G0(k+q, E+e), G0 V G0 (k, E)),
// chi(., .) being the same bilinear integrand as chi0.  Here the per-point pieces are
// two kernels around the existing inversion and contraction kernels:
//   gvg_kernel      X_p = G_p V G_p from the column-major inversion output (one CTA
//                   per point, G, V and V G staged in shared memory, FP64);
//   operand_kernel  a column-major G_p (or X_p) into the pair-block operand layouts of
//                   the contraction (w G, G^T, w (G - G^+), conj G) with the point weights.
#include "tg_internal.cuh"

#include <algorithm>

namespace tg {

namespace {

// X[p] = G[p] V G[p], all column-major n x n; Gs, T row-major in shared memory
__global__ void __launch_bounds__(256) gvg_kernel(const double2* __restrict__ G, const double2* __restrict__ V, int n,
                                                  int64_t np, double2* __restrict__ X) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int nn = n * n;
  double2* Vs = reinterpret_cast<double2*>(smem);
  double2* Gs = Vs + nn;
  double2* T = Gs + nn;
  for (int e = threadIdx.x; e < nn; e += blockDim.x) {
    const int c = e / n, r = e % n;
    Vs[r * n + c] = V[e];
  }
  for (int64_t p = blockIdx.x; p < np; p += gridDim.x) {
    __syncthreads();
    const double2* g = G + p * (int64_t)nn;
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
      const int c = e / n, r = e % n;
      Gs[r * n + c] = g[e];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
      const int r = e / n, c = e % n;
      double2 s = make_double2(0.0, 0.0);
      for (int m = 0; m < n; ++m) s = cfma(Vs[r * n + m], Gs[m * n + c], s);
      T[e] = s;
    }
    __syncthreads();
    double2* x = X + p * (int64_t)nn;
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
      const int c = e / n, r = e % n;   // column-major write, consecutive threads down a column
      double2 s = make_double2(0.0, 0.0);
      for (int m = 0; m < n; ++m) s = cfma(Gs[r * n + m], T[m * n + c], s);
      x[e] = s;
    }
  }
}

// out[p][o] = transform of G_p at the pair-block slot o (outmap[o] = r * n + c), p in the pass
__global__ void operand_kernel(const double2* __restrict__ G, int n, int64_t np, int64_t p0, PointSet pts, int mode,
                               const int* __restrict__ outmap, double2* __restrict__ out) {
  const int64_t nn = (int64_t)n * n;
  const int64_t total = np * nn;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pl = idx / nn;
    const int o = (int)(idx % nn);
    const int rc = outmap[o];
    const int r = rc / n, c = rc % n;
    const double2* g = G + pl * nn;
    const int64_t p = p0 + pl;
    double w;
    if (pts.kind == 0) {
      w = pts.w[p];
    } else {
      w = pts.p2[p / pts.nk] * pts.w[p % pts.nk];
    }
    const double2 grc = g[(int64_t)c * n + r];
    double2 v;
    if (mode == MODE_A_IMAG) {
      v = cscale(grc, w);
    } else if (mode == MODE_B_IMAG) {
      v = g[(int64_t)r * n + c];   // G^T
    } else if (mode == MODE_A_REAL) {
      const double2 gcr = g[(int64_t)r * n + c];
      v = cscale(make_double2(grc.x - gcr.x, grc.y + gcr.y), w);
    } else {
      v = cconj(grc);
    }
    out[idx] = v;
  }
}

// out[p][o] = transform of the column-major G_p (n x n) at slot o of an operand layout with
// ld slots per point (outmap[o] = r * n + c, a subset of G's entries in pair-block order);
// the weights follow the point traversal of the Green-function launch g (tabulated k-major
// or the flattened list), as the fused output stages do
__global__ void gather_kernel(GreenArgs g, const double2* __restrict__ G, int mode, const int* __restrict__ outmap,
                              int64_t ld, double2* __restrict__ out, int16_t* __restrict__ eout) {
  const int n = g.n;
  const int64_t nn = (int64_t)n * n;
  const int64_t total = g.np * ld;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pl = idx / ld;
    const int o = (int)(idx - pl * ld);
    const int rc = outmap[o];
    const int r = rc / n, c = rc - r * n;
    const double2* gp = G + pl * nn;
    const int64_t wi = g.p0 + pl;
    double w;
    if (g.htab || g.eigU || g.triQ) {   // k-major: an H(k) table, or its decompositions
      const int64_t ik = wi / g.n_e, ie = wi % g.n_e;
      w = g.pts.kind == 0 ? g.pts.w[ie * g.nk_tab + ik] : g.pts.p2[ie] * g.pts.w[ik];
    } else if (g.pts.kind == 0) {
      w = g.pts.w[wi];
    } else if (g.pts.kind == 1) {
      w = g.pts.p2[wi / g.pts.nk] * g.pts.w[wi % g.pts.nk];
    } else {
      w = 1.0;
    }
    const double2 grc = gp[(int64_t)c * n + r];
    double2 v;
    if (mode == MODE_A_IMAG) {
      v = cscale(grc, w);
    } else if (mode == MODE_B_IMAG) {
      v = gp[(int64_t)r * n + c];   // G^T
    } else if (mode == MODE_A_REAL) {
      const double2 gcr = gp[(int64_t)r * n + c];
      v = cscale(make_double2(grc.x - gcr.x, grc.y + gcr.y), w);
    } else {
      v = cconj(grc);
    }
    out[idx] = v;
    if (eout) eout[idx] = exponent_code16(v);
  }
}

}  // namespace

cudaError_t launch_gather(const GreenArgs& g, const double2* G, int mode, const int* outmap, int64_t ld, double2* out,
                          int16_t* eout, int num_sms, cudaStream_t s) {
  if (g.np <= 0) return cudaSuccess;
  if (mode != MODE_A_IMAG && mode != MODE_B_IMAG && mode != MODE_A_REAL && mode != MODE_B_REAL)
    return cudaErrorInvalidValue;
  const int64_t total = g.np * ld;
  const int64_t grid = std::min<int64_t>((total + 255) / 256, (int64_t)num_sms * 16);
  gather_kernel<<<(unsigned)grid, 256, 0, s>>>(g, G, mode, outmap, ld, out, eout);
  return cudaGetLastError();
}

size_t gvg_smem_bytes(int n) { return sizeof(double2) * 3 * (size_t)n * n; }

cudaError_t launch_gvg(const double2* G, const double2* V, int n, int64_t np, double2* X, int num_sms,
                       cudaStream_t s) {
  if (np <= 0) return cudaSuccess;
  const size_t smem = gvg_smem_bytes(n);
  cudaError_t e = cudaFuncSetAttribute(gvg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gvg_kernel, 256, smem);
  if (e != cudaSuccess) return e;
  if (per_sm <= 0) return cudaErrorInvalidValue;
  const int64_t grid = std::min<int64_t>(np, (int64_t)num_sms * per_sm);
  gvg_kernel<<<(unsigned)grid, 256, smem, s>>>(G, V, n, np, X);
  return cudaGetLastError();
}

cudaError_t launch_operand(const double2* G, int n, int64_t np, int64_t p0, const PointSet& pts, int mode,
                           const int* outmap, double2* out, int num_sms, cudaStream_t s) {
  if (np <= 0) return cudaSuccess;
  const int64_t total = np * (int64_t)n * n;
  const int64_t grid = std::min<int64_t>((total + 255) / 256, (int64_t)num_sms * 16);
  operand_kernel<<<(unsigned)grid, 256, 0, s>>>(G, n, np, p0, pts, mode, outmap, out);
  return cudaGetLastError();
}

}  // namespace tg
