// H(k) = h0 + sum_neighbours t0i exp(i k.R) for a list of k points, written
// as a row-major table H[k][r][c] (calchk + hamilt_local, mod_hamiltonian.F90:35-87,
// 183-243; the table is the reference's fullhk of fullhamiltk, :246-301).
//
// Two kernels: phases exp(i (k+q).R_n) per (k, neighbour cell), then one
// thread per matrix entry summing the hopping blocks of its site pair.  The
// table write dominates: the pair is HBM-bound (16 n^2 bytes per k written,
// the hopping table and phases come from L2).
#include "tg_internal.cuh"

#include <algorithm>

namespace tg {

namespace {

__global__ void phase_kernel(const double* __restrict__ kp, int64_t nk, const double* __restrict__ q,
                             const double* __restrict__ R, int n_neigh, double2* __restrict__ ph) {
  const int64_t total = nk * n_neigh;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = e / n_neigh;
    const int nb = (int)(e % n_neigh);
    const double th = (kp[3 * k] + q[0]) * R[3 * nb] + (kp[3 * k + 1] + q[1]) * R[3 * nb + 1] +
                      (kp[3 * k + 2] + q[2]) * R[3 * nb + 2];
    double s, c;
    sincos(th, &s, &c);
    ph[e] = make_double2(c, s);
  }
}

// one thread per (k, r, c); row-major H[k][r][c]
__global__ void hk_table_kernel(int n, int64_t nk, const double2* __restrict__ ph, int n_neigh,
                                const int* __restrict__ pair_start, const int* __restrict__ pair_neigh,
                                const double2* __restrict__ pair_t, int nmax, int n_atoms,
                                const int* __restrict__ row_atom, const int* __restrict__ row_orb,
                                const int* __restrict__ row_spin, const double2* __restrict__ h0,
                                double2* __restrict__ H) {
  const int64_t nn = (int64_t)n * n;
  const int64_t total = nk * nn;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = e / nn;
    const int rc = (int)(e % nn);
    const int r = rc / n, c = rc % n;
    double2 h = h0[(size_t)c * n + r];
    if (row_spin[r] == row_spin[c]) {
      const int pb = row_atom[r] * n_atoms + row_atom[c];
      const int orr = row_orb[r], oc = row_orb[c];
      const double2* phk = ph + k * n_neigh;
      for (int b = pair_start[pb]; b < pair_start[pb + 1]; ++b)
        h = cfma(phk[pair_neigh[b]], pair_t[(size_t)b * nmax * nmax + oc * nmax + orr], h);
    }
    H[e] = h;
  }
}

}  // namespace

cudaError_t launch_hk_table(const GreenArgs& a, const double* kp, int64_t nk, const double* d_q, double2* phase_ws,
                            double2* H, cudaStream_t s) {
  if (nk <= 0) return cudaSuccess;
  const int64_t np_ = nk * (a.n_neigh > 0 ? a.n_neigh : 1);
  if (a.n_neigh > 0) {
    int blocks = (int)std::min<int64_t>((np_ + 255) / 256, 148 * 32);
    phase_kernel<<<blocks, 256, 0, s>>>(kp, nk, d_q, a.R, a.n_neigh, phase_ws);
  }
  const int64_t total = nk * (int64_t)a.n * a.n;
  int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 64);
  hk_table_kernel<<<blocks, 256, 0, s>>>(a.n, nk, phase_ws, a.n_neigh, a.pair_start, a.pair_neigh, a.pair_t, a.nmax,
                                         a.n_atoms, a.row_atom, a.row_orb, a.row_spin, a.h0, H);
  return cudaGetLastError();
}

}  // namespace tg
