// Exchange coupling J_ij(q) of jij_energy (source/jij_energy.F90:6-242), normal state.
//
// With dBxc/dm on the d orbitals, A^i_mu = sum_a c^i_{mu a} sigma^d_a
// (c^i_{mu a} = -Um_i / 2 (delta_{mu a} - e_{i mu} e_{i a}), e_i the d-moment direction),
//   J_ij^{mu nu}(q) = -1/(2 pi) sum_{k,E} w [ Tr(A^i_mu G_ij(k) A^j_nu G_ji(k - q))
//                                          + conj Tr(A^i_mu G_ij(k - q) A^j_nu G_ji(k)) ],
// so everything reduces to two d-orbital GG tensors per site pair,
//   T [s', t, t', s] = sum_{alpha in d(i), beta in d(j)} w G_a(i s' alpha, j t beta) G_b(j t' beta, i s alpha)
// with (G_a, G_b) = (G(k), G(k - q)) and, for T', the two swapped.  jij_kernel
// accumulates both tensors for every site pair from the column-major inversion
// outputs of a pass (one CTA per point at a time, each thread owning tensor entries of
// a per-CTA slice); the 3 x 3 spin algebra runs on the host.
#include "tg_internal.cuh"

#include <algorithm>

namespace tg {

namespace {

struct JijArgs {
  const double2* Ga = nullptr;   // [np][n][n] G(k), column-major
  const double2* Gb = nullptr;   // [np][n][n] G(k - q)
  int64_t p0 = 0, np = 0;
  const double* w = nullptr;     // point weights of the imaginary-axis list
  int n = 0, n_atoms = 0;
  const int* ia = nullptr;       // first row of each site
  const int* norb = nullptr;
  const int* dstart = nullptr;   // [n_atoms + 1] offsets into dlist
  const int* dlist = nullptr;    // d orbitals (local index) of every site
  double2* partial = nullptr;    // [grid][n_atoms^2][2][16]
};

__global__ void __launch_bounds__(256) jij_kernel(JijArgs a) {
  const int nat = a.n_atoms, n = a.n;
  const int len = nat * nat * 32;
  double2* mine = a.partial + (size_t)blockIdx.x * len;
  for (int64_t pl = blockIdx.x; pl < a.np; pl += gridDim.x) {
    const double w = a.w[a.p0 + pl];
    const double2* ga = a.Ga + pl * (int64_t)n * n;
    const double2* gb = a.Gb + pl * (int64_t)n * n;
    for (int o = threadIdx.x; o < len; o += blockDim.x) {
      const int q = o & 15, swap = (o >> 4) & 1, pair = o >> 5;
      const int i = pair / nat, j = pair % nat;
      const int sp = q & 1, t = (q >> 1) & 1, tp = (q >> 2) & 1, s = (q >> 3) & 1;
      const double2* X = swap ? gb : ga;
      const double2* Y = swap ? ga : gb;
      const int ni = a.norb[i], nj = a.norb[j];
      double2 acc = make_double2(0.0, 0.0);
      for (int da = a.dstart[i]; da < a.dstart[i + 1]; ++da) {
        const int al = a.dlist[da];
        const int r1 = a.ia[i] + sp * ni + al, c2 = a.ia[i] + s * ni + al;
        for (int db = a.dstart[j]; db < a.dstart[j + 1]; ++db) {
          const int be = a.dlist[db];
          const int c1 = a.ia[j] + t * nj + be, r2 = a.ia[j] + tp * nj + be;
          acc = cfma(X[(int64_t)c1 * n + r1], Y[(int64_t)c2 * n + r2], acc);
        }
      }
      mine[o] = cfma(make_double2(w, 0.0), acc, mine[o]);
    }
  }
}

}  // namespace

cudaError_t launch_jij(const double2* Ga, const double2* Gb, int64_t p0, int64_t np, const double* w, int n,
                       int n_atoms, const int* ia, const int* norb, const int* dstart, const int* dlist,
                       double2* partial, int grid, cudaStream_t s) {
  if (np <= 0) return cudaSuccess;
  JijArgs a;
  a.Ga = Ga;
  a.Gb = Gb;
  a.p0 = p0;
  a.np = np;
  a.w = w;
  a.n = n;
  a.n_atoms = n_atoms;
  a.ia = ia;
  a.norb = norb;
  a.dstart = dstart;
  a.dlist = dlist;
  a.partial = partial;
  jij_kernel<<<grid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace tg
