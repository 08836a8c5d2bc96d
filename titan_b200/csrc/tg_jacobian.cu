// Self-consistency Jacobian and the (V, B) adjoint from the GG tensor.
//
// Both are contractions of the device-computed tensor
//   T[s',t,t',s; i,g; j,h] = sum_p w_p sum_{mu in g, nu in h} G(i s' mu, j t nu) G(j t' nu, i s mu)
// with Pauli matrices on the two spin pairs:
//   V(i,g; j,h; a,b) = Re sum sigma_a[s][s'] sigma_b[t][t'] T[s',t,t',s]
//                    = Re Tr[P_ig sigma_a G P_jh sigma_b G]   (summed over the mesh).
// The host part here is O(n_atoms^2 nd^2 256) and runs on the CPU.
#include <cmath>
#include <cstring>
#include <algorithm>
#include <vector>

#include "../../include/titan_gpu.h"

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

struct C2 {
  double re, im;
};

// sigma_a[s][s'] (0 = up), a = 0 (identity), 1 (x), 2 (y), 3 (z)
const C2 kSigma[4][2][2] = {
    {{{1, 0}, {0, 0}}, {{0, 0}, {1, 0}}},
    {{{0, 0}, {1, 0}}, {{1, 0}, {0, 0}}},
    {{{0, 0}, {0, -1}}, {{0, 1}, {0, 0}}},
    {{{1, 0}, {0, 0}}, {{0, 0}, {-1, 0}}},
};

// Re sum_{s,s',t,t'} sigma_a[s][s'] sigma_b[t][t'] T[s' + 2t + 4t' + 8s]; T16 holds 16 complex
double vertex(const double* T16, int a, int b) {
  double acc = 0.0;
  for (int s = 0; s < 2; ++s)
    for (int sp = 0; sp < 2; ++sp) {
      const C2 x = kSigma[a][s][sp];
      if (x.re == 0.0 && x.im == 0.0) continue;
      for (int t = 0; t < 2; ++t)
        for (int tp = 0; tp < 2; ++tp) {
          const C2 y = kSigma[b][t][tp];
          if (y.re == 0.0 && y.im == 0.0) continue;
          const int q = sp + 2 * t + 4 * tp + 8 * s;
          const double xr = x.re * y.re - x.im * y.im, xi = x.re * y.im + x.im * y.re;
          acc += xr * T16[2 * q] - xi * T16[2 * q + 1];
        }
    }
  return acc;
}

bool nonzero(double u) { return std::fabs(u) > 1e-8; }

}  // namespace

extern "C" {

int tg_jacobian_layout(int n_atoms, const int* norb, int norb_max, const int* dmask, const double* Un,
                       const double* Um, int fixEf, int* per) {
  if (n_atoms <= 0 || !norb || !dmask || !Un || !Um || norb_max <= 0) return TG_ERR_ARG;
  int acc = 0;
  for (int i = 0; i < n_atoms; ++i) {
    int nd = 0;
    for (int o = 0; o < norb[i] && o < norb_max; ++o) nd += dmask[(size_t)i * norb_max + o] ? 1 : 0;
    if (per) per[i] = acc;
    acc += (nonzero(Un[i]) ? nd : 0) + (nonzero(Um[i]) ? 3 : 0);
  }
  if (per) per[n_atoms] = acc;
  return acc + (fixEf ? 0 : 1);
}

int tg_jacobian_assemble(int n_atoms, const int* norb, int norb_max, const int* dmask, const double* Un,
                         const double* Um, int fixEf, int nrow, int ncol, const double* T, const double* D, int neq,
                         double* jac) {
  if (n_atoms <= 0 || !norb || !dmask || !Un || !Um || !T || !jac || (!fixEf && !D)) return TG_ERR_ARG;
  std::vector<int> per(n_atoms + 1);
  const int n = tg_jacobian_layout(n_atoms, norb, norb_max, dmask, Un, Um, fixEf, per.data());
  if (n < 0 || n != neq) return TG_ERR_ARG;
  std::vector<std::vector<int>> dl(n_atoms);
  for (int i = 0; i < n_atoms; ++i)
    for (int o = 0; o < norb[i]; ++o)
      if (dmask[(size_t)i * norb_max + o]) dl[i].push_back(o);
  for (int i = 0; i < n_atoms; ++i) {
    if ((int)dl[i].size() + 1 > nrow || (int)dl[i].size() > ncol) return TG_ERR_ARG;
  }
  std::memset(jac, 0, sizeof(double) * (size_t)neq * neq);
  auto J = [&](int r, int c) -> double& { return jac[(size_t)c * neq + r]; };   // column-major
  auto Tblk = [&](int i, int j, int g, int h) {
    return T + 2 * 16 * ((((size_t)i * n_atoms + j) * nrow + g) * ncol + h);
  };
  for (int j = 0; j < n_atoms; ++j) {
    const int ndj = (int)dl[j].size();
    // column variables of site j: (column, Pauli b, coefficient, orbital weight of column group h)
    struct ColVar {
      int col, b;
      double c;
      int flip;   // charge variable: d orbital whose weight is 1 - 2 = -1 (else -1 for none)
    };
    std::vector<ColVar> vars;
    int kj = per[j];
    if (nonzero(Un[j])) {
      for (int m = 0; m < ndj; ++m) vars.push_back({kj + m, 0, -0.5 * Un[j], m});
      kj += ndj;
    }
    if (nonzero(Um[j]))
      for (int sp = 1; sp <= 3; ++sp) vars.push_back({kj + sp - 1, sp, -0.5 * Um[j], -1});
    for (int i = 0; i < n_atoms; ++i) {
      const int ndi = (int)dl[i].size();
      const int nrow_i = ndi + 1;   // d orbitals one by one, then the rest
      for (const ColVar& v : vars) {
        // W(g, a) = c sum_h m_h V(i,g; j,h; a,b)
        auto W = [&](int g, int a) {
          double s = 0.0;
          for (int h = 0; h < ndj; ++h) {
            const double m = (h == v.flip) ? -1.0 : 1.0;
            s += m * vertex(Tblk(i, j, g, h), a, v.b);
          }
          return v.c * s;
        };
        int ki = per[i];
        if (nonzero(Un[i])) {
          for (int m = 0; m < ndi; ++m) J(ki + m, v.col) += W(m, 0);
          ki += ndi;
        }
        if (!fixEf) {
          double s = 0.0;
          for (int g = 0; g < nrow_i; ++g) s += W(g, 0);
          J(neq - 1, v.col) += s;
        }
        if (nonzero(Um[i]))
          for (int sg = 1; sg <= 3; ++sg) {
            double s = 0.0;
            for (int g = 0; g < ndi; ++g) s += W(g, sg);
            J(ki + sg - 1, v.col) += s;
          }
      }
    }
  }
  if (!fixEf) {
    // D(4, norb_max, n_atoms): sum_k w_k tr_spin[sigma_a G_ii(mu, mu)] at Ef + i eta
    auto Dim = [&](int i, int mu, int a) { return D[2 * (a + 4 * ((size_t)mu + (size_t)norb_max * i)) + 1]; };
    for (int i = 0; i < n_atoms; ++i) {
      int ki = per[i];
      if (nonzero(Un[i])) {
        for (int m = 0; m < (int)dl[i].size(); ++m) J(ki + m, neq - 1) -= Dim(i, dl[i][m], 0);
        ki += (int)dl[i].size();
      }
      for (int mu = 0; mu < norb[i]; ++mu) J(neq - 1, neq - 1) -= Dim(i, mu, 0);
      if (nonzero(Um[i]))
        for (int sg = 1; sg <= 3; ++sg) {
          double s = 0.0;
          for (int mu : dl[i]) s += Dim(i, mu, sg);
          J(ki + sg - 1, neq - 1) -= s;
        }
    }
  }
  for (size_t e = 0; e < (size_t)neq * neq; ++e) jac[e] /= kPi;
  // minus the identity on the first neq - 1 diagonal entries, also with a fixed Fermi level
  // (the reference loops i = 1, neq - 1 in both cases)
  for (int k = 0; k < neq - 1; ++k) J(k, k) -= 1.0;
  return TG_OK;
}

int tg_jacobian(tg_ctx* ctx, double Ef, double eta, const int* dmask, const double* Un, const double* Um, int fixEf,
                int neq, double* jac) {
  if (!ctx || !dmask || !Un || !Um || !jac) return TG_ERR_ARG;
  int n_atoms = 0, norb_max = 0;
  int rc = tg_system_shape(ctx, &n_atoms, &norb_max, nullptr);
  if (rc) return rc;
  std::vector<int> norb(n_atoms);
  rc = tg_system_shape(ctx, &n_atoms, &norb_max, norb.data());
  if (rc) return rc;
  int nd_max = 0;
  for (int i = 0; i < n_atoms; ++i) {
    int nd = 0;
    for (int o = 0; o < norb[i]; ++o) nd += dmask[(size_t)i * norb_max + o] ? 1 : 0;
    nd_max = nd > nd_max ? nd : nd_max;
  }
  const int n = tg_jacobian_layout(n_atoms, norb.data(), norb_max, dmask, Un, Um, fixEf, nullptr);
  if (n != neq) return TG_ERR_ARG;
  const int nrow = nd_max + 1, ncol = nd_max;
  std::vector<double> T((size_t)2 * 16 * n_atoms * n_atoms * nrow * (ncol > 0 ? ncol : 1), 0.0);
  if (ncol > 0) {
    rc = tg_gg_tensor(ctx, Ef, eta, 1, dmask, T.data());
    if (rc) return rc;
  }
  std::vector<double> D;
  if (!fixEf) {
    D.assign((size_t)2 * 4 * norb_max * n_atoms, 0.0);
    rc = tg_fermi_column(ctx, Ef, eta, D.data());
    if (rc) return rc;
  }
  return tg_jacobian_assemble(n_atoms, norb.data(), norb_max, dmask, Un, Um, fixEf, nrow, ncol > 0 ? ncol : 1,
                              T.data(), fixEf ? nullptr : D.data(), neq, jac);
}

int tg_adjoint_vb(tg_ctx* ctx, double Ef, double eta, double* A) {
  if (!ctx || !A) return TG_ERR_ARG;
  int n_atoms = 0, norb_max = 0;
  int rc = tg_system_shape(ctx, &n_atoms, &norb_max, nullptr);
  if (rc) return rc;
  std::vector<double> T((size_t)2 * 16 * n_atoms * n_atoms, 0.0);
  rc = tg_gg_tensor(ctx, Ef, eta, 0, nullptr, T.data());
  if (rc) return rc;
  const int m = 4 * n_atoms;
  for (int i = 0; i < n_atoms; ++i)
    for (int j = 0; j < n_atoms; ++j) {
      const double* T16 = T.data() + 2 * 16 * ((size_t)i * n_atoms + j);
      for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) A[(size_t)(b + 4 * j) * m + (a + 4 * i)] = vertex(T16, a, b) / kPi;
    }
  return TG_OK;
}

int tg_adjoint_vb_orbitals(tg_ctx* ctx, double Ef, double eta, const int* mask, double* A) {
  if (!mask) return tg_adjoint_vb(ctx, Ef, eta, A);
  if (!ctx || !A) return TG_ERR_ARG;
  int n_atoms = 0, norb_max = 0;
  int rc = tg_system_shape(ctx, &n_atoms, &norb_max, nullptr);
  if (rc) return rc;
  std::vector<int> norb(n_atoms);
  rc = tg_system_shape(ctx, &n_atoms, &norb_max, norb.data());
  if (rc) return rc;
  // the orbital-resolved tensor with the masked orbitals as the resolved ones: row groups
  // g < n_i (one masked orbital each, then the rest), column groups h < n_i
  std::vector<int> nsel(n_atoms, 0);
  int nmax_sel = 0;
  for (int i = 0; i < n_atoms; ++i) {
    for (int o = 0; o < norb[i]; ++o) nsel[i] += mask[(size_t)i * norb_max + o] ? 1 : 0;
    nmax_sel = std::max(nmax_sel, nsel[i]);
  }
  if (nmax_sel == 0) return TG_ERR_ARG;
  const int nrow = nmax_sel + 1, ncol = nmax_sel;
  std::vector<double> T((size_t)2 * 16 * n_atoms * n_atoms * nrow * ncol, 0.0);
  rc = tg_gg_tensor(ctx, Ef, eta, 1, mask, T.data());
  if (rc) return rc;
  const int m = 4 * n_atoms;
  std::vector<double> S(2 * 16);
  for (int i = 0; i < n_atoms; ++i)
    for (int j = 0; j < n_atoms; ++j) {
      std::fill(S.begin(), S.end(), 0.0);
      for (int g = 0; g < nsel[i]; ++g)
        for (int h = 0; h < nsel[j]; ++h) {
          const double* T16 = T.data() + 2 * 16 * ((((size_t)i * n_atoms + j) * nrow + g) * ncol + h);
          for (int e = 0; e < 32; ++e) S[e] += T16[e];
        }
      for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) A[(size_t)(b + 4 * j) * m + (a + 4 * i)] = vertex(S.data(), a, b) / kPi;
    }
  return TG_OK;
}

}  // extern "C"
