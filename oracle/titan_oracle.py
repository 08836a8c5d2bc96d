"""CPU oracle for the k-mesh x complex-energy Green-function path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only the tests, the
smoke check and the CPU-baseline leg of the benchmark may import it.  The
product path (titan_b200) never calls it.

It restates the reference's FP64 algorithm with numpy/LAPACK:

* ``hk``                 -- calchk, source/mod_hamiltonian.F90:183-243
* ``green``              -- green + invers, source/mod_greenfunction.F90:19-75,
                            source/mod_tools.F90:796-829 (LAPACK inverse)
* ``eintshechi``         -- source/eintshechi.F90:2-178; the 16 spin-block
                            products are taken verbatim from the index tables
                            of lines 86-104 (imaginary axis) and 146-164 (real
                            axis), NOT from the GEMM re-formulation the GPU
                            path uses, so the two are independent
* ``umatrix`` / ``dyson`` -- source/mod_susceptibilities.F90:106-159,
                            source/calculate_chi.F90:85-89
* ``site_reduce``        -- source/calculate_chi.F90:91-107
* ``expectation``        -- source/mod_expectation.F90:28-149
* ``gs_orbital``         -- source/mod_expectation.F90:912-982 (orbital density)
* ``jacobian``           -- source/mod_self_consistency.F90:795-1205
* ``self_consistency``   -- Newton iteration on sc_eqs
                            (source/mod_self_consistency.F90:1516-1833); the
                            root is the one SLATEC dnsqe converges to
"""
from __future__ import annotations

import math

import numpy as np

PI = 4.0 * math.atan(1.0)
TPI = 2.0 * PI

# ---------------------------------------------------------------------------
# Index tables of eintshechi.F90:86-104 (imaginary axis).  For chi element
# (s1, s2): TERM1 gives the spin blocks of  gf?? (nu,gama,i,j,1) * gf?? (xi,mu,j,i,2)
# and TERM2 those of conjg( gf?? (mu,xi,i,j,2) * gf?? (gama,nu,j,i,1) ).
# ---------------------------------------------------------------------------
TERM1 = {(1, 1): ("dd", "uu"), (1, 2): ("du", "uu"), (1, 3): ("dd", "du"), (1, 4): ("du", "du"),
         (2, 1): ("ud", "uu"), (2, 2): ("uu", "uu"), (2, 3): ("ud", "du"), (2, 4): ("uu", "du"),
         (3, 1): ("dd", "ud"), (3, 2): ("du", "ud"), (3, 3): ("dd", "dd"), (3, 4): ("du", "dd"),
         (4, 1): ("ud", "ud"), (4, 2): ("uu", "ud"), (4, 3): ("ud", "dd"), (4, 4): ("uu", "dd")}
TERM2 = {(1, 1): ("uu", "dd"), (1, 2): ("uu", "ud"), (1, 3): ("ud", "dd"), (1, 4): ("ud", "ud"),
         (2, 1): ("uu", "du"), (2, 2): ("uu", "uu"), (2, 3): ("ud", "du"), (2, 4): ("ud", "uu"),
         (3, 1): ("du", "dd"), (3, 2): ("du", "ud"), (3, 3): ("dd", "dd"), (3, 4): ("dd", "ud"),
         (4, 1): ("du", "du"), (4, 2): ("du", "uu"), (4, 3): ("dd", "du"), (4, 4): ("dd", "uu")}
# eintshechi.F90:146-164 (real axis): (gf??(nu,gama,i,j,1) - conjg(gf??(gama,nu,j,i,1))) * conjg(gf??(mu,xi,i,j,2))
REAL = {(1, 1): ("dd", "dd", "uu"), (1, 2): ("du", "ud", "uu"), (1, 3): ("dd", "dd", "ud"), (1, 4): ("du", "ud", "ud"),
        (2, 1): ("ud", "du", "uu"), (2, 2): ("uu", "uu", "uu"), (2, 3): ("ud", "du", "ud"), (2, 4): ("uu", "uu", "ud"),
        (3, 1): ("dd", "dd", "du"), (3, 2): ("du", "ud", "du"), (3, 3): ("dd", "dd", "dd"), (3, 4): ("du", "ud", "dd"),
        (4, 1): ("ud", "du", "du"), (4, 2): ("uu", "uu", "du"), (4, 3): ("ud", "du", "dd"), (4, 4): ("uu", "uu", "dd")}
_SPIN = {"u": 0, "d": 1}


class Model:
    """Dense hopping matrices T_k (one per neighbour) and h0 for numpy evaluation."""

    def __init__(self, system, h0):
        self.system = system
        self.h0 = np.asarray(h0, dtype=complex)
        cv, bi, ish, t = system.neighbor_table()
        n = system.dimH
        ia = system.ia()
        norbs = system.norbs
        nn = cv.shape[0]
        T = np.zeros((nn, n, n), dtype=complex)
        for k in range(nn):
            j = int(bi[k])
            for i in range(system.n_atoms):
                if not ish[k, i]:
                    continue
                blk = t[k, i, :norbs[j], :norbs[i]]
                # calchk: rows of atom j (neighbour), columns of atom i; both spins
                T[k, ia[j][0]:ia[j][1], ia[i][0]:ia[i][1]] += blk
                T[k, ia[j][2]:ia[j][3], ia[i][2]:ia[i][3]] += blk
        self.R = cv
        self.T = T
        self.n = n

    def hk(self, kp):
        """H(k) = h0 + sum_neigh exp(i k.R) T_neigh, kp: [P, 3] -> [P, n, n]."""
        kp = np.atleast_2d(kp)
        ph = np.exp(1j * (kp @ self.R.T))                      # [P, nNeigh]
        H = np.tensordot(ph, self.T, axes=([1], [0]))           # [P, n, n]
        return H + self.h0[None]

    def green(self, z, kp):
        """G = (z 1 - h0 - H_nl(k))^-1 for arrays z [P] and kp [P, 3]."""
        H = self.hk(kp)
        z = np.broadcast_to(np.asarray(z, dtype=complex), (H.shape[0],))
        A = z[:, None, None] * np.eye(self.n)[None] - H
        return np.linalg.inv(A)


def _blk(G, ia, norbs, i, j, spins):
    si, sj = _SPIN[spins[0]], _SPIN[spins[1]]
    r0 = ia[i][0] + si * norbs[i]
    c0 = ia[j][0] + sj * norbs[j]
    return G[:, r0:r0 + norbs[i], c0:c0 + norbs[j]]


def _chunks(P, size):
    for s in range(0, P, size):
        yield slice(s, min(P, s + size))


def _sel_blk(sel):
    """_blk restricted to the orbitals sel[i] of every site (both spins)."""
    def blk(G, ia, norbs, i, j, spins):
        si, sj = _SPIN[spins[0]], _SPIN[spins[1]]
        r = ia[i][0] + si * norbs[i] + np.asarray(sel[i], dtype=np.int64)
        c = ia[j][0] + sj * norbs[j] + np.asarray(sel[j], dtype=np.int64)
        return G[:, r[:, None], c[None, :]]
    return blk


def sel_sigmaimunu2i(sel):
    """0-based chi row map [4, nAtoms, nc, nc] over the orbital subset sel[i] of each site:
    the order of sigmaimunu2i (mod_System.F90:176-187) restricted to those orbitals (local
    indices 0..nc_i-1 in the order of sel[i])."""
    nmax = max(len(x) for x in sel)
    idx = np.full((4, len(sel), nmax, nmax), -1, dtype=np.int64)
    k = 0
    for i, x in enumerate(sel):
        for mu in range(len(x)):
            for nu in range(len(x)):
                for sg in range(4):
                    idx[sg, i, mu, nu] = k
                    k += 1
    return idx


def _scatter_fn(s, sel=None):
    sidx = s.sigmaimunu2i() if sel is None else sel_sigmaimunu2i(sel)
    norbs = s.norbs if sel is None else [len(x) for x in sel]

    def scatter(target, i, j, s1, s2, block):
        # block[mu, nu, gama, xi] -> target[sigmaimunu2i(s1,i,mu,nu), sigmaimunu2i(s2,j,gama,xi)]
        ni, nj = norbs[i], norbs[j]
        rows = sidx[s1 - 1, i, :ni, :ni].reshape(-1)
        cols = sidx[s2 - 1, j, :nj, :nj].reshape(-1)
        target[np.ix_(rows, cols)] += block.reshape(ni * ni, nj * nj)
    return scatter


def _imag_terms(s, g1, g2, w, target, scatter, _blk=_blk):
    """Imaginary-axis integrand of eintshechi.F90:86-104 for G1 = g1, G2 = g2 (weights w), added to target."""
    ia = s.ia()
    norbs = s.norbs
    for j in range(s.n_atoms):
        for i in range(s.n_atoms):
            for (s1, s2), (x1, y1) in TERM1.items():
                a = _blk(g1, ia, norbs, i, j, x1) * w[:, None, None]   # [P, nu, gama]
                b = _blk(g2, ia, norbs, j, i, y1)                      # [P, xi, mu]
                t1 = np.einsum("pvg,pxm->mvgx", a, b, optimize=True)
                x2s, y2s = TERM2[(s1, s2)]
                c = _blk(g2, ia, norbs, i, j, x2s) * w[:, None, None]  # [P, mu, xi]
                d = _blk(g1, ia, norbs, j, i, y2s)                     # [P, gama, nu]
                t2 = np.conj(np.einsum("pmx,pgv->mvgx", c, d, optimize=True))
                scatter(target, i, j, s1, s2, t1 + t2)


def _real_terms(s, g1, g2, w, target, scatter, _blk=_blk):
    """Real-axis integrand of eintshechi.F90:146-164 for G1 = g1, G2 = g2 (weights w), added to target."""
    ia = s.ia()
    norbs = s.norbs
    for j in range(s.n_atoms):
        for i in range(s.n_atoms):
            for (s1, s2), (a1, a2, b1) in REAL.items():
                A = _blk(g1, ia, norbs, i, j, a1) - np.conj(np.swapaxes(_blk(g1, ia, norbs, j, i, a2), 1, 2))
                A = A * w[:, None, None]                           # [P, nu, gama]
                B = np.conj(_blk(g2, ia, norbs, i, j, b1))          # [P, mu, xi]
                blk = -1j * np.einsum("pvg,pmx->mvgx", A, B, optimize=True)
                scatter(target, i, j, s1, s2, blk)


def _real_list(real_bz, x2, p2):
    """Every (energy, k) pair of the real-axis loops (eintshechi.F90:112-170) as one flat list."""
    kpr, wr = real_bz
    nkr = kpr.shape[0]
    xs = np.repeat(np.asarray(x2, float), nkr)
    ws = np.repeat(np.asarray(p2, float), nkr) * np.tile(wr, len(x2))
    ks = np.tile(kpr, (len(x2), 1))
    return xs, ws, ks


def eintshechi(model: Model, mesh, real_bz, q, e, Ef, eta, etap, x2=None, p2=None, chunk=4096, sel=None):
    """chi0_HF(q, e) of eintshechi.F90:2-178 (before the MPI reduction).

    ``mesh`` is the imaginary-axis (E, k) list; ``real_bz`` = (kp, w) of the
    real-axis BZ; (x2, p2) the real-axis energy points (generated by the caller
    with generate_real_epoints).  Returns chiorb_hf[dimens, dimens]; with ``sel``
    (per site, the local orbital indices kept) only the sub-block over those
    orbitals, in the sigmaimunu2i order restricted to them (sel_sigmaimunu2i), with
    the same per-element sums.
    """
    s = model.system
    D = s.dimens if sel is None else 4 * sum(len(x) ** 2 for x in sel)
    blk = _blk if sel is None else _sel_blk(sel)
    chi = np.zeros((D, D), dtype=complex)
    fint = np.zeros((D, D), dtype=complex)
    q = np.asarray(q, float)
    scatter = _scatter_fn(s, sel)
    y = mesh.point_energy()
    for sl in _chunks(mesh.n_points, chunk):
        kp = mesh.kp[sl]
        g1 = model.green(Ef + e + 1j * (y[sl] + eta), kp + q[None, :])   # gfq
        g2 = model.green(Ef + 1j * (y[sl] + etap), kp)                   # gf
        _imag_terms(s, g1, g2, mesh.weight[sl], chi, scatter, blk)
    if x2 is not None and len(x2) > 0:
        xs, ws, ks = _real_list(real_bz, x2, p2)
        for sl in _chunks(xs.shape[0], chunk):
            g1 = model.green(xs[sl] + e + 1j * eta, ks[sl] + q[None, :])
            g2 = model.green(xs[sl] + 1j * etap, ks[sl])
            _real_terms(s, g1, g2, ws[sl], fint, scatter, blk)
    return (chi + fint) / TPI


def sel_rows(system, sel):
    """Rows of the full chiorb_hf that the orbital subset sel keeps, in the subset's order."""
    sidx = system.sigmaimunu2i()
    sub = sel_sigmaimunu2i(sel)
    rows = np.zeros(4 * sum(len(x) ** 2 for x in sel), dtype=np.int64)
    for i, x in enumerate(sel):
        for a, mu in enumerate(x):
            for b, nu in enumerate(x):
                for sg in range(4):
                    rows[sub[sg, i, a, b]] = sidx[sg, i, mu, nu]
    return rows


def eintshechi_linear_soc(model0: Model, vsoc, mesh, real_bz, q, e, Ef, eta, etap, x2=None, p2=None, chunk=2048):
    """eintshechilinearsoc (eintshechi.F90:182-414): chi_HF of G0 = (z - H0)^-1, H0 the
    Hamiltonian without the local SOC (hamiltklinearsoc, mod_hamiltonian.F90:304-396), and its
    first-order SOC correction
        chi_lsoc = chi(G0 V G0 (k+q, E+e), G0(k, E)) + chi(G0(k+q, E+e), G0 V G0 (k, E)),  V = vsoc
    (greenlinearsoc, mod_greenfunction.F90:141-202).  Returns (chiorb_hf, chiorb_hflsoc).
    The real-axis sum runs over every real point; the reference's loop stops after
    realBZ%workload points (the first real energy only, eintshechi.F90:321)."""
    s = model0.system
    D = s.dimens
    V = np.asarray(vsoc, complex)
    chi = np.zeros((D, D), dtype=complex)
    lsoc = np.zeros((D, D), dtype=complex)
    q = np.asarray(q, float)
    scatter = _scatter_fn(s)
    y = mesh.point_energy()
    for sl in _chunks(mesh.n_points, chunk):
        kp = mesh.kp[sl]
        w = mesh.weight[sl]
        g1 = model0.green(Ef + e + 1j * (y[sl] + eta), kp + q[None, :])
        g2 = model0.green(Ef + 1j * (y[sl] + etap), kp)
        v1, v2 = g1 @ V @ g1, g2 @ V @ g2
        _imag_terms(s, g1, g2, w, chi, scatter)
        _imag_terms(s, v1, g2, w, lsoc, scatter)
        _imag_terms(s, g1, v2, w, lsoc, scatter)
    if x2 is not None and len(x2) > 0:
        xs, ws, ks = _real_list(real_bz, x2, p2)
        for sl in _chunks(xs.shape[0], chunk):
            g1 = model0.green(xs[sl] + e + 1j * eta, ks[sl] + q[None, :])
            g2 = model0.green(xs[sl] + 1j * etap, ks[sl])
            v1, v2 = g1 @ V @ g1, g2 @ V @ g2
            _real_terms(s, g1, g2, ws[sl], chi, scatter)
            _real_terms(s, v1, g2, ws[sl], lsoc, scatter)
            _real_terms(s, g1, v2, ws[sl], lsoc, scatter)
    return chi / TPI, lsoc / TPI


def umatrix(system):
    """Umatorb of build_identity_and_U_matrix (mod_susceptibilities.F90:106-159)."""
    D = system.dimens
    U = np.zeros((D, D), dtype=complex)
    sidx = system.sigmaimunu2i()
    Un, Um = system.Un(), system.Um()
    for i, dl in enumerate(system.dorbs):
        for xi in dl:
            for ga in dl:
                for nu in dl:
                    for mu in dl:
                        if mu != nu or ga != xi:
                            continue
                        U[sidx[0, i, mu, nu], sidx[0, i, ga, xi]] = Um[i]
                        U[sidx[1, i, mu, nu], sidx[1, i, ga, xi]] = Un[i]
                        U[sidx[2, i, mu, nu], sidx[2, i, ga, xi]] = Un[i]
                        U[sidx[3, i, mu, nu], sidx[3, i, ga, xi]] = Um[i]
    for i, dl in enumerate(system.dorbs):
        for xi in dl:
            for ga in dl:
                for nu in dl:
                    for mu in dl:
                        if mu != xi or nu != ga:
                            continue
                        for a in (1, 2):
                            for b in (1, 2):
                                U[sidx[a, i, mu, nu], sidx[b, i, ga, xi]] -= Un[i]
    return U


def dyson(chi_hf, U):
    """chi_RPA = (1 + chi_HF U)^-1 chi_HF (calculate_chi.F90:85-89)."""
    D = chi_hf.shape[0]
    temp = np.eye(D, dtype=complex) + chi_hf @ U
    return np.linalg.inv(temp) @ chi_hf


def site_reduce(system, chi):
    """4x4 site blocks schi(sigmai2i(s,i), sigmai2i(s',j)) = sum_{mu,nu} chi(s,i,mu,mu; s',j,nu,nu)."""
    nat = system.n_atoms
    sidx = system.sigmaimunu2i()
    out = np.zeros((4 * nat, 4 * nat), dtype=complex)
    for j in range(nat):
        for i in range(nat):
            for sp in range(4):
                for sg in range(4):
                    r = [sidx[sg, i, m, m] for m in range(system.norbs[i])]
                    c = [sidx[sp, j, n, n] for n in range(system.norbs[j])]
                    out[sg * nat + i, sp * nat + j] = chi[np.ix_(r, c)].sum()
    return out


def golden_row(system, e, q_abs, schi, i, j):
    """Values of one output line ((Re, Im) schi(n,i; m,j), n = 1..4), m = 1..4 (mod_susceptibilities.F90:331-336)."""
    nat = system.n_atoms
    vals = [e, q_abs]
    for m in range(4):
        for n in range(4):
            v = schi[n * nat + i, m * nat + j]
            vals += [v.real, v.imag]
    return vals


def expectation(model: Model, mesh, Ef, eta, chunk=4096):
    """rho, mx, my, mz, mp per (site, orbital) (mod_expectation.F90:28-149)."""
    s = model.system
    ia = s.ia()
    nat = s.n_atoms
    nmax = max(s.norbs)
    imguu = np.zeros((nat, nmax))
    imgdd = np.zeros((nat, nmax))
    gud = np.zeros((nat, nmax), dtype=complex)
    gdu = np.zeros((nat, nmax), dtype=complex)
    y = mesh.point_energy()
    for sl in _chunks(mesh.n_points, chunk):
        G = model.green(Ef + 1j * (y[sl] + eta), mesh.kp[sl])
        w = mesh.weight[sl]
        for i in range(nat):
            n = s.norbs[i]
            b = ia[i][0]
            for mu in range(n):
                mup = mu + n
                gud[i, mu] += np.sum(G[:, b + mu, b + mup] * w)
                gdu[i, mu] += np.sum(G[:, b + mup, b + mu] * w)
                imguu[i, mu] += np.sum(G[:, b + mu, b + mu].real * w)
                imgdd[i, mu] += np.sum(G[:, b + mup, b + mup].real * w)
    imguu /= PI
    imgdd /= PI
    mp = (gdu + np.conj(gud)) / PI
    imguu = 0.5 + imguu
    imgdd = 0.5 + imgdd
    for i in range(nat):
        imguu[i, s.norbs[i]:] = 0.0
        imgdd[i, s.norbs[i]:] = 0.0
    rho = imguu + imgdd
    mz = imguu - imgdd
    return rho, mp.real.copy(), mp.imag.copy(), mz, mp


# ---------------------------------------------------------------------------
# Self-consistency unknowns and the analytic Jacobian
# ---------------------------------------------------------------------------
def equation_layout(system, fixEf=False):
    """neq_per_atom and neq (mod_self_consistency.F90:517-523), constr_type = default."""
    per = [0]
    for i in range(system.n_atoms):
        nd = len(system.dorbs[i])
        c = (nd if abs(system.Un()[i]) > 1e-8 else 0) + (3 if abs(system.Um()[i]) > 1e-8 else 0)
        per.append(per[-1] + c)
    neq = per[-1] + (0 if fixEf else 1)
    return per, neq


def _pauli_site(n, which, dorbs, d_only):
    """pauli_orb / pauli_dorb(which) of one site, 2n x 2n (mod_constants.F90:83-148)."""
    P = np.zeros((2 * n, 2 * n), dtype=complex)
    orbs = dorbs if d_only else range(n)
    for mu in orbs:
        nu = mu + n
        if which == 0:
            P[mu, mu] = 1
            P[nu, nu] = 1
        elif which == 1:
            P[mu, nu] = 1
            P[nu, mu] = 1
        elif which == 2:
            P[mu, nu] = -1j
            P[nu, mu] = 1j
        elif which == 3:
            P[mu, mu] = 1
            P[nu, nu] = -1
    return P


def jacobian(model: Model, mesh, real_bz, Ef, eta, fixEf=False, chunk=2048):
    """calcJacobian_greenfunction (mod_self_consistency.F90:795-1205), plain GF path."""
    s = model.system
    per, neq = equation_layout(s, fixEf)
    J = np.zeros((neq, neq))
    ia = s.ia()
    nat = s.n_atoms
    Un, Um = s.Un(), s.Um()
    halfUn = -0.5 * Un
    halfUm = -0.5 * Um

    def site_block(G, i, j):
        return G[:, ia[i][0]:ia[i][3], ia[j][0]:ia[j][3]]

    y = mesh.point_energy()
    for sl in _chunks(mesh.n_points, chunk):
        G = model.green(Ef + 1j * (y[sl] + eta), mesh.kp[sl])
        w = mesh.weight[sl]
        for j in range(nat):
            nj = s.norbs[j]
            dj = s.dorbs[j]
            for i in range(nat):
                ni = s.norbs[i]
                di = s.dorbs[i]
                gij = site_block(G, i, j)
                gji = site_block(G, j, i)
                temp1 = [np.einsum("ab,pbc->pac", _pauli_site(ni, sg, di, sg != 0), gij) for sg in range(4)]

                def diag_sum(t1, t2, orbs_list):
                    # real(temp(mud,mud) + temp(nud,nud)) summed over points with weight
                    d = np.einsum("prc,pcr->pr", t1, t2)          # diag of t1 @ t2
                    vals = []
                    for mu in orbs_list:
                        vals.append(np.sum((d[:, mu] + d[:, mu + ni]) * w).real)
                    return vals

                kountj = per[j]
                if abs(Un[j]) > 1e-8:
                    for nu_i, nud in enumerate(dj):
                        kounti = per[i]
                        pt = _pauli_site(nj, 0, dj, True)
                        pt[nud, nud] -= 2.0
                        pt[nud + nj, nud + nj] -= 2.0
                        t2 = halfUn[j] * np.einsum("ab,pbc->pac", pt, gji)
                        if abs(Un[i]) > 1e-8:
                            v = diag_sum(temp1[0], t2, di)
                            for m, val in enumerate(v):
                                J[kounti + m, kountj + nu_i] += val
                            kounti = per[i] + len(di)
                        if not fixEf:
                            J[neq - 1, kountj + nu_i] += sum(diag_sum(temp1[0], t2, range(ni)))
                        if abs(Um[i]) > 1e-8:
                            for sg in range(1, 4):
                                J[kounti + sg - 1, kountj + nu_i] += sum(diag_sum(temp1[sg], t2, di))
                    kountj = per[j] + len(dj)
                if abs(Um[j]) > 1e-8:
                    t2s = {sp: halfUm[j] * np.einsum("ab,pbc->pac", _pauli_site(nj, sp, dj, True), gji)
                           for sp in range(1, 4)}
                    for sp in range(1, 4):
                        kounti = per[i]
                        if abs(Un[i]) > 1e-8:
                            v = diag_sum(temp1[0], t2s[sp], di)
                            for m, val in enumerate(v):
                                J[kounti + m, kountj + sp - 1] += val
                            kounti = per[i] + len(di)
                        if not fixEf:
                            J[neq - 1, kountj + sp - 1] += sum(diag_sum(temp1[0], t2s[sp], range(ni)))
                        if abs(Um[i]) > 1e-8:
                            for sg in range(1, 4):
                                J[kounti + sg - 1, kountj + sp - 1] += sum(diag_sum(temp1[sg], t2s[sp], di))
    if not fixEf:
        kpr, wr = real_bz
        for sl in _chunks(kpr.shape[0], chunk):
            G = model.green(np.full(kpr[sl].shape[0], Ef + 1j * eta), kpr[sl])
            w = wr[sl]
            for i in range(nat):
                ni = s.norbs[i]
                di = s.dorbs[i]
                gii = site_block(G, i, i)
                kounti = per[i]
                tmp = np.einsum("ab,pbc->pac", _pauli_site(ni, 0, di, False), gii) * w[:, None, None]
                dg = np.einsum("prr->pr", tmp).sum(axis=0)
                if abs(Un[i]) > 1e-8:
                    for m, mud in enumerate(di):
                        J[kounti + m, neq - 1] -= (dg[mud] + dg[mud + ni]).imag
                    kounti = per[i] + len(di)
                J[neq - 1, neq - 1] -= sum((dg[mu] + dg[mu + ni]).imag for mu in range(ni))
                if abs(Um[i]) > 1e-8:
                    for sg in range(1, 4):
                        tmp = np.einsum("ab,pbc->pac", _pauli_site(ni, sg, di, True), gii) * w[:, None, None]
                        dg = np.einsum("prr->pr", tmp).sum(axis=0)
                        J[kounti + sg - 1, neq - 1] -= sum((dg[mud] + dg[mud + ni]).imag for mud in di)
    J /= PI
    for k in range(neq - 1):
        J[k, k] -= 1.0
    return J


def unknowns_from_state(system, state, fixEf=False):
    """set_hamiltonian_variables(set=.false.) (mod_self_consistency.F90:1754-1780)."""
    per, neq = equation_layout(system, fixEf)
    x = np.zeros(neq)
    rd, xd, yd, zd = state.d_totals(system.dorbs)
    for i in range(system.n_atoms):
        k = per[i]
        if abs(system.Un()[i]) > 1e-8:
            for m, mu in enumerate(system.dorbs[i]):
                x[k + m] = state.rho[i, mu]
            k = per[i] + len(system.dorbs[i])
        if abs(system.Um()[i]) > 1e-8:
            x[k:k + 3] = [xd[i], yd[i], zd[i]]
    if not fixEf:
        x[neq - 1] = state.Ef
    return x


def state_from_unknowns(system, x, template, fixEf=False):
    """set_hamiltonian_variables(set=.true.): the inputs that enter hee (and Ef)."""
    from titan_b200.host.system import MagState
    per, neq = equation_layout(system, fixEf)
    st = MagState(template.rho.copy(), np.zeros_like(template.mx), np.zeros_like(template.my),
                  np.zeros_like(template.mz), template.Ef)
    for i in range(system.n_atoms):
        k = per[i]
        dl = system.dorbs[i]
        if abs(system.Un()[i]) > 1e-8:
            for m, mu in enumerate(dl):
                st.rho[i, mu] = x[k + m]
            k = per[i] + len(dl)
        if abs(system.Um()[i]) > 1e-8:
            # only the d totals enter hee; spread them over the d orbitals
            for mu in dl:
                st.mx[i, mu] = x[k] / len(dl)
                st.my[i, mu] = x[k + 1] / len(dl)
                st.mz[i, mu] = x[k + 2] / len(dl)
    if not fixEf:
        st.Ef = float(x[neq - 1])
    return st


def sc_residual(system, model_factory, mesh, x, template, fixEf=False):
    """sc_eqs: fvec = out - in, plus the charge-neutrality line (mod_self_consistency.F90:1516-1628)."""
    per, neq = equation_layout(system, fixEf)
    st_in = state_from_unknowns(system, x, template, fixEf)
    model = model_factory(st_in)
    rho, mx, my, mz, mp = expectation(model, mesh, st_in.Ef, system.eta)
    out = template.__class__(rho, mx, my, mz, st_in.Ef)
    rd, xd, yd, zd = out.d_totals(system.dorbs)
    rdi, xdi, ydi, zdi = st_in.d_totals(system.dorbs)
    f = np.zeros(neq)
    for i in range(system.n_atoms):
        k = per[i]
        dl = system.dorbs[i]
        if abs(system.Un()[i]) > 1e-8:
            for m, mu in enumerate(dl):
                f[k + m] = rho[i, mu] - st_in.rho[i, mu]
            k = per[i] + len(dl)
        if abs(system.Um()[i]) > 1e-8:
            f[k:k + 3] = [xd[i] - xdi[i], yd[i] - ydi[i], zd[i] - zdi[i]]
    if not fixEf:
        f[neq - 1] = rho.sum() - system.total_occupation()
    return f, out, model


def self_consistency(system, model_factory, mesh, real_bz, state0, fixEf=False, tol=1e-12, maxit=40):
    """Newton iteration with the analytic Jacobian to the root dnsqe finds."""
    x = unknowns_from_state(system, state0, fixEf)
    template = state0
    out = None
    for it in range(maxit):
        f, out, model = sc_residual(system, model_factory, mesh, x, template, fixEf)
        Ef = x[-1] if not fixEf else template.Ef
        J = jacobian(model, mesh, real_bz, Ef, system.eta, fixEf)
        dx = np.linalg.solve(J, -f)
        x = x + dx
        if np.max(np.abs(dx)) <= tol * max(1.0, np.max(np.abs(x))):
            break
    f, out, model = sc_residual(system, model_factory, mesh, x, template, fixEf)
    return x, out, f, it + 1


# ---------------------------------------------------------------------------
# Disturbance response (eintshe + calculate_all), source/eintshe.F90:2-309,
# source/dtdksub.F90:2-28, source/calculate_all.F90:72-420.
# Imaginary axis (eintshe.F90:104-179): for (sigma, sigma') the spin blocks
# (X, Y, Z, W) of G1^X(nu,gama;i,j) G2^Y(xi,mu;l,i) + conj(G2^Z(mu,xi;i,l) G1^W(gama,nu;j,i)),
# both terms times dtdk(gama,xi;j,l).
# ---------------------------------------------------------------------------
SHE_IMAG = {(1, 1): ("dd", "uu", "uu", "dd"), (1, 2): ("du", "uu", "uu", "ud"), (1, 3): ("dd", "du", "ud", "dd"),
            (1, 4): ("du", "du", "ud", "ud"),
            (2, 1): ("ud", "uu", "uu", "du"), (2, 2): ("uu", "uu", "uu", "uu"), (2, 3): ("ud", "du", "ud", "du"),
            (2, 4): ("uu", "du", "ud", "uu"),
            (3, 1): ("dd", "ud", "du", "dd"), (3, 2): ("du", "ud", "du", "ud"), (3, 3): ("dd", "dd", "dd", "dd"),
            (3, 4): ("du", "dd", "dd", "ud"),
            (4, 1): ("ud", "ud", "du", "du"), (4, 2): ("uu", "ud", "du", "uu"), (4, 3): ("ud", "dd", "dd", "du"),
            (4, 4): ("uu", "dd", "dd", "uu")}
# Real axis (eintshe.F90:226-249): -i (G1^X(nu,gama;i,j) - conj(G1^X'(gama,nu;j,i))) conj(G2^Y(mu,xi;i,l)) dtdk
SHE_REAL = {(1, 1): ("dd", "dd", "uu"), (1, 2): ("du", "ud", "uu"), (1, 3): ("dd", "dd", "ud"), (1, 4): ("du", "ud", "ud"),
            (2, 1): ("ud", "du", "uu"), (2, 2): ("uu", "uu", "uu"), (2, 3): ("ud", "du", "ud"), (2, 4): ("uu", "uu", "ud"),
            (3, 1): ("dd", "dd", "du"), (3, 2): ("du", "ud", "du"), (3, 3): ("dd", "dd", "dd"), (3, 4): ("du", "ud", "dd"),
            (4, 1): ("ud", "du", "du"), (4, 2): ("uu", "uu", "du"), (4, 3): ("ud", "du", "dd"), (4, 4): ("uu", "uu", "dd")}


def _orbital_offsets(norbs):
    off = [0]
    for n in norbs:
        off.append(off[-1] + n)
    return off


def dtdk(system, kp, ue):
    """dtdksub: sum_neigh i (ue . R) t0i exp(i k . R), spinless orbital space (rows site j, cols site i)."""
    cv, bi, ish, t = system.neighbor_table()
    off = _orbital_offsets(system.norbs)
    kp = np.atleast_2d(kp)
    D = np.zeros((kp.shape[0], off[-1], off[-1]), dtype=complex)
    ph = 1j * (cv @ np.asarray(ue, float))[None, :] * np.exp(1j * kp @ cv.T)
    for k in range(cv.shape[0]):
        j = int(bi[k])
        for i in range(system.n_atoms):
            if ish[k, i]:
                nj, ni = system.norbs[j], system.norbs[i]
                D[:, off[j]:off[j] + nj, off[i]:off[i] + ni] += ph[:, k, None, None] * t[k, i, :nj, :ni][None]
    return D


def _spin_blocks(G, system):
    """{ab: G^{ab}} over all sites in the spinless orbital index space."""
    ia = system.ia()
    out = {}
    for a in "ud":
        for b in "ud":
            rows = [ia[i][0] + _SPIN[a] * system.norbs[i] + m for i in range(system.n_atoms) for m in range(system.norbs[i])]
            cols = [ia[i][0] + _SPIN[b] * system.norbs[i] + m for i in range(system.n_atoms) for m in range(system.norbs[i])]
            out[a + b] = G[:, rows][:, :, cols]
    return out


def eintshe(model: Model, mesh, real_bz, q, e, Ef, eta, etap, x2, p2, efield, chunk=2048):
    """Sum over (k, E) of the disturbance integrand df1iikl (dimens x 4) over 2 pi, before the
    prefactor (eintshe.F90:2-309; the reference multiplies every point by the constant
    prefactor, which is applied once to the sum here)."""
    s = model.system
    sidx = s.sigmaimunu2i()
    off = _orbital_offsets(s.norbs)
    df = np.zeros((s.dimens, 4), dtype=complex)
    q = np.asarray(q, float)

    def accumulate(sig, sigp, blk_num, w, transpose):
        # blk_num[p, (i a), (i b)]: rows nu / cols mu (transpose=False) or rows mu / cols nu
        for i in range(s.n_atoms):
            n = s.norbs[i]
            b = blk_num[:, off[i]:off[i] + n, off[i]:off[i] + n]
            c = np.einsum("p,pab->ab", w, b)
            c = c if transpose else c.T     # -> [mu, nu]
            df[sidx[sig - 1, i, :n, :n].reshape(-1), sigp - 1] += c.reshape(-1)

    y = mesh.point_energy()
    for sl in _chunks(mesh.n_points, chunk):
        kp = mesh.kp[sl]
        w = mesh.weight[sl]
        g1 = _spin_blocks(model.green(Ef + e + 1j * (y[sl] + eta), kp + q[None, :]), s)
        g2 = _spin_blocks(model.green(Ef + 1j * (y[sl] + etap), kp), s)
        D = dtdk(s, kp, efield)
        DT = np.swapaxes(D, 1, 2)
        for (sig, sigp), (X, Y, Z, W) in SHE_IMAG.items():
            t1 = g1[X] @ D @ g2[Y]                                  # [(i nu), (i mu)]
            t2 = np.conj(g2[Z]) @ DT @ np.conj(g1[W])               # [(i mu), (i nu)]
            accumulate(sig, sigp, t1, w, False)
            accumulate(sig, sigp, t2, w, True)
    if x2 is not None and len(x2) > 0:
        kpr, wr = real_bz
        nkr = kpr.shape[0]
        xs = np.repeat(np.asarray(x2, float), nkr)
        ws = np.repeat(np.asarray(p2, float), nkr) * np.tile(wr, len(x2))
        ks = np.tile(kpr, (len(x2), 1))
        for sl in _chunks(xs.shape[0], chunk):
            kp = ks[sl]
            g1 = _spin_blocks(model.green(xs[sl] + e + 1j * eta, kp + q[None, :]), s)
            g2 = _spin_blocks(model.green(xs[sl] + 1j * etap, kp), s)
            D = dtdk(s, kp, efield)
            for (sig, sigp), (X, Xp, Y) in SHE_REAL.items():
                A = g1[X] - np.conj(np.swapaxes(g1[Xp], 1, 2))
                t = -1j * (A @ D @ np.conj(np.swapaxes(g2[Y], 1, 2)))   # [(i nu), (i mu)]
                accumulate(sig, sigp, t, ws[sl], False)
    return df / TPI


def type_lvec(orbs):
    """Types%lvec: L_x, L_y, L_z restricted to a type's orbitals (mod_magnet.F90:295-345)."""
    from titan_b200.host.onsite import l_matrices
    L = l_matrices()
    idx = [o - 1 for o in orbs]
    return L[:, idx][:, :, idx]


def disturbance_outputs(system, chi_hf, tchi_raw, U, lvec, lambda_p, lambda_d, porbs, dorbs, mvec=None, hhw=None):
    """calculate_all.F90:126-420: prefactor, tchiorbiikl, disturbances(7, site), torques(3, 3, site),
    Beff_cart(4, site) and their site sums.  lvec[i] = L (3, nOrb, nOrb) of site i (lpvec at
    theta = phi = 0); porbs/dorbs = local p / d orbital indices per site."""
    nat = system.n_atoms
    D = system.dimens
    sidx = system.sigmaimunu2i()
    prefactor = np.linalg.inv(np.eye(D) + chi_hf @ U)
    T = prefactor @ tchi_raw
    chiorb = prefactor @ chi_hf

    def s2i(sig, i):
        return (sig - 1) * nat + i

    chiinv = np.zeros((4 * nat, 4 * nat), dtype=complex)
    for i in range(nat):
        for j in range(nat):
            for sig in range(1, 5):
                for sigp in range(1, 5):
                    for mu in range(system.norbs[i]):
                        for nu in range(system.norbs[j]):
                            chiinv[s2i(sig, i), s2i(sigp, j)] += chiorb[sidx[sig - 1, i, mu, mu], sidx[sigp - 1, j, nu, nu]]
    chiinv = np.linalg.inv(chiinv)
    dist = np.zeros((7, nat), dtype=complex)
    torq = np.zeros((3, 3, nat), dtype=complex)
    sdmat = np.zeros(4 * nat, dtype=complex)

    def tt(sig, i, mu, nu, col):
        return T[sidx[sig - 1, i, mu, nu], col - 1]

    for i in range(nat):
        for mu in range(system.norbs[i]):
            dist[0, i] += tt(2, i, mu, mu, 2) + tt(2, i, mu, mu, 3) + tt(3, i, mu, mu, 2) + tt(3, i, mu, mu, 3)
            dist[1, i] += tt(1, i, mu, mu, 2) + tt(1, i, mu, mu, 3) + tt(4, i, mu, mu, 2) + tt(4, i, mu, mu, 3)
            dist[2, i] += (tt(1, i, mu, mu, 2) + tt(1, i, mu, mu, 3) - tt(4, i, mu, mu, 2) - tt(4, i, mu, mu, 3)) / 1j
            dist[3, i] += tt(2, i, mu, mu, 2) + tt(2, i, mu, mu, 3) - tt(3, i, mu, mu, 2) - tt(3, i, mu, mu, 3)
        sdmat[s2i(1, i)] = dist[1, i] + 1j * dist[2, i]
        sdmat[s2i(2, i)] = dist[0, i] + dist[3, i]
        sdmat[s2i(3, i)] = dist[0, i] - dist[3, i]
        sdmat[s2i(4, i)] = dist[1, i] - 1j * dist[2, i]
        n = system.norbs[i]
        for mu in range(n):
            for nu in range(n):
                ld = tt(2, i, mu, nu, 2) + tt(2, i, mu, nu, 3) + tt(3, i, mu, nu, 2) + tt(3, i, mu, nu, 3)
                for c in range(3):
                    dist[4 + c, i] += lvec[i][c, mu, nu] * ld
        for lam, orbl in ((lambda_p, porbs[i]), (lambda_d, dorbs[i])):
            for nu in orbl:
                for mu in orbl:
                    lp = lvec[i][:, mu, nu]
                    a = tt(2, i, mu, nu, 2) + tt(2, i, mu, nu, 3) - tt(3, i, mu, nu, 2) - tt(3, i, mu, nu, 3)
                    b = tt(1, i, mu, nu, 2) + tt(1, i, mu, nu, 3) - tt(4, i, mu, nu, 2) - tt(4, i, mu, nu, 3)
                    c = tt(1, i, mu, nu, 2) + tt(1, i, mu, nu, 3) + tt(4, i, mu, nu, 2) + tt(4, i, mu, nu, 3)
                    torq[0, 0, i] += lam * (lp[1] * a) + lam * (1j * lp[2] * b)
                    torq[0, 1, i] += lam * (lp[2] * c) - lam * (lp[0] * a)
                    torq[0, 2, i] += -lam * (1j * lp[0] * b) - lam * (lp[1] * c)
        torq[0, :, i] *= 0.5
        um = system.Um()[i]
        m = np.zeros(3) if mvec is None else mvec[i]
        torq[1, 0, i] = um * (m[2] * dist[2, i] - m[1] * dist[3, i])
        torq[1, 1, i] = um * (m[0] * dist[3, i] - m[2] * dist[1, i])
        torq[1, 2, i] = um * (m[1] * dist[1, i] - m[0] * dist[2, i])
        if hhw is not None:
            h = hhw[i]
            torq[2, 0, i] = 2 * (h[1] * dist[3, i] - h[2] * dist[2, i])
            torq[2, 1, i] = 2 * (h[2] * dist[1, i] - h[0] * dist[3, i])
            torq[2, 2, i] = 2 * (h[0] * dist[2, i] - h[1] * dist[1, i])
    dist[1:4] *= 0.5
    sdmat *= 0.5
    beff = chiinv @ sdmat
    bc = np.zeros((4, nat), dtype=complex)
    for i in range(nat):
        bc[0, i] = beff[s2i(2, i)] + beff[s2i(3, i)]
        bc[1, i] = 0.5 * (beff[s2i(1, i)] + beff[s2i(4, i)])
        bc[2, i] = -0.5j * (beff[s2i(1, i)] - beff[s2i(4, i)])
        bc[3, i] = 0.5 * (beff[s2i(2, i)] - beff[s2i(3, i)])
    return {"tchiorbiikl": T, "disturbances": dist, "torques": torq, "beff": bc,
            "total_disturbances": dist.sum(axis=1), "total_torques": torq.sum(axis=2), "total_beff": bc.sum(axis=1)}


# ---------------------------------------------------------------------------
# Local density of states on the real axis, source/mod_LDOS.F90:95-150 (ldos_energy):
# ldosu(i, mu) = -(1/pi) sum_k w_k Im G(i up mu, i up mu; k, e + i eta), ldosd with the down block.
# ---------------------------------------------------------------------------
def gs_orbital(model: Model, mesh, Ef, eta, chunk=4096):
    """gupgd of calc_GS_L_and_E_greenfunction (mod_expectation.F90:912-982) as [i, a, b] =
    gupgd(a, b, i) = (1/pi) sum w (G(i b up, i a up) + G(i b dn, i a dn))."""
    s = model.system
    ia = s.ia()
    nmax = max(s.norbs)
    out = np.zeros((s.n_atoms, nmax, nmax), dtype=complex)
    y = mesh.point_energy()
    for sl in _chunks(mesh.n_points, chunk):
        G = model.green(Ef + 1j * (y[sl] + eta), mesh.kp[sl])
        w = mesh.weight[sl]
        for i in range(s.n_atoms):
            n = s.norbs[i]
            b = ia[i][0]
            up = G[:, b:b + n, b:b + n]
            dn = G[:, b + n:b + 2 * n, b + n:b + 2 * n]
            # gupgd(nu, mu) += G(mu, nu) + G(mu', nu')
            out[i, :n, :n] += np.einsum("p,pmn->nm", w, up + dn)
    return out / PI


def ldos(model: Model, real_bz, energies, eta, chunk=4096):
    """(ldosu, ldosd) [n_e, nAtoms, nOrbMax] at each energy e (absolute, as green(e, eta) is called)."""
    s = model.system
    kp, w = real_bz
    ia = s.ia()
    nmax = max(s.norbs)
    up = np.zeros((len(energies), s.n_atoms, nmax))
    dn = np.zeros((len(energies), s.n_atoms, nmax))
    for ie, e in enumerate(energies):
        for sl in _chunks(kp.shape[0], chunk):
            G = model.green(np.full(kp[sl].shape[0], e + 1j * eta), kp[sl])
            d = np.einsum('kii->ki', G).imag
            for i in range(s.n_atoms):
                n = s.norbs[i]
                r0 = ia[i][0]
                up[ie, i, :n] -= w[sl] @ d[:, r0:r0 + n]
                dn[ie, i, :n] -= w[sl] @ d[:, r0 + n:r0 + 2 * n]
    return up / PI, dn / PI


# ---------------------------------------------------------------------------
# Sum rule of the static transverse susceptibility, source/mod_sumrule.F90:10-245.
# ---------------------------------------------------------------------------
# spin (+, up, down, -) <-> cartesian (0, x, y, z) transforms, mod_constants.F90:34-44 (row index first)
STOC = np.array([[0, 1, 1, 0], [0.5, 0, 0, 0.5], [-0.5j, 0, 0, 0.5j], [0, 0.5, -0.5, 0]], dtype=complex)
CTOS = np.array([[0, 1, 1j, 0], [0.5, 0, 0, 1], [0.5, 0, 0, -1], [0, 1, -1j, 0]], dtype=complex)


def _levi_civita():
    e = np.zeros((3, 3, 3))
    for a, b, c in ((0, 1, 2), (1, 2, 0), (2, 0, 1)):
        e[a, b, c] = 1.0
        e[a, c, b] = -1.0
    return e


def smunu(model: Model, mesh, Ef, eta, chunk=2048):
    """calcSmunu (mod_sumrule.F90:162-245): S[i, k, mu, nu], k = x, y, z."""
    s = model.system
    ia = s.ia()
    nmax = max(s.norbs)
    blk = [np.zeros((2 * n, 2 * n), dtype=complex) for n in s.norbs]
    y = mesh.point_energy()
    for sl in _chunks(mesh.n_points, chunk):
        G = model.green(Ef + 1j * (y[sl] + eta), mesh.kp[sl])
        for i, n in enumerate(s.norbs):
            r0 = ia[i][0]
            blk[i] += np.einsum('p,pab->ab', mesh.weight[sl], G[:, r0:r0 + 2 * n, r0:r0 + 2 * n])
    S = np.zeros((s.n_atoms, 3, nmax, nmax), dtype=complex)
    for i, n in enumerate(s.norbs):
        A = blk[i]

        def img(sx, sy):
            # img[mu, nu] = (A[nu X, mu Y] + conj(A[mu Y, nu X])) / 2 pi
            ax = A[sx * n:(sx + 1) * n, sy * n:(sy + 1) * n]        # [nu, mu]
            ay = A[sy * n:(sy + 1) * n, sx * n:(sx + 1) * n]        # [mu, nu]
            return (ax.T + np.conj(ay)) / TPI
        uu, dd, ud, du = img(0, 0), img(1, 1), img(0, 1), img(1, 0)
        uu = uu + 0.5 * np.eye(n)
        dd = dd + 0.5 * np.eye(n)
        S[i, 0, :n, :n] = ud + du
        S[i, 1, :n, :n] = (ud - du) * 1j
        S[i, 2, :n, :n] = uu - dd
    return S


def beff_sumrule(system, mvec, lvec, lambda_p, lambda_d, porbs, dorbs, Um, hhw=None):
    """Beffective (mod_sumrule.F90:111-160): Beff[dimens] on the cartesian rows sigma = x, y, z."""
    sidx = system.sigmaimunu2i()
    B = np.zeros(system.dimens, dtype=complex)
    for i in range(system.n_atoms):
        for sg in range(3):
            for mu in dorbs[i]:
                B[sidx[sg + 1, i, mu, mu]] -= 0.5 * Um[i] * mvec[i][sg]
            if hhw is not None:
                for mu in range(system.norbs[i]):
                    B[sidx[sg + 1, i, mu, mu]] += hhw[i][sg]
            for lam, orbl in ((lambda_p[i], porbs[i]), (lambda_d[i], dorbs[i])):
                for nu in orbl:
                    for mu in orbl:
                        B[sidx[sg + 1, i, mu, nu]] += 0.5 * lam * lvec[i][sg, mu, nu]
    return B


def sumrule(system, chi_hf, S, B):
    """sumrule (mod_sumrule.F90:10-107): lhs, rhs [group (i, mu, nu), m, n] and sum |lhs - rhs|;
    groups run over the on-site orbital pairs in sigmaimunu2i order."""
    sidx = system.sigmaimunu2i()
    groups = [(i, mu, nu) for i in range(system.n_atoms) for mu in range(system.norbs[i])
              for nu in range(system.norbs[i])]
    IDX = np.array([[sidx[r, i, mu, nu] for r in range(4)] for (i, mu, nu) in groups])   # [group, spin]
    # cart(p, q) = sum_{r, t} StoC(p, r) chi(r, t) CtoS(t, q) for every pair of groups
    chi4 = chi_hf[IDX[:, :, None, None], IDX[None, None, :, :]]                     # [g, r, h, t]
    cart = np.einsum('pr,grht,tq->gphq', STOC, chi4, CTOS)
    eps = _levi_civita()
    Sg = np.array([S[i, :, mu, nu] for (i, mu, nu) in groups])                       # [g, k]
    lhs = np.einsum('mnk,gk->gmn', eps, Sg)
    Bg = B[IDX]                                                                        # [h, spin]
    rhs = 2.0 * np.einsum('nqp,gmhp,hq->gmn', eps, cart[:, 1:, :, 1:], Bg[:, 1:])
    return lhs, rhs, float(np.sum(np.abs(lhs - rhs)))


# ---------------------------------------------------------------------------
# Exchange coupling J_ij(q), source/jij_energy.F90:6-242 (normal state).
# ---------------------------------------------------------------------------
def dbxc_dm(system, evec, Um, dorbs):
    """dBxc_dm[i][mu] (2 nOrb x 2 nOrb): -Um/2 (sigma^d_mu - (sigma^d . e) e_mu), jij_energy.F90:55-64."""
    sig = [np.array([[0, 1], [1, 0]], complex), np.array([[0, -1j], [1j, 0]]), np.array([[1, 0], [0, -1]], complex)]
    out = []
    for i, n in enumerate(system.norbs):
        P = np.zeros((3, 2 * n, 2 * n), dtype=complex)
        for a in range(3):
            for d in dorbs[i]:
                P[a][np.ix_([d, d + n], [d, d + n])] = sig[a]
        e = np.asarray(evec[i], float)
        pe = P[0] * e[0] + P[1] * e[1] + P[2] * e[2]
        out.append([-0.5 * Um[i] * (P[mu] - pe * e[mu]) for mu in range(3)])
    return out


def jij(model: Model, mesh, q, Ef, eta, evec, Um, dorbs, chunk=1024):
    """J[i, j, mu, nu] = -1/(2 pi) sum w [Tr(A G_ij(k) B G_ji(k-q)) + conj Tr(A G_ij(k-q) B G_ji(k))]."""
    s = model.system
    ia = s.ia()
    nat = s.n_atoms
    A = dbxc_dm(s, evec, Um, dorbs)
    q = np.asarray(q, float)
    J = np.zeros((nat, nat, 3, 3), dtype=complex)
    y = mesh.point_energy()
    blk = [slice(ia[i][0], ia[i][0] + 2 * s.norbs[i]) for i in range(nat)]
    for sl in _chunks(mesh.n_points, chunk):
        z = Ef + 1j * (y[sl] + eta)
        G = model.green(z, mesh.kp[sl])
        Gm = model.green(z, mesh.kp[sl] - q[None, :])
        w = mesh.weight[sl]
        for j in range(nat):
            for i in range(nat):
                gij, gji = G[:, blk[i], blk[j]], G[:, blk[j], blk[i]]
                gijm, gjim = Gm[:, blk[i], blk[j]], Gm[:, blk[j], blk[i]]
                for nu in range(3):
                    for mu in range(3):
                        t1 = np.einsum("ab,pbc,cd,pda->p", A[i][mu], gij, A[j][nu], gjim, optimize=True)
                        t2 = np.einsum("ab,pbc,cd,pda->p", A[i][mu], gijm, A[j][nu], gji, optimize=True)
                        J[i, j, mu, nu] += np.sum(w * (t1 + np.conj(t2)))
    return -J / TPI
