"""numpy GG tensor and Fermi column (test helpers, CPU)."""
import numpy as np

SIG = [np.eye(2), np.array([[0, 1], [1, 0]]), np.array([[0, -1j], [1j, 0]]), np.diag([1.0, -1.0])]


def groups(system, resolved=True):
    rowg, colg = [], []
    for i in range(system.n_atoms):
        d = sorted(system.dorbs[i])
        rest = [o for o in range(system.norbs[i]) if o not in d]
        if resolved:
            rowg.append([[o] for o in d] + [rest])
            colg.append([[o] for o in d])
        else:
            allo = list(range(system.norbs[i]))
            rowg.append([allo])
            colg.append([allo])
    return rowg, colg


def gg_tensor_numpy(system, G, w, resolved=True):
    """T[i, j, g, h, s' + 2t + 4t' + 8s] = sum_p w_p sum_{mu in g, nu in h} G(i s' mu, j t nu) G(j t' nu, i s mu)."""
    ia = system.ia()
    nat = system.n_atoms
    rowg, colg = groups(system, resolved)
    nrow = max(len(r) for r in rowg)
    ncol = max(len(c) for c in colg)
    T = np.zeros((nat, nat, nrow, ncol, 16), complex)
    for i in range(nat):
        ni = system.norbs[i]
        for j in range(nat):
            nj = system.norbs[j]
            for g, rows in enumerate(rowg[i]):
                for h, cols in enumerate(colg[j]):
                    if not rows or not cols:
                        continue
                    for q in range(16):
                        sp, t, tp, s = q & 1, (q >> 1) & 1, (q >> 2) & 1, (q >> 3) & 1
                        r1 = [ia[i][0] + sp * ni + m for m in rows]
                        c1 = [ia[j][0] + t * nj + n for n in cols]
                        r2 = [ia[j][0] + tp * nj + n for n in cols]
                        c2 = [ia[i][0] + s * ni + m for m in rows]
                        A = G[:, r1][:, :, c1]
                        B = G[:, r2][:, :, c2]
                        T[i, j, g, h, q] = np.einsum("p,pab,pba->", w, A, B)
    return T


def fermi_column_numpy(system, G, w):
    ia = system.ia()
    nat, nmax = system.n_atoms, max(system.norbs)
    D = np.zeros((nat, nmax, 4), complex)
    for i in range(nat):
        n = system.norbs[i]
        for mu in range(n):
            for a in range(4):
                for s in range(2):
                    for sp in range(2):
                        if SIG[a][s, sp] != 0:
                            D[i, mu, a] += SIG[a][s, sp] * np.sum(
                                w * G[:, ia[i][0] + sp * n + mu, ia[i][0] + s * n + mu])
    return D
