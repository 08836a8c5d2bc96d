"""Energy contours and Brillouin-zone meshes that define the (k, E) batches.

Host-side restatement of the reference's mesh generation.  These routines only
build the inputs of the hot path (k points, weights, complex energies); the
arithmetic follows the reference line by line so that the same points, the
same boundary duplicates and the same weights come out:

* ``gauleg``                 -- source/EnergyIntegration.F90:125-157
* ``imag_energy_points``     -- source/EnergyIntegration.F90:45-97
* ``real_energy_points``     -- source/EnergyIntegration.F90:99-122
* ``bz_fraction`` (3D/2D/1D) -- source/mod_BrillouinZone.F90:151-238, 315-400, 472-540
* ``get_nkpt``               -- source/adaptiveMesh.F90:199-218
* ``adaptive_ek_mesh``       -- source/adaptiveMesh.F90:23-63, 76-161 (one rank)
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

TPI = 2.0 * (4.0 * math.atan(1.0))


def gauleg(x1: float, x2: float, n: int):
    """Gauss-Legendre abscissae/weights on [x1, x2] (EnergyIntegration.F90:125-157).

    Newton iteration on the Legendre recurrence with the reference's start
    guess and stopping rule (eps = 3e-14), so the points agree to the last bit
    wherever the host arithmetic is IEEE double without contraction.
    """
    x = np.zeros(n)
    w = np.zeros(n)
    m = (n + 1) // 2
    xm = 0.5 * (x2 + x1)
    xl = 0.5 * (x2 - x1)
    eps = 3.0e-14
    for i in range(1, m + 1):
        z = math.cos(3.141592654 * (i - 0.25) / (n + 0.5))
        z1 = 0.0
        pp = 0.0
        while abs(z - z1) > eps:
            p1 = 1.0
            p2 = 0.0
            for j in range(1, n + 1):
                p3 = p2
                p2 = p1
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j
            pp = n * (z * p1 - p2) / (z * z - 1.0)
            z1 = z
            z = z1 - p1 / pp
        x[i - 1] = xm - xl * z
        x[n - i] = xm + xl * z
        w[i - 1] = (2.0 * xl) / ((1.0 - z * z) * pp * pp)
        w[n - i] = w[i - 1]
    return x, w


def imag_energy_points(parts: int, n1gl: int):
    """Imaginary-axis points y and weights (EnergyIntegration.F90:45-97).

    ``parts`` log-spaced intervals of x in [0, 1) mapped by y = x/(1-x),
    w = p/(1-x)^2, then sorted ascending in y with the reference's exchange
    sort (stable for equal keys, which never occur).
    """
    pn1 = parts * n1gl
    x1 = np.zeros(pn1)
    p1 = np.zeros(pn1)
    for k in range(parts, 0, -1):
        if parts != 1:
            if k == 1:
                e1, e2 = 10.0 ** (-2), 1.0
            elif k != parts:
                e1, e2 = 10.0 ** (-k - 1), 10.0 ** (-k)
            else:
                e1, e2 = 0.0, 10.0 ** (-k)
        else:
            e1, e2 = 0.0, 1.0
        xs, ws = gauleg(e1, e2, n1gl)
        x1[(k - 1) * n1gl:k * n1gl] = xs
        p1[(k - 1) * n1gl:k * n1gl] = ws
    y = x1 / (1.0 - x1)
    xx = (1.0 - x1) * (1.0 - x1)
    wght = 1.0 * p1 / xx
    y = list(y)
    wght = list(wght)
    for i in range(pn1):
        for j in range(i + 1, pn1):
            if y[i] > y[j]:
                y[i], y[j] = y[j], y[i]
                wght[i], wght[j] = wght[j], wght[i]
    return np.array(y), np.array(wght)


def real_energy_points(Ef: float, e: float, parts3: int, n3gl: int):
    """Real-axis points on [Ef - e, Ef] (EnergyIntegration.F90:99-122).

    Returns empty arrays when |e| < 1e-15, as the reference then skips the
    real-axis integral (eintshechi.F90:38-39).
    """
    if abs(e) < 1.0e-15:
        return np.zeros(0), np.zeros(0)
    x2 = np.zeros(parts3 * n3gl)
    p2 = np.zeros(parts3 * n3gl)
    for k in range(1, parts3 + 1):
        e1 = Ef - ((parts3 - (k - 1)) * e / parts3)
        e2 = Ef - ((parts3 - k) * e / parts3)
        xs, ws = gauleg(e1, e2, n3gl)
        x2[(k - 1) * n3gl:k * n3gl] = xs
        p2[(k - 1) * n3gl:k * n3gl] = ws
    return x2, p2


def _cross(a, b):
    return np.array([a[1] * b[2] - a[2] * b[1],
                     a[2] * b[0] - a[0] * b[2],
                     a[0] * b[1] - a[1] * b[0]])


def _norm(v):
    return math.sqrt(float(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]))


def reciprocal_vectors(a1, a2, a3, sysdim: int):
    """Reciprocal vectors exactly as the fraction generators build them.

    3D: mod_BrillouinZone.F90:177-180; 2D (note b1 = vol*(a1 x zdir)):
    mod_BrillouinZone.F90:335-341; 1D: mod_BrillouinZone.F90:489-491.
    """
    a1 = np.asarray(a1, float)
    a2 = np.asarray(a2, float)
    a3 = np.asarray(a3, float)
    if sysdim == 3:
        vol = TPI / float(np.dot(a1, _cross(a2, a3)))
        return [vol * _cross(a2, a3), vol * _cross(a3, a1), vol * _cross(a1, a2)]
    if sysdim == 2:
        a1xa2 = _cross(a1, a2)
        zdir = a1xa2 / _norm(a1xa2)
        vol = TPI / float(np.dot(zdir, a1xa2))
        return [vol * _cross(a1, zdir), vol * _cross(zdir, a2)]
    zdir = np.array([0.0, 0.0, 1.0])
    ydir = np.array([0.0, 1.0, 0.0])
    vol = TPI / float(np.dot(zdir, _cross(a1, ydir)))
    return [vol * _cross(zdir, ydir)]


def bz_fraction(a1, a2, a3, sysdim: int, nk):
    """All k points of an nk_x x nk_y x nk_z mesh folded to the 1st BZ.

    Vectorised restatement of gen3DFraction/gen2DFraction/gen1DFraction
    (mod_BrillouinZone.F90:151-238, 315-400, 472-540) for a single rank
    (first = 1, last = total): every mesh point equidistant (within 1e-12)
    from several lattice translates is duplicated with weight
    1/(multiplicity * N).  Returns (kp[K,3], w[K]).
    """
    b = reciprocal_vectors(a1, a2, a3, sysdim)
    if sysdim == 3:
        nx, ny, nz = nk
        nkpt = nx * ny * nz
        bz = [np.zeros(3), b[0], b[1], b[0] + b[1], b[2], b[0] + b[2], b[1] + b[2], b[0] + b[1] + b[2]]
        l = np.arange(nkpt, dtype=np.int64)
        ix = (l // (ny * nz)) % nx
        iy = (l // nz) % ny
        iz = l % nz
        kp = (ix[:, None] * b[0][None, :] / nx + iy[:, None] * b[1][None, :] / ny) + iz[:, None] * b[2][None, :] / nz
        largest = b[0] + b[1] + b[2]
    elif sysdim == 2:
        nx, ny = nk[0], nk[1]
        nkpt = nx * ny
        bz = [np.zeros(3), b[0], b[1], b[0] + b[1]]
        l = np.arange(nkpt, dtype=np.int64)
        ix = (l // ny) % nx
        iy = l % ny
        kp = ix[:, None] * b[0][None, :] / nx + iy[:, None] * b[1][None, :] / ny
        largest = b[0] + b[1]
    else:
        nx = nk[0]
        nkpt = nx
        bz = [np.zeros(3), b[0]]
        ix = np.arange(nkpt, dtype=np.int64)
        kp = ix[:, None] * b[0][None, :] / nx
        largest = b[0]
    ini = 10.0 * _norm(largest)
    diffs = np.stack([kp - v[None, :] for v in bz], axis=1)            # [N, nbz, 3]
    dist = np.sqrt(diffs[..., 0] * diffs[..., 0] + diffs[..., 1] * diffs[..., 1] + diffs[..., 2] * diffs[..., 2])
    smallest = np.minimum(dist.min(axis=1), ini)
    sel = np.abs(dist - smallest[:, None]) < 1.0e-12                    # [N, nbz]
    mult = sel.sum(axis=1)
    pts = diffs[sel]                                                     # row-major: point-major, bz order
    w = np.repeat(1.0 / mult.astype(float), mult) / float(nkpt)
    return pts, w


def count_bz(a1, a2, a3, sysdim: int, nkpt_in: int):
    """Number of folded points (with duplicates) for a mesh of ~nkpt_in points.

    count_3D_BZ / count_2D_BZ / count_1D_BZ (mod_BrillouinZone.F90:240-313, 402-470).
    """
    nk = mesh_dims(sysdim, nkpt_in, exact_root=True)
    kp, _ = bz_fraction(a1, a2, a3, sysdim, nk)
    return kp.shape[0], nk


def mesh_dims(sysdim: int, nall: int, exact_root: bool = False):
    """Per-direction mesh size for ~nall points.

    genLocalEKMesh uses nall**0.333333333333333 (adaptiveMesh.F90:120-135);
    count_3D_BZ uses nall**(1/3) (mod_BrillouinZone.F90:271).
    """
    if sysdim == 3:
        p = (1.0 / 3.0) if exact_root else 0.333333333333333
        n = int(math.ceil(float(nall) ** p))
        return (n, n, n)
    if sysdim == 2:
        n = int(math.ceil(math.sqrt(float(nall)) if exact_root else float(nall) ** 0.5))
        return (n, n, 1)
    return (int(math.ceil(float(nall))), 1, 1)


def get_nkpt(e: float, e0: float, nkpt_total: int, sysdim: int, minimum: int) -> int:
    """k count for imaginary energy e (adaptiveMesh.F90:199-218)."""
    expo = math.sqrt(float(sysdim if sysdim in (1, 2, 3) else 1))
    n = int(math.ceil(nkpt_total / ((e / e0) ** expo)))
    return max(n, minimum)


@dataclass
class EKMesh:
    """Flattened (E, k) list of one integral, the reference's E_k_imag_mesh.

    ``energy_index[p]`` indexes the imaginary-axis energy list, ``kp[p]`` and
    ``weight[p]`` = wght(E) * w_k are the point's k vector and full weight.
    """
    y: np.ndarray            # energies (imaginary parts), per energy index
    wght: np.ndarray         # energy weights
    energy_index: np.ndarray  # [K] int64
    kp: np.ndarray           # [K, 3]
    weight: np.ndarray       # [K]

    @property
    def n_points(self) -> int:
        return int(self.kp.shape[0])

    def point_energy(self) -> np.ndarray:
        return self.y[self.energy_index]


def adaptive_ek_mesh(a1, a2, a3, sysdim: int, y, wght, nkpt_total: int, minimum: int,
                     nk_override=None) -> EKMesh:
    """Imaginary-axis (E, k) mesh with per-energy k counts (adaptiveMesh.F90:23-161).

    One rank owns every point, so firstPoint = 1 and lastPoint = total.
    ``nk_override`` replaces get_nkpt by an explicit per-energy k count (used
    for the log-uniform decay of the batching workload).
    """
    idx, kps, ws = [], [], []
    cache = {}
    for i in range(len(y)):
        if nk_override is not None:
            nall = int(nk_override[i])
        else:
            nall = get_nkpt(float(y[i]), float(y[0]), nkpt_total, sysdim, minimum)
        nk = mesh_dims(sysdim, nall)
        if nk not in cache:
            cache[nk] = bz_fraction(a1, a2, a3, sysdim, nk)
        kp, wk = cache[nk]
        idx.append(np.full(kp.shape[0], i, dtype=np.int64))
        kps.append(kp)
        ws.append(wght[i] * wk)
    return EKMesh(np.asarray(y, float), np.asarray(wght, float), np.concatenate(idx),
                  np.concatenate(kps), np.concatenate(ws))
