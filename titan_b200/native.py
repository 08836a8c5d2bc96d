"""ctypes binding of libtitan_gpu (include/titan_gpu.h).

``GreenGPU`` is the host-side mirror of the reference's Green-function call
surface: ``chi0`` replaces eintshechi(q, e) (eintshechi.F90:2), ``expectation``
replaces expectation_values_greenfunction (mod_expectation.F90:28),
``gg_tensor`` / ``fermi_column`` feed calcJacobian_greenfunction
(mod_self_consistency.F90:795), ``green_batch`` is green() for a batch
(mod_greenfunction.F90:19).  Arrays cross the boundary in Fortran order, as
the C ABI specifies.  There is no CPU fallback: constructing a GreenGPU
without the built library or without a CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtitan_gpu.so")

TG_PREC_FP64 = 0
TG_PREC_SPLIT = 1
# status codes of titan_gpu.h (> 0: 1-based index of a singular (k, z) point)
TG_OK = 0
TG_ERR_ARG = -1
TG_ERR_CUDA = -2
TG_ERR_STATE = -3
TG_ERR_TIMEOUT = -4
TG_ERR_NOMEM = -5
TG_ERR_NUMERIC = -6
_PREC = {"fp64": TG_PREC_FP64, "split": TG_PREC_SPLIT}

_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

SIGNATURES = {
    "tg_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "tg_destroy": (C.c_int, [C.c_void_p]),
    "tg_last_error": (C.c_char_p, [C.c_void_p]),
    "tg_set_system": (C.c_int, [C.c_void_p, C.c_int, _ip, C.c_int, C.c_int, _dp, _ip, _ip, _dp]),
    "tg_set_h0": (C.c_int, [C.c_void_p, C.c_int, _dp]),
    "tg_set_imag_mesh": (C.c_int, [C.c_void_p, C.c_int64, _dp, _dp, _dp]),
    "tg_set_real_mesh": (C.c_int, [C.c_void_p, C.c_int64, _dp, _dp]),
    "tg_chi0": (C.c_int, [C.c_void_p, _dp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _dp, _dp,
                          C.c_int, C.c_int, _dp]),
    "tg_chi0_batch": (C.c_int, [C.c_void_p, _dp, C.c_int, _dp, C.c_double, C.c_double, C.c_double, C.c_int, _dp,
                                _dp, C.c_int, C.c_int, _dp]),
    "tg_expectation": (C.c_int, [C.c_void_p, C.c_double, C.c_double, _dp, _dp, _dp, _dp, _dp]),
    "tg_gg_tensor": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_int, _ip, _dp]),
    "tg_fermi_column": (C.c_int, [C.c_void_p, C.c_double, C.c_double, _dp]),
    "tg_dyson": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp]),
    "tg_set_green_method": (C.c_int, [C.c_void_p, C.c_int]),
    "tg_ldos": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_double, _dp, _dp]),
    "tg_smunu": (C.c_int, [C.c_void_p, C.c_double, C.c_double, _dp]),
    "tg_jij": (C.c_int, [C.c_void_p, _dp, C.c_double, C.c_double, _dp, _dp, _ip, _dp]),
    "tg_chi0_linear_soc": (C.c_int, [C.c_void_p, _dp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _dp,
                                     _dp, _dp, C.c_int, _dp, _dp]),
    "tg_eig_batch": (C.c_int, [C.c_void_p, C.c_int64, _dp, _dp, _dp]),
    "tg_she": (C.c_int, [C.c_void_p, _dp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _dp, _dp, _dp,
                         _dp, C.c_int, _dp]),
    "tg_green_batch": (C.c_int, [C.c_void_p, C.c_int64, _dp, _dp, _dp]),
    "tg_hamiltk_batch": (C.c_int, [C.c_void_p, C.c_int64, _dp, _dp]),
    "tg_last_timing": (C.c_int, [C.c_void_p, _dp]),
    "tg_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "tg_jacobian": (C.c_int, [C.c_void_p, C.c_double, C.c_double, _ip, _dp, _dp, C.c_int, C.c_int, _dp]),
    "tg_jacobian_layout": (C.c_int, [C.c_int, _ip, C.c_int, _ip, _dp, _dp, C.c_int, _ip]),
    "tg_jacobian_assemble": (C.c_int, [C.c_int, _ip, C.c_int, _ip, _dp, _dp, C.c_int, C.c_int, C.c_int, _dp, _dp,
                                       C.c_int, _dp]),
    "tg_adjoint_vb": (C.c_int, [C.c_void_p, C.c_double, C.c_double, _dp]),
    "tg_system_shape": (C.c_int, [C.c_void_p, _ip, _ip, _ip]),
    "tg_expectation_noalloc": (C.c_int, [C.c_void_p, C.c_double, C.c_double, _dp, _dp, _dp, _dp, _dp]),
    "tg_set_chi_orbitals": (C.c_int, [C.c_void_p, _ip]),
    "tg_set_split_chunk": (C.c_int, [C.c_void_p, C.c_int]),
    "tg_gs_orbital": (C.c_int, [C.c_void_p, C.c_double, C.c_double, _dp]),
    "tg_chi0_qbatch": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_int, _dp, C.c_double, C.c_double, C.c_double, C.c_int,
                                 _dp, _dp, C.c_int, C.c_int, _dp]),
    "tg_fp64_peak": (C.c_int, [C.c_void_p, _dp, _dp]),
    "tg_set_autotune": (C.c_int, [C.c_void_p, C.c_int]),
    "tg_tuning": (C.c_int, [C.c_void_p, _ip, _ip]),
    "tg_chi0_error_bound": (C.c_int, [C.c_void_p, C.c_int, _dp]),
    "tg_rcp_check": (C.c_int, [C.c_int64, _dp, _dp]),
    "tg_adjoint_vb_orbitals": (C.c_int, [C.c_void_p, C.c_double, C.c_double, _ip, _dp]),
}


def fp64_peak():
    """(DFMA, DMMA) FP64 TFLOP/s measured on the current device (tg_fp64_peak)."""
    lib = load_library()
    a, b = C.c_double(), C.c_double()
    rc = lib.tg_fp64_peak(None, C.byref(a), C.byref(b))
    if rc != 0:
        raise TitanGPUError(rc, "tg_fp64_peak failed")
    return a.value, b.value


class TitanGPUError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def load_library(path: str = LIB_PATH):
    """Load the shared library and declare every entry point of titan_gpu.h."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is not built (run: python -m titan_b200.build)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _p(a, ctype=C.c_double):
    return a.ctypes.data_as(C.POINTER(ctype))


def jacobian_inputs(system):
    """dmask(norb_max, n_atoms), Un, Um and norb arrays of a system for the Jacobian entry points."""
    nat = system.n_atoms
    nmax = max(system.norbs)
    dmask = np.zeros((nat, nmax), np.int32)
    for i, dl in enumerate(system.dorbs):
        dmask[i, list(dl)] = 1
    return (dmask, np.ascontiguousarray(system.Un(), np.float64), np.ascontiguousarray(system.Um(), np.float64),
            np.ascontiguousarray(system.norbs, np.int32))


def jacobian_layout(system, fixEf=False):
    """(neq, per) of tg_jacobian_layout: unknown count and first unknown of each site."""
    lib = load_library()
    dmask, Un, Um, norb = jacobian_inputs(system)
    per = np.zeros(system.n_atoms + 1, np.int32)
    neq = lib.tg_jacobian_layout(system.n_atoms, _p(norb, C.c_int), dmask.shape[1], _p(dmask, C.c_int), _p(Un),
                                 _p(Um), 1 if fixEf else 0, _p(per, C.c_int))
    if neq < 0:
        raise TitanGPUError(neq, "tg_jacobian_layout: bad arguments")
    return neq, per


def jacobian_assemble(system, T, D, fixEf=False):
    """Host-only tg_jacobian_assemble: T[i, j, g, h, 16] (orbital resolved), D[i, mu, 4]."""
    lib = load_library()
    dmask, Un, Um, norb = jacobian_inputs(system)
    neq, _ = jacobian_layout(system, fixEf)
    T = np.ascontiguousarray(T, np.complex128)
    nrow, ncol = T.shape[2], T.shape[3]
    Dp = _p(np.ascontiguousarray(D, np.complex128).view(np.float64)) if D is not None else None
    J = np.zeros((neq, neq), np.float64, order="F")
    rc = lib.tg_jacobian_assemble(system.n_atoms, _p(norb, C.c_int), dmask.shape[1], _p(dmask, C.c_int), _p(Un),
                                  _p(Um), 1 if fixEf else 0, nrow, ncol, _p(T.view(np.float64)), Dp, neq,
                                  J.ctypes.data_as(_dp))
    if rc != 0:
        raise TitanGPUError(rc, "tg_jacobian_assemble: bad arguments")
    return np.ascontiguousarray(J)


def _fortran_complex(m):
    """numpy [row, col] complex matrix -> Fortran-ordered complex128 buffer."""
    return np.ascontiguousarray(np.asarray(m, dtype=np.complex128).T)


class GreenGPU:
    """One context on one GPU (tg_create / tg_destroy)."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.tg_create(device, C.byref(h))
        if rc != 0:
            raise TitanGPUError(rc, f"tg_create(device={device}) failed (no usable CUDA device?)")
        self.h = h
        self.system = None
        self.dimH = 0
        self.dimens = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.tg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            msg = self.lib.tg_last_error(self.h)
            raise TitanGPUError(rc, msg.decode() if msg else "")
        return rc

    # ---- set-up -----------------------------------------------------------
    def set_system(self, system):
        """Neighbour table of a TBSystem (the calchk data)."""
        cv, bi, ish, t = system.neighbor_table()
        nat = system.n_atoms
        nmax = max(system.norbs)
        norb = np.array(system.norbs, np.int32)
        cvF = np.ascontiguousarray(cv, np.float64)                       # (3, nNeigh) Fortran
        biF = np.ascontiguousarray(bi + 1, np.int32)                     # 1-based
        ishF = np.ascontiguousarray(ish, np.int32)                       # (nAtoms, nNeigh) Fortran
        # t[k, i, b, a] = t0i(b, a, i) of neighbour k -> Fortran t0i(b, a, i, k)
        tF = np.ascontiguousarray(np.transpose(t, (0, 1, 3, 2)), np.complex128)
        rc = self.lib.tg_set_system(self.h, nat, _p(norb, C.c_int), nmax, cv.shape[0], _p(cvF), _p(biF, C.c_int),
                                    _p(ishF, C.c_int), _p(tF.view(np.float64)))
        self._check(rc)
        self.system = system
        self.dimH = system.dimH
        self.dimens = system.dimens
        self.chi_dimens = system.dimens
        self.nmax = nmax

    def set_autotune(self, enable=True):
        self._check(self.lib.tg_set_autotune(self.h, 1 if enable else 0))

    def tuning(self):
        """(K-range splits of the last FP64 call, of the last split-precision call) (tg_tuning)."""
        a, b = C.c_int(), C.c_int()
        self._check(self.lib.tg_tuning(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def error_bound(self, n):
        """Relative normwise bound of the split format for each of the n results of the last
        chi0 call (0 for FP64 results; tg_chi0_error_bound)."""
        out = np.zeros(int(n))
        self._check(self.lib.tg_chi0_error_bound(self.h, int(n), out.ctypes.data_as(_dp)))
        return out

    def set_split_chunk(self, points=0):
        """Points per split-precision chunk (tg_set_split_chunk; 0 = default)."""
        self._check(self.lib.tg_set_split_chunk(self.h, int(points)))

    def set_chi_orbitals(self, sel=None):
        """chi0 over the orbitals sel[i] (local indices) of each site, e.g. the d orbitals
        (system.dorbs); None restores every orbital (tg_set_chi_orbitals)."""
        if sel is None:
            self._check(self.lib.tg_set_chi_orbitals(self.h, None))
            self.chi_dimens = self.dimens
            return
        mask = np.zeros((self.system.n_atoms, self.nmax), np.int32)
        for i, x in enumerate(sel):
            mask[i, list(x)] = 1
        self._check(self.lib.tg_set_chi_orbitals(self.h, _p(mask, C.c_int)))
        self.chi_dimens = 4 * sum(len(x) ** 2 for x in sel)

    def set_h0(self, h0):
        hF = _fortran_complex(h0)
        self._check(self.lib.tg_set_h0(self.h, self.dimH, _p(hF.view(np.float64))))

    def set_imag_mesh(self, ek):
        self.set_imag_mesh_arrays(np.ascontiguousarray(ek.point_energy(), np.float64),
                                  np.ascontiguousarray(ek.kp, np.float64),
                                  np.ascontiguousarray(ek.weight, np.float64))

    def set_imag_mesh_arrays(self, y, kp, w):
        """Flattened (E, k) list from contiguous float64 arrays (may be pinned host memory)."""
        self._check(self.lib.tg_set_imag_mesh(self.h, y.shape[0], _p(y), _p(kp), _p(w)))

    def set_real_mesh(self, kp, w):
        kp = np.ascontiguousarray(kp, np.float64)
        w = np.ascontiguousarray(w, np.float64)
        self._check(self.lib.tg_set_real_mesh(self.h, w.shape[0], _p(kp), _p(w)))

    def setup(self, deck, h0):
        self.set_system(deck.system)
        self.set_h0(h0)
        self.set_imag_mesh(deck.ek)
        self.set_real_mesh(deck.real_kp, deck.real_w)

    # ---- hot path -----------------------------------------------------------
    def chi0(self, q, e, Ef, eta, etap, x2=None, p2=None, precision="fp64"):
        """chiorb_hf(q, e) as a [dimens, dimens] numpy array (eintshechi)."""
        return self.chi0_batch(q, [e], Ef, eta, etap, None if x2 is None else [x2], None if p2 is None else [p2],
                               precision)[0]

    def chi0_batch(self, q, es, Ef, eta, etap, x2s=None, p2s=None, precision="fp64", out=None):
        es = np.ascontiguousarray(es, np.float64)
        nw = es.shape[0]
        nreal = 0
        if x2s is not None:
            nreal = max(len(x) for x in x2s)
        X2 = np.zeros((nw, max(nreal, 1)))
        P2 = np.zeros((nw, max(nreal, 1)))
        if nreal:
            for w in range(nw):
                if len(x2s[w]):
                    X2[w, :len(x2s[w])] = x2s[w]
                    P2[w, :len(p2s[w])] = p2s[w]
        qa = np.ascontiguousarray(q, np.float64)
        D = self.chi_dimens
        buf = out if out is not None else np.empty((nw, D, D), np.complex128)
        rc = self.lib.tg_chi0_batch(self.h, _p(qa), nw, _p(es), Ef, eta, etap, nreal, _p(X2), _p(P2),
                                    _PREC[precision], D, _p(buf.view(np.float64)))
        self._check(rc)
        return np.swapaxes(buf, 1, 2)      # Fortran (row, col) -> numpy [row, col]

    def chi0_qbatch(self, qs, es, Ef, eta, etap, x2s=None, p2s=None, precision="fp64", out=None):
        """chiorb_hf for every (q, e): [n_q, n_omega, dimens, dimens] (tg_chi0_qbatch)."""
        qa = np.ascontiguousarray(np.asarray(qs, np.float64).reshape(-1, 3))
        es = np.ascontiguousarray(es, np.float64)
        nq, nw = qa.shape[0], es.shape[0]
        nreal = max((len(x) for x in x2s), default=0) if x2s is not None else 0
        X2 = np.zeros((nw, max(nreal, 1)))
        P2 = np.zeros((nw, max(nreal, 1)))
        if nreal:
            for w in range(nw):
                X2[w, :len(x2s[w])] = x2s[w]
                P2[w, :len(p2s[w])] = p2s[w]
        D = self.chi_dimens
        buf = out if out is not None else np.empty((nq, nw, D, D), np.complex128)
        rc = self.lib.tg_chi0_qbatch(self.h, nq, _p(qa), nw, _p(es), Ef, eta, etap, nreal, _p(X2), _p(P2),
                                     _PREC[precision], D, _p(buf.view(np.float64)))
        self._check(rc)
        return np.swapaxes(buf, 2, 3)

    def she(self, q, e, Ef, eta, etap, x2, p2, efield, prefactor=None):
        """tchiorbiikl(q, e) as a [dimens, 4] numpy array (eintshe): prefactor . (1/2 pi) sum w df1iikl;
        prefactor None gives the bare integral."""
        qa = np.ascontiguousarray(q, np.float64)
        ue = np.ascontiguousarray(efield, np.float64)
        x2 = np.ascontiguousarray(x2 if x2 is not None else np.zeros(0), np.float64)
        p2 = np.ascontiguousarray(p2 if p2 is not None else np.zeros(0), np.float64)
        D = self.dimens
        pref = None if prefactor is None else _fortran_complex(prefactor)
        out = np.zeros((4, D), np.complex128)      # Fortran (dimens, 4)
        rc = self.lib.tg_she(self.h, _p(qa), e, Ef, eta, etap, x2.shape[0], _p(x2) if x2.shape[0] else None,
                             _p(p2) if p2.shape[0] else None, _p(ue),
                             None if pref is None else _p(pref.view(np.float64)), D, _p(out.view(np.float64)))
        self._check(rc)
        return out.T

    def last_timing(self):
        """Device ms of the last chi0 call (see tg_last_timing)."""
        ms = np.zeros(13)
        self._check(self.lib.tg_last_timing(self.h, _p(ms)))
        return ms

    def profile(self, enable=True):
        self._check(self.lib.tg_profile(self.h, 1 if enable else 0))

    def expectation(self, Ef, eta):
        """rho, mx, my, mz [nAtoms, nOrbMax] and mp (mod_expectation.F90:28-149)."""
        nat = self.system.n_atoms
        out = [np.zeros((nat, self.nmax)) for _ in range(4)]
        mp = np.zeros((nat, self.nmax), np.complex128)
        rc = self.lib.tg_expectation(self.h, Ef, eta, *[_p(o) for o in out], _p(mp.view(np.float64)))
        self._check(rc)
        return out[0], out[1], out[2], out[3], mp

    def expectation_noalloc(self, Ef, eta):
        """expectation() without device allocation during the call (tg_expectation_noalloc)."""
        nat = self.system.n_atoms
        out = [np.zeros((nat, self.nmax)) for _ in range(4)]
        mp = np.zeros((nat, self.nmax), np.complex128)
        rc = self.lib.tg_expectation_noalloc(self.h, Ef, eta, *[_p(o) for o in out], _p(mp.view(np.float64)))
        self._check(rc)
        return out[0], out[1], out[2], out[3], mp

    def gg_tensor(self, Ef, eta, orbital_resolved=True):
        """GG tensor T[i, j, g, h, 16] (see titan_gpu.h)."""
        s = self.system
        nat = s.n_atoms
        dmask = np.zeros((nat, self.nmax), np.int32)
        for i, dl in enumerate(s.dorbs):
            dmask[i, dl] = 1
        if orbital_resolved:
            nrow = max(len(d) for d in s.dorbs) + 1
            ncol = max(len(d) for d in s.dorbs)
        else:
            nrow = ncol = 1
        T = np.zeros((nat, nat, nrow, ncol, 16), np.complex128)
        rc = self.lib.tg_gg_tensor(self.h, Ef, eta, 1 if orbital_resolved else 0, _p(dmask, C.c_int),
                                   _p(T.view(np.float64)))
        self._check(rc)
        return T

    def fermi_column(self, Ef, eta):
        nat = self.system.n_atoms
        D = np.zeros((nat, self.nmax, 4), np.complex128)
        self._check(self.lib.tg_fermi_column(self.h, Ef, eta, _p(D.view(np.float64))))
        return D

    def jacobian(self, Ef, eta, fixEf=False):
        """calcJacobian_greenfunction on the GPU: J[neq, neq] (row = equation, column = unknown)."""
        dmask, Un, Um, _ = jacobian_inputs(self.system)
        neq, _ = jacobian_layout(self.system, fixEf)
        J = np.zeros((neq, neq), np.float64, order="F")
        self._check(self.lib.tg_jacobian(self.h, Ef, eta, _p(dmask, C.c_int), _p(Un), _p(Um), 1 if fixEf else 0, neq,
                                         J.ctypes.data_as(_dp)))
        return np.ascontiguousarray(J)

    def adjoint_vb(self, Ef, eta):
        """A[4 n_atoms, 4 n_atoms] = d(n, mx, my, mz)_i / d(V, Bx, By, Bz)_j (tg_adjoint_vb)."""
        m = 4 * self.system.n_atoms
        A = np.zeros((m, m), np.float64, order="F")
        self._check(self.lib.tg_adjoint_vb(self.h, Ef, eta, A.ctypes.data_as(_dp)))
        return np.ascontiguousarray(A)

    def adjoint_vb_orbitals(self, Ef, eta, sel):
        """adjoint_vb with the fields on, and the observables summed over, the orbitals sel[i]
        of each site (tg_adjoint_vb_orbitals)."""
        m = 4 * self.system.n_atoms
        mask = np.zeros((self.system.n_atoms, self.nmax), np.int32)
        for i, x in enumerate(sel):
            mask[i, list(x)] = 1
        A = np.zeros((m, m), np.float64, order="F")
        self._check(self.lib.tg_adjoint_vb_orbitals(self.h, Ef, eta, _p(mask, C.c_int), A.ctypes.data_as(_dp)))
        return np.ascontiguousarray(A)

    def dyson(self, chi_hf, U):
        n = chi_hf.shape[0]
        a = _fortran_complex(chi_hf)
        u = _fortran_complex(U)
        out = np.empty((n, n), np.complex128)
        self._check(self.lib.tg_dyson(self.h, n, _p(a.view(np.float64)), _p(u.view(np.float64)),
                                      _p(out.view(np.float64))))
        return out.T

    def chi0_linear_soc(self, q, e, Ef, eta, etap, x2, p2, vsoc):
        """(chiorb_hf, chiorb_hflsoc) [dimens, dimens] of eintshechilinearsoc; the context's h0 must exclude
        the SOC blocks vsoc (see TBSystem.linear_soc_split)."""
        qa = np.ascontiguousarray(q, np.float64)
        x2 = np.ascontiguousarray(x2 if x2 is not None else np.zeros(0), np.float64)
        p2 = np.ascontiguousarray(p2 if p2 is not None else np.zeros(0), np.float64)
        V = _fortran_complex(vsoc)
        D = self.dimens
        chi = np.zeros((D, D), np.complex128)
        lsoc = np.zeros((D, D), np.complex128)
        rc = self.lib.tg_chi0_linear_soc(self.h, _p(qa), e, Ef, eta, etap, x2.shape[0], _p(x2) if x2.shape[0] else None,
                                         _p(p2) if p2.shape[0] else None, _p(V.view(np.float64)), D,
                                         _p(chi.view(np.float64)), _p(lsoc.view(np.float64)))
        self._check(rc)
        return chi.T, lsoc.T

    def jij(self, q, Ef, eta, evec, Um):
        """J[i, j, mu, nu] of jij_energy at wave vector q; evec[i] = unit d-moment direction, Um per site."""
        s = self.system
        nat = s.n_atoms
        dmask = np.zeros((nat, self.nmax), np.int32)
        for i, dl in enumerate(s.dorbs):
            dmask[i, dl] = 1
        qa = np.ascontiguousarray(q, np.float64)
        ev = np.ascontiguousarray(evec, np.float64).reshape(nat, 3)
        um = np.ascontiguousarray(Um, np.float64)
        J = np.zeros((3, 3, nat, nat), np.complex128)   # Fortran (i, j, mu, nu) read back as [nu, mu, j, i]
        self._check(self.lib.tg_jij(self.h, _p(qa), Ef, eta, _p(ev), _p(um), _p(dmask, C.c_int), _p(J.view(np.float64))))
        return np.transpose(J, (3, 2, 1, 0))

    def smunu(self, Ef, eta):
        """Smunuiivec as [n_atoms, 3, nOrbMax(mu), nOrbMax(nu)] (calcSmunu, mod_sumrule.F90:162-245)."""
        nat = self.system.n_atoms
        S = np.zeros((nat, 3, self.nmax, self.nmax), np.complex128)   # Fortran (mu, nu, 3, nat) read back
        self._check(self.lib.tg_smunu(self.h, Ef, eta, _p(S.view(np.float64))))
        return np.swapaxes(S, 2, 3)

    def gs_orbital(self, Ef, eta):
        """gupgd[i, a, b] = the reference's gupgd(a, b, i) of calc_GS_L_and_E_greenfunction
        (tg_gs_orbital): (1/pi) sum w (G(i b up, i a up) + G(i b dn, i a dn))."""
        nat = self.system.n_atoms
        P = np.zeros((nat, self.nmax, self.nmax), np.complex128)   # Fortran (a, b, i) read back as [i, b, a]
        self._check(self.lib.tg_gs_orbital(self.h, Ef, eta, _p(P.view(np.float64))))
        return np.swapaxes(P, 1, 2)

    def ldos(self, energies, eta):
        """LDOS up / down [n_e, n_atoms, nOrbMax] on the real-axis BZ (ldos_energy, mod_LDOS.F90:95-150)."""
        e = np.ascontiguousarray(energies, np.float64)
        nat = self.system.n_atoms
        up = np.zeros((e.shape[0], nat, self.nmax))
        dn = np.zeros((e.shape[0], nat, self.nmax))
        self._check(self.lib.tg_ldos(self.h, e.shape[0], _p(e), eta, _p(up), _p(dn)))
        return up, dn

    def set_green_method(self, method):
        """"auto" (default): spectral Green functions for chi0 on tabulated meshes, Gauss-Jordan for the
        disturbance integral; "gauss-jordan": inversion per point everywhere; "spectral": spectral wherever
        the mesh allows (see tg_set_green_method)."""
        self._check(self.lib.tg_set_green_method(self.h, {"auto": 0, "gauss-jordan": 1, "spectral": 2}[method]))

    def eig_batch(self, kp):
        """Eigenvalues [nk, dimH] and eigenvectors [nk, dimH, dimH] (column a = eigenvector a) of H(k)."""
        kp = np.ascontiguousarray(kp, np.float64).reshape(-1, 3)
        nk = kp.shape[0]
        lam = np.zeros((nk, self.dimH))
        U = np.zeros((nk, self.dimH, self.dimH), np.complex128)
        self._check(self.lib.tg_eig_batch(self.h, nk, _p(kp), _p(lam), _p(U.view(np.float64))))
        return lam, U

    def green_batch(self, z, kp):
        z = np.ascontiguousarray(z, np.complex128)
        kp = np.ascontiguousarray(kp, np.float64).reshape(-1, 3)
        nz = z.shape[0]
        G = np.empty((nz, self.dimH, self.dimH), np.complex128)
        self._check(self.lib.tg_green_batch(self.h, nz, _p(z.view(np.float64)), _p(kp), _p(G.view(np.float64))))
        return np.swapaxes(G, 1, 2)

    def hamiltk_batch(self, kp):
        kp = np.ascontiguousarray(kp, np.float64).reshape(-1, 3)
        nk = kp.shape[0]
        H = np.empty((nk, self.dimH, self.dimH), np.complex128)
        self._check(self.lib.tg_hamiltk_batch(self.h, nk, _p(kp), _p(H.view(np.float64))))
        return np.swapaxes(H, 1, 2)
