"""Newton self-consistency on the GPU Green-function path.

The unknowns and equations are those of the reference's dnsqe loop:
  x = (rho of each d orbital when Un != 0, (mxd, myd, mzd) when Um != 0) per
      site, then E_F unless fixEf   (set_hamiltonian_variables,
      source/mod_self_consistency.F90:1754-1780);
  f = out - in for the same quantities, plus sum(rho) - n_total
      (sc_eqs / set_system_of_equations, :1516-1628).
Every Green-function evaluation (expectation values and the Jacobian) runs in
libtitan_gpu (tg_expectation, tg_jacobian); the N-dimensional Newton update
(N <= a few dozen) is solved on the host.  Only the d totals of the moments
enter hee (mod_U_matrix.F90:29-55), so a moment unknown is spread evenly over
the d orbitals of its site when it is written back into a state.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from ..native import jacobian_layout
from .system import MagState


def _nz(u):
    return abs(u) > 1e-8


def unknowns_from_state(system, state, fixEf=False):
    neq, per = jacobian_layout(system, fixEf)
    x = np.zeros(neq)
    _, xd, yd, zd = state.d_totals(system.dorbs)
    Un, Um = system.Un(), system.Um()
    for i in range(system.n_atoms):
        k = per[i]
        dl = sorted(system.dorbs[i])
        if _nz(Un[i]):
            x[k:k + len(dl)] = [state.rho[i, mu] for mu in dl]
            k += len(dl)
        if _nz(Um[i]):
            x[k:k + 3] = [xd[i], yd[i], zd[i]]
    if not fixEf:
        x[neq - 1] = state.Ef
    return x


def state_from_unknowns(system, x, template, fixEf=False):
    neq, per = jacobian_layout(system, fixEf)
    st = MagState(template.rho.copy(), template.mx.copy(), template.my.copy(), template.mz.copy(), template.Ef)
    Un, Um = system.Un(), system.Um()
    for i in range(system.n_atoms):
        k = per[i]
        dl = sorted(system.dorbs[i])
        if _nz(Un[i]):
            for m, mu in enumerate(dl):
                st.rho[i, mu] = x[k + m]
            k += len(dl)
        if _nz(Um[i]):
            for comp, arr in enumerate((st.mx, st.my, st.mz)):
                arr[i, :] = 0.0
                arr[i, dl] = x[k + comp] / len(dl)
    if not fixEf:
        st.Ef = float(x[neq - 1])
    return st


def residual(gpu, system, x, template, fixEf=False):
    """f(x) of sc_eqs with the GPU expectation values; returns (f, output state)."""
    neq, per = jacobian_layout(system, fixEf)
    st_in = state_from_unknowns(system, x, template, fixEf)
    gpu.set_h0(system.h0(st_in))
    rho, mx, my, mz, _ = gpu.expectation(st_in.Ef, system.eta)
    out = MagState(rho, mx, my, mz, st_in.Ef)
    _, xd, yd, zd = out.d_totals(system.dorbs)
    _, xdi, ydi, zdi = st_in.d_totals(system.dorbs)
    Un, Um = system.Un(), system.Um()
    f = np.zeros(neq)
    for i in range(system.n_atoms):
        k = per[i]
        dl = sorted(system.dorbs[i])
        if _nz(Un[i]):
            f[k:k + len(dl)] = [rho[i, mu] - st_in.rho[i, mu] for mu in dl]
            k += len(dl)
        if _nz(Um[i]):
            f[k:k + 3] = [xd[i] - xdi[i], yd[i] - ydi[i], zd[i] - zdi[i]]
    if not fixEf:
        f[neq - 1] = rho.sum() - system.total_occupation()
    return f, out


@dataclass
class NewtonResult:
    x: np.ndarray
    state: MagState
    residual: np.ndarray
    iterations: int
    converged: bool


def newton(gpu, system, state0, fixEf=False, tol=1e-12, maxit=40, max_step=None, ftol=None):
    """Newton iteration x <- x - J(x)^-1 f(x) with the analytic GPU Jacobian.

    The mesh must already be on the context (tg_set_imag_mesh, and
    tg_set_real_mesh for the E_F column).  Converged when the step is below
    tol * max(1, |x|) (the reference's mag_tol = 1e-12, :10), or, when ftol is given,
    when max |f| <= ftol.

    max_step globalises the iteration far from the fixed point, where the reference
    relies on the trust region of SLATEC dnsqe (mod_dnsqe.F90): the Newton step is
    scaled so that no unknown moves by more than max_step, then halved until
    |f| decreases (|f(x + t dx)| <= (1 - 1e-4 t) |f(x)|, t >= 1/1024).  Near the
    fixed point the full step is taken and this is the plain iteration.
    """
    x = unknowns_from_state(system, state0, fixEf)
    converged = False
    it = 0
    f, _ = residual(gpu, system, x, state0, fixEf)   # leaves h0(x) on the context
    for it in range(1, maxit + 1):
        if ftol is not None and np.max(np.abs(f)) <= ftol:
            converged = True
            it -= 1
            break
        Ef = float(x[-1]) if not fixEf else state0.Ef
        J = gpu.jacobian(Ef, system.eta, fixEf)
        dx = np.linalg.solve(J, -f)
        t = 1.0
        if max_step is not None:
            t = min(1.0, max_step / max(np.max(np.abs(dx)), 1e-300))
            n0 = np.linalg.norm(f)
            while True:
                fn, _ = residual(gpu, system, x + t * dx, state0, fixEf)
                if np.linalg.norm(fn) <= (1.0 - 1e-4 * t) * n0 or t < 1.0 / 1024:
                    break
                t *= 0.5
            x = x + t * dx
            f = fn
        else:
            x = x + dx
            f, _ = residual(gpu, system, x, state0, fixEf)
        if np.max(np.abs(t * dx)) <= tol * max(1.0, np.max(np.abs(x))):
            converged = True
            break
    f, out = residual(gpu, system, x, state0, fixEf)
    return NewtonResult(x, out, f, it, converged)
