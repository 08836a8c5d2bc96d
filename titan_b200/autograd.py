"""torch.autograd bridge for the site occupations and moments.

``expectation_vb(V, B, gpu, system, h0, Ef, eta)`` returns x[i] = (n, mx, my,
mz) of every site for h0 + sum_i P_i (V_i sigma_0 + B_i . sigma), computed by
tg_expectation on the GPU.  Its backward pass is the hand-written adjoint
tg_adjoint_vb (one GG-tensor pass at the perturbed h0):
dx_{i,a}/dp_{j,b} = (1/pi) sum_{k,E} w Re Tr[P_i sigma_a G P_j sigma_b G].
PyTorch is the autograd host only; every Green function is computed by the
CUDA library, there is no CPU path.
"""
from __future__ import annotations

import numpy as np
import torch

from .host.vb import site_observables, vb_perturbation


class ExpectationVB(torch.autograd.Function):
    @staticmethod
    def forward(ctx, V, B, gpu, system, h0, Ef, eta):
        Vn = V.detach().cpu().numpy().astype(np.float64)
        Bn = B.detach().cpu().numpy().astype(np.float64).reshape(system.n_atoms, 3)
        hp = np.asarray(h0, complex) + vb_perturbation(system, Vn, Bn)
        gpu.set_h0(hp)
        rho, mx, my, mz, _ = gpu.expectation(Ef, eta)
        x = site_observables(system, rho, mx, my, mz)
        ctx.gpu, ctx.system, ctx.hp, ctx.Ef, ctx.eta = gpu, system, hp, Ef, eta
        ctx.dtype, ctx.device = V.dtype, V.device
        return torch.from_numpy(x).to(dtype=torch.float64, device=V.device)

    @staticmethod
    def backward(ctx, gx):
        gpu, system = ctx.gpu, ctx.system
        gpu.set_h0(ctx.hp)
        A = gpu.adjoint_vb(ctx.Ef, ctx.eta)                      # [4 nat, 4 nat]
        g = A.T @ gx.detach().cpu().numpy().astype(np.float64).reshape(-1)
        g = torch.from_numpy(g.reshape(system.n_atoms, 4)).to(dtype=ctx.dtype, device=ctx.device)
        return g[:, 0].contiguous(), g[:, 1:].contiguous(), None, None, None, None, None


def expectation_vb(V, B, gpu, system, h0, Ef, eta):
    return ExpectationVB.apply(V, B, gpu, system, h0, Ef, eta)
