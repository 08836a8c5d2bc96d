"""Sharding the (E, k) work list over ranks, one GPU per rank.

The chi0 integral is a sum over independent quadrature points, so a rank
integrates its share and one all-reduce adds the dimens x dimens partials: the
reference's split of E_k_imag_mesh over MPI ranks (adaptiveMesh.F90:76-161)
followed by the MPI_Allreduce of eintshechi.F90:176.  Shares:

* imaginary axis, uniform mesh (every energy uses the same k list): each rank
  takes a contiguous k range of every energy, so its share keeps the
  energy-major structure the GPU path tabulates H(k) for;
* imaginary axis, adaptive mesh: a contiguous range of the flattened list,
  balanced by point count;
* real axis: a contiguous range of the real-axis BZ points (all energies).
"""
from __future__ import annotations

import numpy as np

from .mesh import EKMesh


def split_range(n: int, rank: int, world: int):
    """[lo, hi) of rank's contiguous share of n items (sizes differ by at most one)."""
    lo = (n * rank) // world
    hi = (n * (rank + 1)) // world
    return lo, hi


def uniform_blocks(ek: EKMesh):
    """(n_e, nk) when the flattened list is n_e energy blocks over one k list, else None."""
    K = ek.n_points
    if K == 0:
        return None
    e = ek.energy_index
    nk = int(np.argmax(e != e[0])) if np.any(e != e[0]) else K
    if nk == 0 or K % nk:
        return None
    ne = K // nk
    blocks_e = e.reshape(ne, nk)
    if not np.all(blocks_e == blocks_e[:, :1]):
        return None
    kp = ek.kp.reshape(ne, nk, 3)
    if not np.all(kp == kp[:1]):
        return None
    return ne, nk


def shard_imag_mesh(ek: EKMesh, rank: int, world: int) -> EKMesh:
    ub = uniform_blocks(ek)
    if ub is not None:
        ne, nk = ub
        lo, hi = split_range(nk, rank, world)
        sel = (np.arange(ne)[:, None] * nk + np.arange(lo, hi)[None, :]).reshape(-1)
    else:
        lo, hi = split_range(ek.n_points, rank, world)
        sel = np.arange(lo, hi)
    return EKMesh(ek.y, ek.wght, ek.energy_index[sel], ek.kp[sel], ek.weight[sel])


def shard_real_bz(kp, w, rank: int, world: int):
    lo, hi = split_range(len(w), rank, world)
    return kp[lo:hi], w[lo:hi]


def allreduce_sum_complex(a: np.ndarray, group=None) -> np.ndarray:
    """Sum a complex128 array over the process group (NCCL on GPUs, gloo on CPUs)."""
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(np.ascontiguousarray(a, np.complex128).view(np.float64)).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy().view(np.complex128).reshape(a.shape)


def chi0_sharded(gpu, deck, h0, q, e, x2, p2, precision="split", rank=0, world=1, group=None):
    """chi0(q, e) over the whole mesh: this rank's share on its GPU, then one all-reduce."""
    s = deck.system
    gpu.set_system(s)
    gpu.set_h0(h0)
    gpu.set_imag_mesh(shard_imag_mesh(deck.ek, rank, world))
    rk, rw = shard_real_bz(deck.real_kp, deck.real_w, rank, world)
    gpu.set_real_mesh(rk, rw)
    chi = gpu.chi0(np.asarray(q, float), e, s.Ef, s.eta, s.etap, x2, p2, precision)
    return allreduce_sum_complex(chi, group) if world > 1 else chi
