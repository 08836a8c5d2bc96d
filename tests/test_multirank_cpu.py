"""Multi-rank logic on CPU: gloo, world size 2 (no GPU).

* the mesh shares cover every point exactly once and keep the weights;
* the sharded integral plus the all-reduce equals the single-rank integral
  (the oracle integrates each share);
* the bench's max/sum reductions work on a gloo group.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import titan_oracle as O
        from titan_b200.host import synthetic
        from titan_b200.host.sharding import allreduce_sum_complex, shard_imag_mesh, shard_real_bz
        from titan_b200.host.system import initial_state
        import bench
        deck = synthetic.make_deck("bcc1", nk=(3, 3, 3), n1gl=4, parts=1, n3gl=4)
        s = deck.system
        h0 = s.h0(initial_state(s))
        e = 0.05
        x2, p2 = deck.real_points(e, s.Ef)
        ek = shard_imag_mesh(deck.ek, rank, world)
        rk, rw = shard_real_bz(deck.real_kp, deck.real_w, rank, world)
        local = O.eintshechi(O.Model(s, h0), ek, (rk, rw), np.zeros(3), e, s.Ef, s.eta, s.etap, x2, p2)
        total = allreduce_sum_complex(local)
        mx = bench.allreduce_max(float(rank + 1), world)
        sm = bench.allreduce_sum(float(rank + 1), world)
        bench.barrier(world)
        if rank == 0:
            ref = O.eintshechi(O.Model(s, h0), deck.ek, (deck.real_kp, deck.real_w), np.zeros(3), e, s.Ef, s.eta,
                               s.etap, x2, p2)
            np.save(out, np.array([np.linalg.norm(total - ref) / np.linalg.norm(ref), mx, sm]))
    finally:
        dist.destroy_process_group()


def test_shards_cover_the_mesh():
    from titan_b200.host import synthetic
    from titan_b200.host.sharding import shard_imag_mesh, shard_real_bz, uniform_blocks
    deck = synthetic.make_deck("sq2", nk=(5, 5, 1), n1gl=4, parts=1, n3gl=4)
    ek = deck.ek
    assert uniform_blocks(ek) is not None
    for world in (1, 2, 3):
        parts = [shard_imag_mesh(ek, r, world) for r in range(world)]
        assert sum(p.n_points for p in parts) == ek.n_points
        assert np.isclose(sum(p.weight.sum() for p in parts), ek.weight.sum(), rtol=1e-13, atol=0)
        assert all(uniform_blocks(p) is not None for p in parts if p.n_points)
        rk = [shard_real_bz(deck.real_kp, deck.real_w, r, world) for r in range(world)]
        assert sum(len(w) for _, w in rk) == len(deck.real_w)


def test_sharded_chi0_allreduce_gloo(tmp_path):
    world = 2
    out = str(tmp_path / "res.npy")
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    rel, mx, sm = np.load(out)
    assert rel < 1e-13
    assert mx == 2.0 and sm == 3.0
