"""Run the oracle's chi0 on shares of a golden deck's mesh in spawned worker
processes and add the shares (test helper, CPU)."""
import os
from concurrent.futures import ProcessPoolExecutor
from multiprocessing import get_context

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    from titan_b200.host.deck import Deck
    from titan_b200.host.system import read_sc_file
    d = Deck.from_directory(os.path.join(GOLDEN, name))
    st = read_sc_file(os.path.join(GOLDEN, name, "selfconsistency.dat"), d.system.norbs)
    d.system.Ef = st.Ef
    return d, st


def _share(args):
    name, rank, world, idx = args
    from oracle import titan_oracle as O
    from titan_b200.host.sharding import shard_imag_mesh, shard_real_bz
    d, st = _load(name)
    s = d.system
    e = float(d.frequencies()[idx])
    x2, p2 = d.real_points(e, s.Ef)
    ek = shard_imag_mesh(d.ek, rank, world)
    rk = shard_real_bz(d.real_kp, d.real_w, rank, world)
    return O.eintshechi(O.Model(s, s.h0(st)), ek, rk, np.zeros(3), e, s.Ef, s.eta, s.etap, x2, p2)


def chi_parallel(name, idx=0, workers=4):
    with ProcessPoolExecutor(workers, mp_context=get_context("spawn")) as ex:
        parts = list(ex.map(_share, [(name, r, workers, idx) for r in range(workers)]))
    return sum(parts)


def _she_share(args):
    name, rank, world, idx = args
    from oracle import titan_oracle as O
    from titan_b200.host.sharding import shard_imag_mesh, shard_real_bz
    d, st = _load(name)
    s = d.system
    e = float(d.frequencies()[idx])
    x2, p2 = d.real_points(e, s.Ef)
    ek = shard_imag_mesh(d.ek, rank, world)
    rk = shard_real_bz(d.real_kp, d.real_w, rank, world)
    return O.eintshe(O.Model(s, s.h0(st)), ek, rk, np.zeros(3), e, s.Ef, s.eta, s.etap, x2, p2, d.params["efield"])


def she_parallel(name, idx=0, workers=4):
    with ProcessPoolExecutor(workers, mp_context=get_context("spawn")) as ex:
        parts = list(ex.map(_she_share, [(name, r, workers, idx) for r in range(workers)]))
    return sum(parts)
