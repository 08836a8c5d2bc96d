import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def fe_deck():
    """The reference's Fe_bulk_susc example deck with its golden SC state loaded."""
    from titan_b200.host.deck import Deck
    from titan_b200.host.system import read_sc_file
    d = Deck.from_directory(os.path.join(GOLDEN, "Fe_bulk_susc"))
    st = read_sc_file(os.path.join(GOLDEN, "Fe_bulk_susc", "selfconsistency.dat"), d.system.norbs)
    d.system.Ef = st.Ef
    d.state = st
    return d


@pytest.fixture(scope="session")
def fe_chi_golden():
    def rows(name):
        return [[float(x) for x in l.split()] for l in open(os.path.join(GOLDEN, "Fe_bulk_susc", name))
                if not l.strip().startswith("#")]
    return rows("chihf_1_1.dat"), rows("chi_1_1.dat")


def small_system(seed=0, nk=(4, 4, 4), n1gl=8, parts=1):
    """A seeded small bcc 1-atom spd deck (same generator as the benchmark configs)."""
    from titan_b200.host import synthetic
    return synthetic.make_deck("bcc1", seed=seed, nk=nk, n1gl=n1gl, parts=parts)


@pytest.fixture
def rng():
    return np.random.default_rng(1234)
