import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
CASES = sorted(d for d in os.listdir(GOLDEN) if os.path.isfile(os.path.join(GOLDEN, d, "golden.npz")))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_case(name):
    """Golden case: parameter dict, potential, database and the reference's outputs."""
    from meamzilla_b200.potential import Database, PotentialFile, read_param
    d = os.path.join(GOLDEN, name)
    par = read_param(os.path.join(d, "param"))
    pot = PotentialFile.read(os.path.join(d, par["startpot"][0]))
    db = Database.read(os.path.join(d, par["config"][0]), pot)
    gold = dict(np.load(os.path.join(d, "golden.npz")))
    w = dict(energy_weight=float(par.get("energy_weight", ["0"])[0]),
             stress_weight=float(par.get("stress_weight", ["0"])[0]),
             embed_extrap=int(par.get("embed_extrap", ["0"])[0]))
    return dict(dir=d, param=par, pot=pot, db=db, gold=gold, weights=w)


def oracle_for(case):
    import oracle
    pot = case["pot"]
    return oracle.CRestatement(case["db"].view(), [pot.spline(s) for s in range(pot.nsplines)], pot.style, pot.ntypes,
                               **case["weights"])


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


@pytest.fixture(scope="session")
def gpu_available():
    import torch
    return torch.cuda.is_available()
