"""The benchmarked configuration in full: the two-species 2000-cell MEAM
database (405,730 atoms, 17.7 M pair slots, 386 M triplets), FP64 against the
C restatement of the reference objective, objective, ErrorVec and forces;
mixed precision (both the row kernels and the triplet-moment path) against
it at the mixed bars.  Slow: the oracle takes about a quarter of a minute per
coefficient vector."""
import os

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

FP64_OBJ = 1e-12
FP64_FORCE = 1e-10
# ErrorVec entries relative to max(|entry|, 1): an entry is a difference of
# sums over up to ~1e5 terms (cell energies and stresses of 1000-atom cells,
# forces that cancel across a neighbour row), summed in another order here
FP64_ERRVEC = 1e-10
MIX_OBJ = 1e-6
MIX_FORCE = 1e-5


@pytest.fixture(scope="module")
def meam2k():
    from meamzilla_b200 import synth
    from meamzilla_b200.potential import Database, PotentialFile
    spec, cells = synth.make_workload("meam2k", seed=0)
    rng = np.random.default_rng(11)
    for c in cells:
        c.energy0 = rng.normal(-3, 0.1)
        c.force0 = rng.normal(0, 0.3, (c.natoms, 3))
        c.stress0 = rng.normal(0, 1e-3, 6)
    pot = PotentialFile.from_spec(spec)
    db = Database.from_cells(cells, pot)
    x = pot.coeffs()
    X = np.stack([x, synth.perturbed(x, 1, 0.05, seed=12)[0]])
    return pot, db, X


def _evaluator(pot, db, fm):
    from meamzilla_b200.potential import Evaluator
    old = os.environ.get("MZ_FM")
    os.environ["MZ_FM"] = fm
    try:
        return Evaluator(db, pot, 1.0, 1.0, 0, max_candidates=2)
    finally:
        if old is None:
            del os.environ["MZ_FM"]
        else:
            os.environ["MZ_FM"] = old


def test_meam2k_fp64_and_mixed_vs_oracle(meam2k):
    import oracle
    from meamzilla_b200.potential import MZ_FP64, MZ_MIXED
    pot, db, X = meam2k
    assert db.stats()["ntriplets"] > 3e8
    rows = _evaluator(pot, db, "0")
    out = rows.objective(X, MZ_FP64, forces=True, errvec=True)
    mix_rows = rows.objective(X, MZ_MIXED, forces=True)
    del rows
    moments = _evaluator(pot, db, "2")
    mix_fm = moments.objective(X, MZ_MIXED, forces=True)
    assert moments.moment_path(MZ_MIXED, False)
    orc = oracle.CRestatement.for_evaluator(moments)
    del moments
    for c in range(2):
        r = orc.objective(X[c], full=True)
        assert rel(out["obj"][c], r["obj"]) <= FP64_OBJ, (out["obj"][c], r["obj"])
        assert np.max(np.abs(out["forces"][c] - r["forces"])) <= FP64_FORCE
        scale = np.maximum(np.abs(r["errvec"]), 1.0)
        d = np.abs(out["errvec"][c] - r["errvec"]) / scale
        assert np.max(d) <= FP64_ERRVEC, (int(np.argmax(d)), float(np.max(d)))
        for mix in (mix_rows, mix_fm):
            assert rel(mix["obj"][c], r["obj"]) <= MIX_OBJ
            assert np.max(np.abs(mix["forces"][c] - r["forces"])) <= MIX_FORCE
