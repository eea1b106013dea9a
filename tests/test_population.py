"""Batched population evaluation on the 500-cell single-species MEAM
workload (atom counts log-uniform in [16, 512]): 256 coefficient vectors
(teacher + N(0, 0.05), the GA population and annealing chains of
opt_genalg.cpp:143-150 / opt_simann.cpp:120-135) in one call, in FP64 and in
mixed precision, each candidate's objective checked: FP64 against the oracle
(a sample of candidates, 1e-12 relative), mixed against FP64 (1e-6)."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

NCAND = 256


def test_population_of_256_on_500_cells():
    import oracle
    from meamzilla_b200 import synth
    from meamzilla_b200.potential import MZ_FP64, MZ_MIXED, Database, Evaluator, PotentialFile
    spec, cells = synth.make_workload("meam500", seed=0)
    pot = PotentialFile.from_spec(spec)
    db = Database.from_cells(cells, pot, device=0)
    t = Evaluator(db, pot, 1.0, 1.0, 0, max_candidates=1).objective(pot.coeffs()[None, :], MZ_FP64, forces=True,
                                                                      energy=True, stress=True)
    synth.set_teacher_targets(cells, t["energy"][0], t["stress"][0], t["forces"][0], seed=4100)
    db = Database.from_cells(cells, pot, device=0)
    ev = Evaluator(db, pot, 1.0, 1.0, 0, max_candidates=NCAND)
    X = synth.perturbed(pot.coeffs(), NCAND, 0.05, seed=4200)
    o64 = ev.objective(X, MZ_FP64)
    om = ev.objective(X, MZ_MIXED)
    assert np.all(np.isfinite(o64)) and np.all(o64 > 0)
    err = np.abs(om - o64) / np.abs(o64)
    assert err.max() <= 1e-6, err.max()
    # a second call replays the captured launch sequence: identical results
    assert np.array_equal(ev.objective(X, MZ_MIXED), om)
    orc = oracle.CRestatement(db.view(), [pot.spline(s) for s in range(pot.nsplines)], pot.style, pot.ntypes,
                              1.0, 1.0)
    for c in (0, 101, 255):
        assert rel(o64[c], orc.objective(X[c])) <= 1e-12, c
