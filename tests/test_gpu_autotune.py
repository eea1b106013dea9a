"""The launch autotuner (mz_tuning): the first objective call of a precision,
with and without the gradient, times the forward and the adjoint at three
atom-block sizes (and the adjoint at two persistent-grid sizes) and keeps the
fastest.  Every variant must give the same objective, forces and residual
vector, bit for bit, and the same gradient to rounding; MZ_TUNE=0 keeps the
first variant."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _workload():
    from meamzilla_b200 import synth
    from meamzilla_b200.potential import Database, PotentialFile
    spec, cells = synth.make_workload("meam2k", seed=21, ncells=40)
    rng = np.random.default_rng(5)
    for c in cells:
        c.energy0 = float(rng.normal(-3.0, 0.1))
        c.force0 = rng.normal(0.0, 0.3, (c.natoms, 3))
        c.stress0 = rng.normal(0.0, 1e-3, 6)
    pot = PotentialFile.from_spec(synth.in_range_variant(spec))
    return pot, Database.from_cells(cells, pot)


def test_tuned_and_untuned_variants_agree(monkeypatch):
    from meamzilla_b200 import synth
    from meamzilla_b200.potential import MZ_FP64, MZ_MIXED, Evaluator
    pot, db = _workload()
    X = synth.perturbed(pot.coeffs(), 4, 0.01, seed=6)
    monkeypatch.setenv("MZ_TUNE", "0")
    fixed = Evaluator(db, pot, 1.0, 1.0, 0, max_candidates=4)
    monkeypatch.delenv("MZ_TUNE")
    tuned = Evaluator(db, pot, 1.0, 1.0, 0, max_candidates=4)
    for prec, gtol in ((MZ_FP64, 1e-11), (MZ_MIXED, 1e-5)):
        a = fixed.objective(X, prec, errvec=True, forces=True)
        b = tuned.objective(X, prec, errvec=True, forces=True)
        for k in ("obj", "errvec", "forces"):
            assert np.array_equal(a[k], b[k]), (prec, k)
        oa, ga = fixed.objective_grad(X, prec)
        ob, gb = tuned.objective_grad(X, prec)
        assert np.array_equal(oa, ob)
        assert np.max(np.abs(ga - gb)) <= gtol * np.max(np.abs(ga)), prec
        t0, t1 = fixed.tuning(prec, True), tuned.tuning(prec, True)
        assert t0["forward_block_slots"] == 256 and t0["adjoint_block_slots"] == 256
        assert t1["forward_block_slots"] in (256, 192, 128) and t1["adjoint_block_slots"] in (256, 192, 128)
        assert t1["adjoint_ctas"] >= 1
    # the tuned choice is fixed for the context: a repeat is bit-identical
    oc, gc = tuned.objective_grad(X, MZ_MIXED)
    assert np.array_equal(gc, gb)
