"""Powell against the reference's own OptPowell (opt_powell.cpp:96-315).

tests/golden/eam_powell4 holds a 14-coefficient EAM fit (targets = the
reference's teacher outputs, a seeded start) and powell.npz: F and the
coefficients after each of the reference's first 8 outer steps (it stops
after 5, the later entries repeat), run by the compiled reference
(tests/golden/make_golden.py --powell).

F = R + c: c is the gauge punishment DUMMY_WEIGHT * U'(rho mid)
(pot_eam_spline.cpp:211-218), constant here because U is fixed, and R the
sum of squared residuals, which Powell drives to 0.  Powell's path is
chaotically sensitive to rounding: Brent's line search stops at a relative
tolerance of 0.1 and the secant updates follow the points it returns, so a
1e-15 relative change of F changes R after one outer step by 2x, and a
1e-14 change can cost the fit an extra outer step or two.  The bars are:
  * every outer step lowers F (both implementations);
  * after the first outer step the reference's R, and this
    implementation's, lie inside the band that the oracle-driven Powell
    reaches from the same start when F is scaled by 1, 1 +- 1e-15 and
    1 +- 1e-14, widened 4x either way (BAND);
  * at the end (the outer loop's own stopping rule, at most 8 steps) both
    have converged: R <= 1e-11 of the starting R, and the coefficients agree
    with the reference's final ones to 3e-5 (max abs) -- the reference ends
    4.9e-7 from the teacher.
"""
import os

import numpy as np
import pytest

from test_optimize_cpu import OracleEvaluator

HERE = os.path.dirname(os.path.abspath(__file__))
CASE = os.path.join(HERE, "golden", "eam_powell4")
SCALES = (1.0, 1.0 + 1e-15, 1.0 - 1e-15, 1.0 + 1e-14, 1.0 - 1e-14)
BAND = 4.0
CONVERGED = 1e-11
DX = 3e-5
STEPS = 8


class Scaled(OracleEvaluator):
    """The oracle with F multiplied by `f` (residuals by sqrt(f))."""

    def __init__(self, orc, ncoeff, f):
        super().__init__(orc, ncoeff)
        self.f = f

    def objective(self, X, precision=0):
        return super().objective(X) * self.f

    def residuals(self, X):
        o, E = super().residuals(X)
        return o * self.f, E * np.sqrt(self.f)


@pytest.fixture(scope="module")
def case():
    import oracle
    from meamzilla_b200.potential import Database, PotentialFile
    g = dict(np.load(os.path.join(CASE, "powell.npz")))
    pot = PotentialFile.read(os.path.join(CASE, "start.pot"))
    db = Database.read(os.path.join(CASE, "db.conf"), pot)
    orc = oracle.CRestatement(db.view(), [pot.spline(s) for s in range(pot.nsplines)], pot.style, pot.ntypes,
                              1.0, 1.0)
    g["c"] = orc.objective(g["x_teacher"])
    return pot, db, orc, g


def _band(orc, P, g):
    """R after the first outer step, over the scaled oracles."""
    from meamzilla_b200.optimize import powell_fit
    R = []
    for f in SCALES:
        ev = Scaled(orc, P, f)
        _, F, _ = powell_fit(ev, g["x0"], max_steps=1, residuals=ev.residuals)
        R.append(F / f - g["c"])
    return min(R) / BAND, max(R) * BAND


def _check(path, g, band):
    """path: [(F, x)] after each outer step of this implementation, run to
    the outer loop's stop."""
    R0 = float(g["obj0"]) - g["c"]
    F = [p[0] for p in path]
    Rref = g["F"] - g["c"]
    assert all(b <= a for a, b in zip([float(g["obj0"])] + F, F))
    assert all(b <= a for a, b in zip(np.r_[g["obj0"], g["F"]], g["F"]))
    lo, hi = band
    assert lo <= Rref[0] <= hi, (Rref[0], band)
    assert lo <= F[0] - g["c"] <= hi, (F[0] - g["c"], band)
    assert Rref[-1] <= CONVERGED * R0 and F[-1] - g["c"] <= CONVERGED * R0, (Rref[-1], F[-1] - g["c"])
    assert np.max(np.abs(path[-1][1] - g["X"][-1])) <= DX


def test_golden_case_is_the_documented_one(case):
    pot, db, orc, g = case
    assert pot.ncoeff == 14 and g["X"].shape == (STEPS, 14)
    # the start's F from the oracle equals the reference's
    assert abs(orc.objective(g["x0"]) - g["obj0"]) <= 1e-12 * g["obj0"]


def test_powell_path_matches_reference_on_cpu(case):
    from meamzilla_b200.optimize import powell_fit
    pot, db, orc, g = case
    band = _band(orc, pot.ncoeff, g)
    ev = OracleEvaluator(orc, pot.ncoeff)
    _, _, info = powell_fit(ev, g["x0"], max_steps=STEPS, residuals=ev.residuals)
    _check(info["outer_history"], g, band)


@pytest.mark.gpu
def test_powell_path_matches_reference_on_gpu(case):
    """The same fit with the GPU evaluator's FP64 residuals and the device
    normal equations (mz_gram_device)."""
    from meamzilla_b200.optimize import powell_fit
    from meamzilla_b200.potential import MZ_FP64, Evaluator
    pot, db, orc, g = case
    band = _band(orc, pot.ncoeff, g)
    ev = Evaluator(db, pot, 1.0, 1.0, 0, max_candidates=pot.ncoeff)
    _, _, info = powell_fit(ev, g["x0"], max_steps=STEPS, precision=MZ_FP64)
    _check(info["outer_history"], g, band)
