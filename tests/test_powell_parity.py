"""Powell against the reference's own OptPowell (opt_powell.cpp:96-315).

tests/golden/eam_powell4 holds a 14-coefficient EAM fit (targets = the
reference's teacher outputs, a seeded start) and powell.npz: F and the
coefficients after each of the reference's first 4 outer steps, run by the
compiled reference (tests/golden/make_golden.py --powell).

F = R + c: c is the gauge punishment DUMMY_WEIGHT * U'(rho mid)
(pot_eam_spline.cpp:211-218), constant here because U is fixed, and R the
sum of squared residuals, which Powell drives to 0.  Powell's path is
chaotically sensitive to rounding: Brent's line search stops at a relative
tolerance of 0.1 and the secant updates follow the points it returns, so a
1e-15 relative change of F changes R after an outer step by up to 3x.  The
bars are therefore:
  * every outer step lowers F (both implementations);
  * after outer step k the reference's R, and this implementation's, lie
    inside the band of R that the oracle-driven Powell reaches from the same
    start when F is scaled by 1, 1 +- 1e-15 and 1 + 3e-15, widened 4x either
    way (BAND);
  * after 4 outer steps both have converged: R <= 1e-8 of the starting R,
    and the coefficients agree to 1e-4 (max abs), the reference's own
    distance to the teacher after 4 steps being 1.2e-5.
"""
import os

import numpy as np
import pytest

from test_optimize_cpu import OracleEvaluator

HERE = os.path.dirname(os.path.abspath(__file__))
CASE = os.path.join(HERE, "golden", "eam_powell4")
SCALES = (1.0, 1.0 + 1e-15, 1.0 - 1e-15, 1.0 + 3e-15)
BAND = 4.0
CONVERGED = 1e-8
DX = 1e-4


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


def _band(orc, P, g, steps=4):
    from meamzilla_b200.optimize import powell_fit
    R = []
    for f in SCALES:
        ev = Scaled(orc, P, f)
        _, _, info = powell_fit(ev, g["x0"], max_steps=steps, residuals=ev.residuals)
        R.append([F / f - g["c"] for F, _ in info["outer_history"][:steps]])
    return np.array(R)


def _check(path, g, band):
    """path: [(F, x)] after each outer step of this implementation."""
    K = len(g["F"])
    R0 = float(g["obj0"]) - g["c"]
    Rref = g["F"] - g["c"]
    F = [p[0] for p in path]
    assert len(path) >= K
    assert all(b <= a for a, b in zip([float(g["obj0"])] + F, F))
    assert all(b <= a for a, b in zip(np.r_[g["obj0"], g["F"]], g["F"]))
    lo, hi = band.min(axis=0) / BAND, band.max(axis=0) * BAND
    for k in range(K):
        assert lo[k] <= Rref[k] <= hi[k], (k, Rref[k], lo[k], hi[k])
        assert lo[k] <= F[k] - g["c"] <= hi[k], (k, F[k] - g["c"], lo[k], hi[k])
    assert Rref[K - 1] <= CONVERGED * R0 and F[K - 1] - g["c"] <= CONVERGED * R0
    assert np.max(np.abs(path[K - 1][1] - g["X"][K - 1])) <= DX


def test_golden_case_is_the_documented_one(case):
    pot, db, orc, g = case
    assert pot.ncoeff == 14 and g["X"].shape == (4, 14)
    # the start's F from the oracle equals the reference's
    assert abs(orc.objective(g["x0"]) - g["obj0"]) <= 1e-12 * g["obj0"]


def test_powell_path_matches_reference_on_cpu(case):
    from meamzilla_b200.optimize import powell_fit
    pot, db, orc, g = case
    band = _band(orc, pot.ncoeff, g)
    ev = OracleEvaluator(orc, pot.ncoeff)
    _, _, info = powell_fit(ev, g["x0"], max_steps=4, residuals=ev.residuals)
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
    _, _, info = powell_fit(ev, g["x0"], max_steps=4, precision=MZ_FP64)
    _check(info["outer_history"], g, band)
