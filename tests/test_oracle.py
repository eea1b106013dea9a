"""The CPU oracle (C restatement over the evaluator's neighbour lists) against
the golden vectors the reference program produced (tests/golden/make_golden.py).
These pin the oracle before it is trusted as the GPU checker."""
import os

import numpy as np
import pytest

from conftest import CASES, GOLDEN, load_case, oracle_for, rel


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_goldens(name):
    case = load_case(name)
    g = case["gold"]
    orc = oracle_for(case)
    for sfx, x in (("", g["coeff"]), ("2", g["coeff2"])):
        r = orc.objective(x, full=True)
        assert rel(r["obj"], float(g["obj" + sfx])) <= 1e-12, (name, sfx, r["obj"], g["obj" + sfx])
        ev = g["errvec" + sfx]
        assert r["errvec"].shape == ev.shape
        scale = np.maximum(np.abs(ev), 1.0)
        assert np.max(np.abs(r["errvec"] - ev) / scale) <= 1e-12
        assert np.max(np.abs(r["forces"].ravel() - g["force" + sfx])) <= 1e-10
        assert np.allclose(r["energy"], g["energy" + sfx], rtol=1e-12, atol=1e-12)
        assert np.allclose(r["stress"].ravel(), g["stress" + sfx], rtol=1e-10, atol=1e-13)
        if sfx == "" and "dens" in g:
            assert np.allclose(r["dens"], g["dens"], rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("name", CASES)
def test_coefficient_layout_matches_reference(name):
    """Potential::coeff(i) order: the reference's dump equals our layout."""
    case = load_case(name)
    assert np.array_equal(case["pot"].coeffs(), case["gold"]["coeff"])


def test_oracle_against_live_reference(tmp_path):
    """Fresh random database, oracle vs the compiled reference (skipped
    where the reference binary was not built)."""
    import oracle
    from meamzilla_b200 import synth
    from meamzilla_b200.potential import Database, PotentialFile
    if not os.path.exists(oracle.MZREF):
        pytest.skip("oracle/_ref/mzref not built")
    pot, cells = synth.make_workload("meam2k", seed=21, ncells=3)
    rng = np.random.default_rng(0)
    for c in cells:
        c.energy0 = rng.normal(-3, 0.1)
        c.force0 = rng.normal(0, 0.3, (c.natoms, 3))
    par = synth.write_case(str(tmp_path), pot, cells)
    ref = oracle.run_reference(par)
    pf = PotentialFile.read(str(tmp_path / "start.pot"))
    db = Database.read(str(tmp_path / "db.conf"), pf)
    orc = oracle.CRestatement(db.view(), [pf.spline(s) for s in range(pf.nsplines)], pf.style, pf.ntypes, 1.0, 1.0)
    r = orc.objective(pf.coeffs(), full=True)
    assert rel(r["obj"], ref["obj"]) <= 1e-12
    assert np.max(np.abs(r["forces"].ravel() - ref["force"])) <= 1e-10
    assert np.array_equal(np.sort(r["dens"]), np.sort(ref["dens"])) or np.allclose(r["dens"], ref["dens"], rtol=1e-14)


@pytest.mark.parametrize("name", CASES)
def test_tangent_oracle_matches_central_differences(name):
    """The tangent-linear restatement (exact directional derivatives) against
    central differences: the reference's own (h = 1e-6, golden `fdgrad`) where
    the case has them, and the oracle's otherwise.  Central differences carry
    O(h^2) truncation and rounding error, about 1e-9 of the largest
    component here, so the bar is 1e-8 of max|g|.  The objective the tangent
    pass returns is the plain restatement's, bit for bit."""
    case = load_case(name)
    g = case["gold"]
    orc = oracle_for(case)
    x = g["coeff"]
    grad = orc.gradient(x)
    obj, _ = orc.tangent(x, np.zeros_like(x))
    assert obj == orc.objective(x)
    if "fdgrad" in g:
        fd = g["fdgrad"]
    else:
        fd = np.zeros_like(x)
        for i in range(x.size):
            h = 1e-6 * max(1.0, abs(x[i]))
            e = np.zeros_like(x)
            e[i] = h
            fd[i] = (orc.objective(x + e) - orc.objective(x - e)) / (2 * h)
    scale = np.max(np.abs(grad))
    assert np.max(np.abs(grad - fd)) <= 1e-8 * scale, (name, np.max(np.abs(grad - fd)) / scale)


def test_tangent_oracle_is_linear_in_the_direction():
    """d/dt F(x + t (a u + b v)) = a dF.u + b dF.v (forward mode is linear in
    the direction), on a two-species MEAM case."""
    case = load_case("meam_sparse")
    orc = oracle_for(case)
    x = case["gold"]["coeff"]
    rng = np.random.default_rng(3)
    u, v = rng.standard_normal(x.size), rng.standard_normal(x.size)
    du, dv = orc.tangent(x, u)[1], orc.tangent(x, v)[1]
    dw = orc.tangent(x, 2.0 * u - 0.5 * v)[1]
    assert abs(dw - (2.0 * du - 0.5 * dv)) <= 1e-12 * (abs(2.0 * du) + abs(0.5 * dv))
