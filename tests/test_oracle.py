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
