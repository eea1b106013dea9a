"""Potential::rescale restated on the host (PotMEAM::rescale
pot_meam.cpp:281-375 with rescale_3body :497-525; PotEAM::rescale
pot_eam.cpp:257-389 with the U'(mid) gauge) against the reference's own
rescale, run on every golden case by the compiled reference (rescale.npz,
tests/golden/make_golden.py).  The densities are the reference's
(pair/spline has none and never rescales, potential.cpp:258-261).  Cubic
splines match bit for bit.  spline5eq re-samples through the second and fourth derivatives
from a 2n x 2n solve, which the reference hands to LAPACK dgesv and the
host solves by its own elimination, so there the values agree to rounding
(1e-13 relative)."""
import os

import numpy as np
import pytest

from conftest import CASES, load_case


def _ref_splines(dump):
    ret, nspl = int(dump[0]), int(dump[1])
    out, o = [], 2
    for _ in range(nspl):
        n = int(dump[o]); o += 1
        x = dump[o:o + n]; o += n
        y = dump[o:o + n]; o += n
        grad = dump[o:o + 2]; o += 2
        nat = dump[o:o + 2].astype(int); o += 2
        step = dump[o]; o += 1
        out.append(dict(n=n, x=x, y=y, grad=grad, nat=tuple(nat), step=step))
    assert o == dump.size
    return ret, out


@pytest.mark.parametrize("flag", [0, 1])
@pytest.mark.parametrize("name", CASES)
def test_rescale_matches_reference(name, flag):
    case = load_case(name)
    pot, db = case["pot"].copy(), case["db"]
    ret, ref = _ref_splines(np.load(os.path.join(case["dir"], "rescale.npz"))["flag%d" % flag])
    dens = case["gold"]["dens"] if "dens" in case["gold"] else np.zeros(db.stats()["natoms"])
    changed, a, b = pot.rescale(db, dens, flag)
    assert int(changed) == ret
    assert pot.nsplines == len(ref)
    for s, r in enumerate(ref):
        sp = pot.spline(s)
        assert sp["nknots"] == r["n"] and sp["nat"] == r["nat"]
        np.testing.assert_array_equal(sp["x"], r["x"])
        g_ours = sp["grad"][[i for i in range(2)]] * (1 - np.array(sp["nat"]))
        g_ref = r["grad"] * (1 - np.array(r["nat"]))
        if sp["quintic"]:
            np.testing.assert_allclose(sp["y"], r["y"], rtol=1e-13, atol=1e-15)
            np.testing.assert_allclose(g_ours, g_ref, rtol=1e-13, atol=1e-15)
        else:
            np.testing.assert_array_equal(sp["y"], r["y"])
            np.testing.assert_array_equal(g_ours, g_ref)
        assert sp["step"] == r["step"]


def test_rescale_never_and_unchanged_potential():
    case = load_case("meam_mix6")
    pot = case["pot"].copy()
    before = [pot.spline(s)["y"].copy() for s in range(pot.nsplines)]
    changed, a, b = pot.rescale(case["db"], case["gold"]["dens"], -1)
    assert not changed and a == 0 and b == 0
    for s in range(pot.nsplines):
        np.testing.assert_array_equal(pot.spline(s)["y"], before[s])
    with pytest.raises(ValueError):
        pot.rescale(case["db"], case["gold"]["dens"][:-1], 1)
