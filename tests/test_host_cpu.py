"""Host side of the C ABI (no GPU): exports, file formats, parameter layout,
and the errors the reference raises (as status codes)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, load_case, oracle_for, rel


def test_library_exports_every_declared_function():
    from meamzilla_b200._lib import LIB_PATH, lib
    lib()  # builds if needed
    with open(os.path.join(ROOT, "include", "mz_b200.h")) as fh:
        text = fh.read()
    names = sorted(set(re.findall(r"^\s*(?:mz_status|void\s*\*?|const char\s*\*)\s*(mz_\w+)\(", text, re.M)))
    assert len(names) >= 30
    so = C.CDLL(LIB_PATH)
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing


def test_potential_write_read_round_trip(tmp_path):
    from meamzilla_b200.potential import Database, PotentialFile
    case = load_case("meam2_edge")
    pot = case["pot"]
    x = pot.coeffs()
    path = str(tmp_path / "pot.out")
    pot.write(path)
    again = PotentialFile.read(path)
    # Spline3Eq::write_basis_fn prints 15 significant digits (spline3eq.cpp:250-251)
    np.testing.assert_allclose(again.coeffs(), x, rtol=1e-14, atol=1e-300)
    for s in range(pot.nsplines):
        a, b = pot.spline(s), again.spline(s)
        assert a["nknots"] == b["nknots"] and a["nat"] == b["nat"] and a["grad_fixed"] == b["grad_fixed"]
        assert np.array_equal(a["y_fixed"], b["y_fixed"])


def test_coefficient_layout_skips_fixed_values():
    """Fixed knots, natural ends and fixed slopes are not coefficients
    (spline3eq.cpp:77-100, 376-382)."""
    case = load_case("meam2_edge")
    pot = case["pot"]
    n = 0
    for s in range(pot.nsplines):
        sp = pot.spline(s)
        n += int(np.sum(sp["y_fixed"] == 0))
        n += sum(1 for e in range(2) if not sp["grad_fixed"][e] and not sp["nat"][e])
    assert n == pot.ncoeff == case["gold"]["coeff"].size


def test_set_coeffs_changes_only_free_values():
    case = load_case("meam2_edge")
    pot = case["pot"]
    before = [pot.spline(s) for s in range(pot.nsplines)]
    x = pot.coeffs()
    pot.set_coeffs(x + 1.0)
    after = [pot.spline(s) for s in range(pot.nsplines)]
    for a, b in zip(before, after):
        fixed = a["y_fixed"] == 1
        assert np.array_equal(a["y"][fixed], b["y"][fixed])
        assert np.allclose(b["y"][~fixed], a["y"][~fixed] + 1.0)
    pot.set_coeffs(x)


def test_spline_eval_matches_reference_formula():
    """Value and slope inside and (linear) outside the knots (spline3eq.h:204-236)."""
    case = load_case("eam_bcc3")
    pot = case["pot"]
    s = 2  # U
    sp = pot.spline(s)
    lo, hi = sp["left"], sp["right"]
    v_lo, g_lo = pot.spline_eval(s, lo)
    v_out, g_out = pot.spline_eval(s, lo - 0.3)
    assert g_out == sp["grad"][0]
    assert abs(v_out - (sp["y"][0] + sp["grad"][0] * (-0.3))) < 1e-15
    assert abs(v_lo - sp["y"][0]) < 1e-14
    v_hi, _ = pot.spline_eval(s, hi)
    assert abs(v_hi - sp["y"][-1]) < 1e-14


# ------------------------------------------------------------------ errors

def _status(fn, *args):
    from meamzilla_b200._lib import MzError
    with pytest.raises(MzError) as e:
        fn(*args)
    return e.value.status, str(e.value)


def test_missing_files_are_io_errors(tmp_path):
    from meamzilla_b200.potential import Database, PotentialFile
    st, msg = _status(PotentialFile.read, str(tmp_path / "nope"))
    assert st == 2 and "cannot open" in msg
    pot = load_case("eam_bcc3")["pot"]
    st, _ = _status(Database.read, str(tmp_path / "nope.conf"), pot)
    assert st == 2


@pytest.mark.parametrize("text,status,phrase", [
    ("comment\n#X eam/spline 1\n", 3, "#T"),
    ("comment\n#T eam/spline 1\n#B spline3eq\n", 3, "#P"),
    ("comment\n#T meam 1\n#P\n", 5, "not implemented"),
    ("comment\n#T eam/spline 1\n#P\n#B spline7eq\n1 2 3\n", 5, "spline7eq"),
    # bases may mix (one per function): a truncated spline5eq block after a spline3eq one
    ("comment\n#T eam/spline 1\n#P\n#B spline3eq\n1.8 5.0 3\n0 0\n1 1\n0 1\n0 1\n0 1\n#B spline5eq\n1 2 3\n", 3,
     "unexpected end"),
    ("comment\n#T eam/spline 1\n#P\n#B spline3eq\n1.8 5.0 10\n0 7\n1 1\n0 1\n", 3, "constraint"),
    ("comment\n#T eam/spline 1\n#P\n#B spline3eq\n1.8 5.0 4\n0 0\n1 1\n0 1\n0 x\n", 3, "knot line"),
])
def test_malformed_potential_files(text, status, phrase):
    from meamzilla_b200.potential import PotentialFile
    st, msg = _status(PotentialFile.parse, text)
    assert st == status and phrase in msg


def _conf(tmp_path, body):
    p = tmp_path / "c.conf"
    p.write_text(body)
    return str(p)


def test_malformed_config_files(tmp_path):
    from meamzilla_b200.potential import Database
    pot = load_case("eam_bcc3")["pot"]
    cases = [
        ("#X 3 0 0\n#F\n0 0 0 0 0 0 0\n", "(#N ...) is missing"),
        ("#N 2 1\n#X 6 0 0\n#Y 0 6 0\n#Z 0 0 6\n#F\n0 0 0 0 0 0 0\n0 3 0 0 0 0 0\n0 0 3 0 0 0 0\n", "too many atoms"),
        ("#N 1 1\n#X 6 0 0\n#Y 0 6 0\n#Z 0 0 6\n#F\n3 0 0 0 0 0 0\n", "incorrect atom type"),
        ("#N 1 1\n#X 6 0 0\n#Y 0 6 0\n#Z 0 0 6\n#E abc\n#F\n0 0 0 0 0 0 0\n", "energy (#E ...) incorrect"),
    ]
    for body, phrase in cases:
        st, msg = _status(Database.read, _conf(tmp_path, body), pot)
        assert st == 3 and phrase in msg, (phrase, msg)


def test_pair_shorter_than_first_knot_is_range_error(tmp_path):
    """check_pair throws for r below a spline's first knot (pair_eam_spline.cpp:61-65)."""
    from meamzilla_b200.potential import Database
    pot = load_case("eam_bcc3")["pot"]
    body = "#N 2 1\n#X 8 0 0\n#Y 0 8 0\n#Z 0 0 8\n#F\n0 0 0 0 0 0 0\n0 1.5 0 0 0 0 0\n"
    st, msg = _status(Database.read, _conf(tmp_path, body), pot)
    assert st == 4 and "too short" in msg


def test_pair_spline_lists_hold_each_pair_once():
    """pair/spline lists every pair once (dbl_cnt_pair_ = 0, config.cpp:181-185):
    for atom i of a cell the neighbours j >= i, the atom's own images
    included; the double-counted list of the same cells holds every other
    pair twice.  A database built for one kind of list is refused by an
    evaluator of the other kind."""
    from meamzilla_b200 import synth
    from meamzilla_b200._lib import MzError
    from meamzilla_b200.potential import Database, Evaluator, PotentialFile
    case = load_case("pair_bcc1")
    half = case["db"].view()
    eam = PotentialFile.from_spec(synth.teacher_potential("eam/spline", 1, 5.0, seed=1))
    full = Database.read(os.path.join(case["dir"], "db.conf"), eam).view()
    a0 = half["cell_atom0"]

    def pairs(v):
        out = []
        for i in range(v["natoms"]):
            for s in range(v["pair_off"][i], v["pair_off"][i + 1]):
                out.append((i, int(v["pair_nbr"][s]), round(float(v["pair_r"][s]), 9)))
        return out

    h, f = pairs(half), pairs(full)
    assert all(j >= i for i, j, _ in h)
    self_h = sorted(p for p in h if p[0] == p[1])
    other_h = sorted(p for p in h if p[0] != p[1])
    assert self_h == sorted(p for p in f if p[0] == p[1])
    assert len(f) == len(self_h) + 2 * len(other_h)
    assert a0[-1] == half["natoms"]
    with pytest.raises(MzError) as e:
        Evaluator(case["db"], eam)
    assert "another potential style" in str(e.value)


def test_read_param_first_key_wins(tmp_path):
    from meamzilla_b200.potential import read_param
    p = tmp_path / "param"
    p.write_text("config a.conf\n\n  \nenergy_weight 2\nenergy_weight 5\r\nstartpot s.pot\n")
    d = read_param(str(p))
    assert d["config"] == ["a.conf"] and d["energy_weight"] == ["2"] and d["startpot"] == ["s.pot"]


def test_modify_coeff_gaussian_bump():
    """Potential.modify_coeff restates Spline::modify_coeff (spline.cpp:120-149)."""
    from meamzilla_b200.potential import Potential

    class FakeEv:
        def __init__(self, pot):
            self.pot = pot

    case = load_case("eam_bcc3")
    pot = case["pot"]
    p = Potential.__new__(Potential)
    p.ev = FakeEv(pot)
    p.x = pot.coeffs().copy()
    x0 = p.x.copy()
    p.modify_coeff(3, 0.5, 1.0)  # knot 3 of phi
    d = p.x - x0
    for i in range(-3, 5):  # knots 0..7 of phi; knot -1 does not exist
        assert abs(d[3 + i] - 0.3989422804014326779 * np.exp(-i * i * 0.5) * 0.5) < 1e-15
    assert np.all(d[8:] == 0)
    p.x = x0.copy()
    p.modify_coeff(10, 0.25, 1.0)  # phi's left end slope
    assert p.x[10] == x0[10] + 0.25 and np.count_nonzero(p.x - x0) == 1
