"""The reference's data files (Potential::write_data, potential.cpp:325-342:
.rho .energy .stress .force .error .punish) written from the reference's
own evaluated arrays (golden.npz) must equal, byte for byte, the files the
compiled reference wrote for the same potential (ref.* in each case).
pair/spline writes neither .rho nor .punish (potential.cpp:713-725)."""
import os

import numpy as np
import pytest

from conftest import CASES, load_case

EXTS = ("rho", "energy", "stress", "force", "error", "punish")


@pytest.mark.parametrize("name", CASES)
def test_data_files_match_reference_bytes(name, tmp_path):
    from meamzilla_b200.potential import write_data_arrays
    case = load_case(name)
    g = case["gold"]
    w = case["weights"]
    prefix = str(tmp_path / "out")
    write_data_arrays(case["db"], case["pot"], w["energy_weight"], w["stress_weight"], g["errvec"], g["energy"],
                      g["stress"], g["force"], g.get("dens"), prefix)
    for ext in EXTS:
        ref = os.path.join(case["dir"], "ref." + ext)
        assert os.path.exists(prefix + "." + ext) == os.path.exists(ref), ext
        if not os.path.exists(ref):
            continue
        with open(prefix + "." + ext) as a, open(ref) as b:
            assert a.read() == b.read(), ext


def test_data_file_numbering(tmp_path):
    from meamzilla_b200.potential import write_data_arrays
    case = load_case("eam_bcc3")
    g = case["gold"]
    write_data_arrays(case["db"], case["pot"], 1.0, 1.0, g["errvec"], g["energy"], g["stress"], g["force"], g["dens"],
                      str(tmp_path / "out"), 3)
    assert all(os.path.exists(str(tmp_path / ("out.%s.3" % e))) for e in EXTS)
