"""Neighbour lists built on the GPU (mz_db_build_device / mz_db_read_device)
against the host builder: every array of the database identical, bit for
bit (pair order, r, unit vectors, knots, shifts, incoming lists), and the
same errors (Config::find_pairs config.cpp:143-234, check_pair
pair_meam_spline.cpp:50-99, Spline::get_knotshift spline.cpp:74-99)."""
import os

import numpy as np
import pytest

from conftest import CASES, GOLDEN, load_case

pytestmark = pytest.mark.gpu


def _same(a, b):
    va, vb = a.view(), b.view()
    assert va.keys() == vb.keys()
    for k in va:
        x, y = va[k], vb[k]
        if isinstance(x, np.ndarray):
            assert x.dtype == y.dtype and x.shape == y.shape, k
            assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), k
        else:
            assert x == y, k


@pytest.mark.parametrize("name", CASES)
def test_device_lists_match_host_on_golden_configs(name):
    from meamzilla_b200.potential import Database
    case = load_case(name)
    conf = os.path.join(case["dir"], case["param"]["config"][0])
    _same(Database.read(conf, case["pot"]), Database.read(conf, case["pot"], device=0))


@pytest.mark.parametrize("workload,ncells", [("meam2k", 60), ("meam500", 40), ("eam54", 20)])
def test_device_lists_match_host_on_synthetic_cells(workload, ncells):
    from meamzilla_b200 import synth
    from meamzilla_b200.potential import Database, PotentialFile
    spec, cells = synth.make_workload(workload, seed=11, ncells=ncells)
    pot = PotentialFile.from_spec(spec)
    a, b = Database.from_cells(cells, pot), Database.from_cells(cells, pot, device=0)
    assert a.stats() == b.stats()
    _same(a, b)


def test_device_lists_report_the_first_short_pair(tmp_path):
    """Two cells with pairs shorter than the first knot: both builders name
    the first one, with the reference's message."""
    from meamzilla_b200._lib import MzError
    from meamzilla_b200.potential import Database
    pot = load_case("eam_bcc3")["pot"]
    cell_ok = "#N 2 1\n#X 8 0 0\n#Y 0 8 0\n#Z 0 0 8\n#F\n0 0 0 0 0 0 0\n0 2.5 0 0 0 0 0\n"
    cell_bad1 = "#N 2 1\n#X 8 0 0\n#Y 0 8 0\n#Z 0 0 8\n#F\n0 0 0 0 0 0 0\n0 1.5 0 0 0 0 0\n"
    cell_bad2 = "#N 3 1\n#X 9 0 0\n#Y 0 9 0\n#Z 0 0 9\n#F\n0 0 0 0 0 0 0\n0 4 0 0 0 0 0\n0 0 1.2 0 0 0 0 0\n"
    p = tmp_path / "c.conf"
    p.write_text(cell_ok + cell_bad1 + cell_bad2)
    msgs = []
    for dev in (None, 0):
        with pytest.raises(MzError) as e:
            Database.read(str(p), pot, device=dev)
        msgs.append((e.value.status, str(e.value)))
    assert msgs[0] == msgs[1]
    assert msgs[0][0] == 4 and "cell=1" in msgs[0][1] and "too short" in msgs[0][1]
