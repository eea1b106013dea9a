"""The no-allocation objective entry point (mz_objective_noalloc).

It serves callers that cannot call cudaMalloc (code inside another
framework's allocator, or under a fixed device-memory budget): it stages the
database and all scratch in one file-scope device array instead of the
context's buffers.  Its results must equal the ordinary entry point's
(mz_objective through an Evaluator) to the FP64 parity tolerances, on two
calls in a row (the second call reuses the array the first one filled).

This file sorts last so that a run stopping at the first failure has already
run every other test; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from conftest import load_case, rel

pytestmark = pytest.mark.gpu

FP64_OBJ = 1e-12
FP64_FORCE = 1e-10


def _noalloc(case, x):
    from meamzilla_b200 import _lib
    from meamzilla_b200._lib import check, lib, ptr
    w = case["weights"]
    s = _lib.Settings(w["energy_weight"], w["stress_weight"], w["embed_extrap"], 0, 1, 0)
    n = case["db"].stats()["natoms"]
    obj = np.zeros(1)
    forces = np.zeros((n, 3))
    x = np.ascontiguousarray(x, dtype=np.float64)
    check(lib().mz_objective_noalloc(case["db"].handle, case["pot"].handle, C.byref(s), ptr(x), ptr(obj),
                                     ptr(forces)))
    return obj[0], forces


@pytest.mark.parametrize("name", ["meam_mix6", "meam2_edge", "eam_bcc3", "pair_bcc1"])
def test_noalloc_matches_objective_two_calls(name):
    from meamzilla_b200.potential import MZ_FP64, Evaluator
    case = load_case(name)
    g = case["gold"]
    ev = Evaluator(case["db"], case["pot"], max_candidates=1, **case["weights"])
    for x in (g["coeff"], g["coeff2"]):  # two calls in a row
        ref = ev.objective(x[None, :], MZ_FP64, forces=True)
        obj, forces = _noalloc(case, x)
        assert rel(obj, ref["obj"][0]) <= FP64_OBJ
        assert np.max(np.abs(forces - ref["forces"][0])) <= FP64_FORCE


def test_noalloc_allocates_no_device_memory():
    """After a first call (which loads the kernels and looks up the array's
    address), further calls leave the device's free memory unchanged."""
    import torch
    case = load_case("meam_mix6")
    g = case["gold"]
    _noalloc(case, g["coeff"])
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for x in (g["coeff"], g["coeff2"], g["coeff"]):
        _noalloc(case, x)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0


def test_noalloc_rejects_bad_device_ordinal():
    from meamzilla_b200 import _lib
    from meamzilla_b200._lib import MzError, lib, ptr
    case = load_case("eam_bcc3")
    w = case["weights"]
    for dev in (-1, 1 << 20):
        s = _lib.Settings(w["energy_weight"], w["stress_weight"], w["embed_extrap"], dev, 1, 0)
        x = np.ascontiguousarray(case["gold"]["coeff"])
        obj = np.zeros(1)
        with pytest.raises(MzError) as e:
            _lib.check(lib().mz_objective_noalloc(case["db"].handle, case["pot"].handle, C.byref(s), ptr(x),
                                                  ptr(obj), None))
        assert "MZ_ERR_ARG" in str(e.value) and "ordinal" in str(e.value)


def test_noalloc_rejects_database_beyond_its_array():
    from meamzilla_b200 import synth
    from meamzilla_b200._lib import MzError
    from meamzilla_b200.potential import Database, PotentialFile
    spec, cells = synth.make_workload("meam2k", seed=4, ncells=200)
    pot = PotentialFile.from_spec(spec)
    db = Database.from_cells(cells, pot)
    case = dict(db=db, pot=pot, weights=dict(energy_weight=1.0, stress_weight=1.0, embed_extrap=0))
    with pytest.raises(MzError) as e:
        _noalloc(case, pot.coeffs())
    assert "MZ_ERR_RANGE" in str(e.value) and "bytes of scratch" in str(e.value)
