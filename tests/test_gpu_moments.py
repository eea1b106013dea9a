"""The triplet-moment path of mixed-precision meam/spline (mz_fm.cuh) against
the FP64 path, the oracle and the row kernels' mixed path.

The path rewrites the candidates' triplet sums as contractions of per-slot
moments in the B-spline bases of f and g (an exact re-parametrisation), so
its results carry only the mixed path's FP32 rounding: objective within 1e-6
relative and forces within 1e-5 eV/A of FP64, gradient within 1e-4 of its
largest component, the bars of the row kernels' mixed path.  MZ_FM=2 in the
environment at construction forces the path on, MZ_FM=0 off."""
import os

import numpy as np
import pytest

from conftest import load_case, oracle_for

pytestmark = pytest.mark.gpu

OBJ = 1e-6
FORCE = 1e-5
GRAD = 1e-4

MEAM_CASES = ["meam_mix6", "meam2_edge", "meam_sparse", "meam_inrange_w"]


def _evaluator(case, ncand, fm="2"):
    from meamzilla_b200.potential import Evaluator
    old = os.environ.get("MZ_FM")
    os.environ["MZ_FM"] = fm
    try:
        return Evaluator(case["db"], case["pot"], max_candidates=ncand, **case["weights"])
    finally:
        if old is None:
            del os.environ["MZ_FM"]
        else:
            os.environ["MZ_FM"] = old


def _err(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", MEAM_CASES)
def test_moment_path_objective_forces_gradient(name):
    from meamzilla_b200.potential import MZ_FP64, MZ_MIXED
    case = load_case(name)
    g = case["gold"]
    x = np.stack([g["coeff"], g["coeff2"]])
    ev = _evaluator(case, 2)
    o32, g32 = ev.objective_grad(x, MZ_MIXED)
    assert ev.moment_path(MZ_MIXED, True)
    o64, g64 = ev.objective_grad(x, MZ_FP64)
    assert np.all(np.abs(o32 - o64) <= OBJ * np.abs(o64)), (o32, o64)
    for c in range(2):
        assert _err(g32[c], g64[c]) <= GRAD, (name, c, _err(g32[c], g64[c]))
    f32 = ev.objective(x, MZ_MIXED, forces=True, errvec=True, energy=True, stress=True)
    f64 = ev.objective(x, MZ_FP64, forces=True, errvec=True, energy=True, stress=True)
    assert ev.moment_path(MZ_MIXED, False)
    assert np.max(np.abs(f32["forces"] - f64["forces"])) <= FORCE
    assert np.array_equal(f32["obj"], o32)
    orc = oracle_for(case)
    for c in range(2):
        assert abs(o32[c] - orc.objective(x[c])) <= OBJ * abs(o64[c])
    np.testing.assert_allclose(f32["energy"], f64["energy"], rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(f32["stress"], f64["stress"], rtol=1e-5, atol=1e-7)
    scale = np.maximum(np.abs(f64["errvec"]), 1.0)
    assert np.max(np.abs(f32["errvec"] - f64["errvec"]) / scale) <= 1e-5


def test_moment_path_many_candidates_in_groups():
    """More than 64 candidates run as several candidate groups."""
    from meamzilla_b200.potential import MZ_FP64, MZ_MIXED
    case = load_case("meam2_edge")
    rng = np.random.default_rng(5)
    x0 = case["gold"]["coeff"]
    x = x0[None, :] + rng.normal(0.0, 0.01, (70, x0.size))
    ev = _evaluator(case, 70)
    o32, g32 = ev.objective_grad(x, MZ_MIXED)
    o64, g64 = ev.objective_grad(x, MZ_FP64)
    assert np.all(np.abs(o32 - o64) <= OBJ * np.abs(o64))
    for c in (0, 31, 64, 69):
        assert _err(g32[c], g64[c]) <= GRAD


def test_moment_path_matches_row_kernels_mixed():
    """The moment path and the row kernels' mixed path agree to their FP32
    rounding on a 60-cell two-species workload of the benchmark's rules."""
    from meamzilla_b200 import synth
    from meamzilla_b200.potential import MZ_FP64, MZ_MIXED, Database, PotentialFile
    spec, cells = synth.make_workload("meam2k", seed=3, ncells=60)
    pot = PotentialFile.from_spec(spec)
    db = Database.from_cells(cells, pot)
    case = dict(db=db, pot=pot, weights=dict(energy_weight=1.0, stress_weight=1.0, embed_extrap=0))
    x = synth.perturbed(pot.coeffs(), 8, 0.05, seed=9)
    a = _evaluator(case, 8, "2")
    b = _evaluator(case, 8, "0")
    oa, ga = a.objective_grad(x, MZ_MIXED)
    ob, gb = b.objective_grad(x, MZ_MIXED)
    o64, g64 = b.objective_grad(x, MZ_FP64)
    assert a.moment_path(MZ_MIXED, True) and not b.moment_path(MZ_MIXED, True)
    assert np.all(np.abs(oa - o64) <= OBJ * np.abs(o64))
    for c in range(8):
        assert _err(ga[c], g64[c]) <= GRAD
        assert _err(ga[c], gb[c]) <= 2 * GRAD
    fa = a.objective(x[:2], MZ_MIXED, forces=True)["forces"]
    f64 = b.objective(x[:2], MZ_FP64, forces=True)["forces"]
    assert np.max(np.abs(fa - f64)) <= FORCE


def _evaluator8(case, ncand, fm8):
    old = os.environ.get("MZ_FM8")
    os.environ["MZ_FM8"] = fm8
    try:
        return _evaluator(case, ncand, "2")
    finally:
        if old is None:
            del os.environ["MZ_FM8"]
        else:
            os.environ["MZ_FM8"] = old


@pytest.mark.parametrize("ncand", [64, 24, 8])
def test_integer_tensor_core_forward(ncand):
    """The forward contraction on the tensor cores (four 8-bit digits per
    operand, exact integer sums) against the CUDA-core FP32 contraction and
    FP64: objective, forces and gradient at the mixed bars, the integer path
    no less accurate than the FP32 one (twice its error at most, plus 1e-12),
    for full and partial candidate groups on a 60-cell two-species
    workload of the benchmark's rules."""
    from meamzilla_b200 import synth
    from meamzilla_b200.potential import MZ_FP64, MZ_MIXED, Database, PotentialFile
    spec, cells = synth.make_workload("meam2k", seed=3, ncells=60)
    pot = PotentialFile.from_spec(spec)
    db = Database.from_cells(cells, pot)
    case = dict(db=db, pot=pot, weights=dict(energy_weight=1.0, stress_weight=1.0, embed_extrap=0))
    x = synth.perturbed(pot.coeffs(), ncand, 0.05, seed=21)
    a = _evaluator8(case, ncand, "1")
    b = _evaluator8(case, ncand, "0")
    oa, ga = a.objective_grad(x, MZ_MIXED)
    ob, gb = b.objective_grad(x, MZ_MIXED)
    assert a.moment_path(MZ_MIXED, True) == 3 and b.moment_path(MZ_MIXED, True) == 1
    o64, g64 = b.objective_grad(x, MZ_FP64)
    ea, eb = np.abs(oa - o64) / np.abs(o64), np.abs(ob - o64) / np.abs(o64)
    assert np.all(ea <= OBJ), ea.max()
    assert ea.max() <= 2 * eb.max() + 1e-12, (ea.max(), eb.max())
    for c in range(0, ncand, max(1, ncand // 8)):
        assert _err(ga[c], g64[c]) <= GRAD
    fa = a.objective(x[:2], MZ_MIXED, forces=True)["forces"]
    fb = b.objective(x[:2], MZ_MIXED, forces=True)["forces"]
    f64 = b.objective(x[:2], MZ_FP64, forces=True)["forces"]
    assert np.max(np.abs(fa - f64)) <= FORCE
    assert np.max(np.abs(fa - f64)) <= 2 * np.max(np.abs(fb - f64)) + 1e-12
    # repeatable: integer sums in a fixed order
    oa2, _ = a.objective_grad(x, MZ_MIXED)
    assert np.array_equal(oa, oa2)


def test_integer_adjoint_against_cuda_core_adjoint():
    """The adjoint contraction on the tensor cores (MN-major moment digits,
    Z digits made in the kernel with one scale per span of 8 tiles and
    candidate, exact class sums over a span) against the CUDA-core one
    reading the same moment digits: gradients agree to the mixed path's
    rounding and both meet the bar against FP64; the integer one is within
    1e-6 of the gradient's largest component (its quantisation is 2^-31 of
    each span's largest operand)."""
    from meamzilla_b200 import synth
    from meamzilla_b200.potential import MZ_FP64, MZ_MIXED, Database, PotentialFile
    spec, cells = synth.make_workload("meam2k", seed=4, ncells=40)
    pot = PotentialFile.from_spec(spec)
    db = Database.from_cells(cells, pot)
    case = dict(db=db, pot=pot, weights=dict(energy_weight=1.0, stress_weight=1.0, embed_extrap=0))
    x = synth.perturbed(pot.coeffs(), 32, 0.05, seed=23)
    old = os.environ.get("MZ_FM8ADJ")
    os.environ["MZ_FM8ADJ"] = "0"
    try:
        b = _evaluator8(case, 32, "1")
    finally:
        if old is None:
            del os.environ["MZ_FM8ADJ"]
        else:
            os.environ["MZ_FM8ADJ"] = old
    a = _evaluator8(case, 32, "1")
    oa, ga = a.objective_grad(x, MZ_MIXED)
    ob, gb = b.objective_grad(x, MZ_MIXED)
    assert a.moment_path(MZ_MIXED, True) == 3 and b.moment_path(MZ_MIXED, True) == 2
    np.testing.assert_array_equal(oa, ob)  # the same forward
    o64, g64 = b.objective_grad(x, MZ_FP64)
    for c in range(32):
        assert _err(ga[c], g64[c]) <= GRAD
        assert _err(gb[c], g64[c]) <= GRAD
        assert _err(ga[c], gb[c]) <= GRAD
    assert max(_err(ga[c], g64[c]) for c in range(32)) <= 1e-6, [_err(ga[c], g64[c]) for c in range(32)]
