"""Hand-written adjoint against central finite differences.

The reference has no gradient: its optimizers difference compute()
(opt_powell.cpp:348-389).  The GPU gradient is checked against central
differences of the CPU oracle (h = 1e-5 |x|), against the reference's own
central differences (golden fdgrad, h = 1e-6), and the mixed-precision
gradient against the FP64 one.  Errors are measured against the largest
gradient component (the components span many decades)."""
import numpy as np
import pytest

from conftest import CASES, load_case, oracle_for

pytestmark = pytest.mark.gpu

GRAD_FD = 1e-6      # FP64 adjoint vs oracle central differences
GRAD_REF_FD = 1e-5  # vs the reference's h = 1e-6 differences (their own error)
GRAD_MIX = 1e-4     # mixed-precision adjoint vs FP64 adjoint
GRAD_MIX_SPLINE = 1e-3  # the same per spline, against the spline's largest component


def _fd(orc, x, rel_h=1e-5):
    g = np.zeros_like(x)
    for i in range(x.size):
        h = rel_h * max(1.0, abs(x[i]))
        xp = x.copy()
        xp[i] += h
        xm = x.copy()
        xm[i] -= h
        g[i] = (orc.objective(xp) - orc.objective(xm)) / (2 * h)
    return g


def _err(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", CASES)
def test_fp64_gradient_vs_finite_differences(name):
    from meamzilla_b200.potential import MZ_FP64, Evaluator
    case = load_case(name)
    g = case["gold"]
    ev = Evaluator(case["db"], case["pot"], max_candidates=2, **case["weights"])
    x = np.stack([g["coeff"], g["coeff2"]])
    obj, grad = ev.objective_grad(x, MZ_FP64)
    orc = oracle_for(case)
    for c in range(2):
        assert abs(obj[c] - orc.objective(x[c])) <= 1e-12 * abs(obj[c])
        fd = _fd(orc, x[c])
        assert _err(grad[c], fd) <= GRAD_FD, (name, c, _err(grad[c], fd))
    if "fdgrad" in g:
        assert _err(grad[0], g["fdgrad"]) <= GRAD_REF_FD


@pytest.mark.parametrize("name", ["meam_mix6", "meam2_edge", "eam_bcc3", "pair_mix2", "jmeam_inrange1",
                                  "jmeam2_mix2", "meam_q5_inrange", "eam_q5", "gmeam_q5", "jmeam_q5",
                                  "jmeam2_q5mix2", "meam_mixb2", "eam_mixb"])
def test_mixed_gradient_vs_fp64(name):
    from meamzilla_b200.potential import MZ_FP64, MZ_MIXED, Evaluator
    case = load_case(name)
    g = case["gold"]
    ev = Evaluator(case["db"], case["pot"], max_candidates=2, **case["weights"])
    x = np.stack([g["coeff"], g["coeff2"]])
    o64, g64 = ev.objective_grad(x, MZ_FP64)
    o32, g32 = ev.objective_grad(x, MZ_MIXED)
    assert np.all(np.abs(o32 - o64) <= 1e-6 * np.abs(o64))
    for c in range(2):
        assert _err(g32[c], g64[c]) <= GRAD_MIX


def test_gradient_objective_equals_plain_objective():
    """mz_objective_grad's objective is the same number mz_objective returns."""
    from meamzilla_b200.potential import MZ_FP64, Evaluator
    case = load_case("meam2_edge")
    ev = Evaluator(case["db"], case["pot"], max_candidates=3, **case["weights"])
    rng = np.random.default_rng(1)
    x = case["gold"]["coeff"][None, :] + rng.normal(0, 0.02, (3, case["gold"]["coeff"].size))
    o1 = ev.objective(x, MZ_FP64)
    o2, _ = ev.objective_grad(x, MZ_FP64)
    assert np.array_equal(o1, o2)


def _spline_slices(pot):
    """Coefficient ranges of the splines, in order: each spline's free knot
    values, then its free end slopes (spline3eq.cpp:77-100, 376-382)."""
    out, lo = [], 0
    for s in range(pot.nsplines):
        sp = pot.spline(s)
        n = int(np.sum(sp["y_fixed"] == 0)) + sum(1 for e in range(2) if not sp["grad_fixed"][e] and not sp["nat"][e])
        out.append((lo, lo + n))
        lo += n
    return out if lo == pot.ncoeff else None


@pytest.mark.parametrize("name", ["meam_mix6", "meam2_edge", "eam_bcc3", "pair_mix2", "jmeam_inrange1",
                                  "jmeam2_mix2"])
def test_mixed_gradient_vs_fp64_per_spline(name):
    """The same comparison per spline, each block against its own largest
    component: an error confined to a spline with small gradients (the
    angular g, the f of MEAM) is not hidden by the largest components of
    another spline."""
    from meamzilla_b200.potential import MZ_FP64, MZ_MIXED, Evaluator
    case = load_case(name)
    g = case["gold"]
    slices = _spline_slices(case["pot"])
    assert slices is not None
    ev = Evaluator(case["db"], case["pot"], max_candidates=2, **case["weights"])
    x = np.stack([g["coeff"], g["coeff2"]])
    _, g64 = ev.objective_grad(x, MZ_FP64)
    _, g32 = ev.objective_grad(x, MZ_MIXED)
    for c in range(2):
        top = np.max(np.abs(g64[c]))
        for s, (lo, hi) in enumerate(slices):
            if hi == lo or np.max(np.abs(g64[c, lo:hi])) < 1e-6 * top:
                continue
            assert _err(g32[c, lo:hi], g64[c, lo:hi]) <= GRAD_MIX_SPLINE, (name, c, s)
