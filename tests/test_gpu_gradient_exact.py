"""FP64 adjoint against the exact gradient of the tangent-linear oracle.

The oracle's forward-mode restatement (oracle/mz_oracle.c,
mzo_objective_tangent) differentiates the reference objective statement by
statement, so it carries no finite-difference error: the FP64 adjoint must
agree with it to rounding.  The bar per component is 1e-10 of the component
plus 1e-13 of the largest component (a component many decades below the
largest one is a sum of terms that nearly cancel)."""
import os

import numpy as np
import pytest

from conftest import CASES, load_case, oracle_for

pytestmark = pytest.mark.gpu

REL = 1e-10
FLOOR = 1e-13


def _check(g, t):
    bar = REL * np.abs(t) + FLOOR * np.max(np.abs(t))
    err = np.abs(g - t)
    return bool(np.all(err <= bar)), float(np.max(err / np.maximum(np.abs(t), 1e-300))), \
        float(np.max(err) / np.max(np.abs(t)))


@pytest.mark.parametrize("name", CASES)
def test_fp64_gradient_matches_tangent_oracle(name):
    from meamzilla_b200.potential import MZ_FP64, Evaluator
    case = load_case(name)
    g = case["gold"]
    ev = Evaluator(case["db"], case["pot"], max_candidates=2, **case["weights"])
    x = np.stack([g["coeff"], g["coeff2"]])
    obj, grad = ev.objective_grad(x, MZ_FP64)
    orc = oracle_for(case)
    for c in range(2):
        t = orc.gradient(x[c])
        ok, worst_rel, worst_max = _check(grad[c], t)
        assert ok, (name, c, worst_rel, worst_max)


def _evaluator_with(env, case):
    from meamzilla_b200.potential import Evaluator
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return Evaluator(case["db"], case["pot"], max_candidates=2, **case["weights"])
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


@pytest.mark.parametrize("name", ["meam_mix6", "gmeam_mix2", "jmeam2_mix2", "meam_q5_inrange", "eam_bcc3",
                                  "gmeam_q5mix2", "jmeam2_q5mix2"])
def test_fp64_gradient_is_bitwise_reproducible(name):
    """Three calls give the same bits, and so do evaluators whose launch
    variants differ: the first variant (MZ_TUNE=0), the tuner's choice, and
    fixed persistent-CTA counts (MZ_ADJ_CTAS) of 1, 3 and 7."""
    from meamzilla_b200.potential import MZ_FP64
    case = load_case(name)
    g = case["gold"]
    x = np.stack([g["coeff"], g["coeff2"]])
    ev = _evaluator_with({}, case)
    runs = [ev.objective_grad(x, MZ_FP64)[1] for _ in range(3)]
    assert np.array_equal(runs[0], runs[1]) and np.array_equal(runs[0], runs[2])
    for env in ({"MZ_TUNE": "0"}, {"MZ_ADJ_CTAS": "1"}, {"MZ_ADJ_CTAS": "3"}, {"MZ_ADJ_CTAS": "7"}):
        other = _evaluator_with(env, case).objective_grad(x, MZ_FP64)[1]
        assert np.array_equal(runs[0], other), env
