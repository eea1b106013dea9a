"""The restated golden-section bracket and Brent minimiser (line_min.cpp:83-151,
line_min_brent.cpp:37-126) on functions with known minima."""
import math

import pytest

from meamzilla_b200.optimize import FitError, _bracket, _brent


@pytest.mark.parametrize("x0,scale", [(0.37, 1.0), (-2.5, 3.0), (12.0, 0.01), (0.05, 100.0)])
def test_bracket_and_brent_find_minimum(x0, scale):
    calls = []

    def f(x):
        calls.append(x)
        return scale * (x - x0) ** 2 + 1.0

    a, b, c, Fa, Fb, Fc = _bracket(f)
    assert min(a, c) < x0 < max(a, c) or abs(b - x0) < 1e-12
    assert Fb < Fa and Fb < Fc
    x1, x2, F1, F2 = _brent(f, a, b, c, Fb)
    # Brent stops at a relative tolerance of TOL = 0.1 (line_min_brent.h:30)
    assert abs(x1 - x0) <= 0.1 * abs(x1) + 1e-6
    assert F1 <= F2 and F1 >= 1.0


def test_bracket_gives_up_on_monotone_function():
    with pytest.raises(FitError):
        _bracket(lambda x: -x)
