"""The Powell driver's host logic on CPU, with the C oracle standing in for
the device residuals (opt_powell.cpp:96-315, line_min.cpp:83-151,
line_min_brent.cpp:37-126)."""
import numpy as np
import pytest


class OracleEvaluator:
    """The slice of Evaluator that powell_fit uses, over the oracle."""

    def __init__(self, orc, ncoeff):
        self.orc = orc
        self.ncoeff = ncoeff
        self.esize = orc.esize

    def objective(self, X, precision=0):
        return np.array([self.orc.objective(x) for x in np.atleast_2d(X)])

    def residuals(self, X):
        import torch
        outs = [self.orc.objective(x, full=True) for x in np.atleast_2d(X)]
        return (torch.tensor([o["obj"] for o in outs], dtype=torch.float64),
                torch.tensor(np.stack([o["errvec"] for o in outs]), dtype=torch.float64))


def exact_target_eam(ncells=6, seed=5):
    """EAM workload (densities inside U's range) whose targets are the
    teacher's own energies, stresses and forces."""
    import oracle
    from meamzilla_b200 import synth
    from meamzilla_b200.potential import Database, PotentialFile
    spec, cells = synth.make_workload("eam54", seed=seed, ncells=ncells)
    pot = PotentialFile.from_spec(synth.in_range_variant(spec))
    db = Database.from_cells(cells, pot)

    def bound():
        return oracle.CRestatement(db.view(), [pot.spline(s) for s in range(pot.nsplines)], pot.style, pot.ntypes,
                                   1.0, 1.0)

    r = bound().objective(pot.coeffs(), full=True)
    db.set_targets(r["energy"], r["stress"].ravel(), r["forces"].ravel())
    return pot, OracleEvaluator(bound(), pot.ncoeff)


def test_powell_converges_on_exact_targets():
    from meamzilla_b200.optimize import powell_fit
    pot, ev = exact_target_eam()
    x0 = pot.coeffs() + np.random.default_rng(9).normal(0.0, 0.01, pot.ncoeff)
    F0 = float(ev.objective(x0)[0])
    x, F, info = powell_fit(ev, x0, max_steps=5, residuals=ev.residuals)
    assert F < 1e-5 * F0
    hist = [h[1] for h in info["history"]]
    assert all(b <= a * (1 + 1e-12) for a, b in zip(hist, hist[1:]))
    assert info["outer"] == 5 and info["evals"] > 5 * (pot.ncoeff + 1)
    assert float(ev.objective(x)[0]) == F


def test_powell_stops_on_max_evals():
    from meamzilla_b200.optimize import powell_fit
    pot, ev = exact_target_eam()
    x0 = pot.coeffs() + np.random.default_rng(10).normal(0.0, 0.01, pot.ncoeff)
    _, F, info = powell_fit(ev, x0, max_steps=50, residuals=ev.residuals, max_evals=2 * pot.ncoeff)
    assert info["evals"] < 4 * pot.ncoeff and info["outer"] <= 2


def test_powell_reports_a_coefficient_the_objective_ignores():
    """gamma_init returns the first column with |gamma| < NOTHING and Powell
    stops ("fit impossible", opt_powell.cpp:147-153, 376-381)."""
    import torch
    from meamzilla_b200.optimize import powell_fit
    pot, ev = exact_target_eam()
    dead = 3

    def residuals(X):
        X = np.array(np.atleast_2d(X))
        X[:, dead] = pot.coeffs()[dead]  # coefficient 3 has no effect
        return ev.residuals(X)

    msgs = []
    x0 = pot.coeffs() + 0.01
    x, F, info = powell_fit(ev, x0, max_steps=3, residuals=residuals, log=msgs.append)
    assert info["outer"] == 0 and np.array_equal(x, x0)
    assert any("coefficient %d" % dead in m and "impossible" in m for m in msgs)


def test_powell_rescales_when_a_coefficient_is_ignored():
    """With rescale on, a coefficient that F ignores triggers
    Potential::rescale(1), F is recomputed and gamma_init retried
    (opt_powell.cpp:138-146); here the rescaled potential depends on every
    coefficient again, so the fit goes on."""
    from meamzilla_b200.optimize import powell_fit
    pot, ev = exact_target_eam()
    dead = 3
    calls = []

    def residuals(X):
        X = np.array(np.atleast_2d(X))
        X[:, dead] = pot.coeffs()[dead]
        return ev.residuals(X)

    def rescaler(e, x, flag):
        calls.append(flag)
        return (ev, x.copy(), ev.residuals) if flag == 1 else None

    msgs = []
    x0 = pot.coeffs() + 0.01
    x, F, info = powell_fit(ev, x0, max_steps=2, residuals=residuals, rescale=1, rescaler=rescaler, log=msgs.append)
    assert calls[0] == 1 and info["rescales"][0] == (0, "flag 1")
    assert any("trying to rescale" in m for m in msgs)
    assert info["outer"] == 2 and F < float(ev.objective(x0)[0])

    # a rescale that changes nothing leaves the fit impossible
    calls.clear()
    x, F, info = powell_fit(ev, x0, max_steps=2, residuals=residuals, rescale=1,
                            rescaler=lambda e, x, flag: calls.append(flag))
    assert calls == [1] and info["outer"] == 0


def test_powell_trial_rescale_every_fourth_step():
    """Every 4th outer step a trial Potential::rescale(0) is kept when F does
    not rise and dropped otherwise (opt_powell.cpp:262-292)."""
    from meamzilla_b200.optimize import powell_fit
    pot, ev = exact_target_eam()
    x0 = pot.coeffs() + np.random.default_rng(9).normal(0.0, 0.01, pot.ncoeff)

    class Other(OracleEvaluator):
        pass

    other = Other(ev.orc, ev.ncoeff)
    seen = []

    def keep(e, x, flag):  # the same potential under another evaluator: F2 == F
        seen.append((flag, e))
        return other, x.copy(), other.residuals

    x, F, info = powell_fit(ev, x0, max_steps=5, residuals=ev.residuals, rescale=1, rescaler=keep)
    assert [f for f, _ in seen] == [0] and seen[0][1] is ev
    assert info["rescales"] == [(3, "flag 0")] and info["evaluator"] is other

    def worse(e, x, flag):
        return other, x + 0.05, other.residuals

    x, F, info = powell_fit(ev, x0, max_steps=5, residuals=ev.residuals, rescale=1, rescaler=worse)
    assert info["rescales"] == [] and info["evaluator"] is ev
    hist = [h[0] for h in info["outer_history"]]
    assert all(b <= a for a, b in zip(hist, hist[1:]))

    # rescale 0: no trial
    seen.clear()
    powell_fit(ev, x0, max_steps=5, residuals=ev.residuals, rescale=0, rescaler=keep)
    assert seen == []
