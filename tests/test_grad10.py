"""The 10-point gradient check on the 200-cell single-species MEAM workload.

Fixture (tests/golden/meam200_grad10/grad10.npz, written by make_golden.py
--grad10 with the compiled reference): 10 seeded coefficient vectors per
variant (the teacher as generated, and its in-range variant), the
reference's objective at each and its central differences (h = 1e-6,
Potential::compute differenced as opt_powell.cpp:363-384 does).  The
database is regenerated from the seeds; its targets are the teacher's
outputs + seeded noise, so they agree with the fixture's to rounding.

CPU: the oracle against the fixture.  GPU: the hand-written adjoint through
torch.autograd (meamzilla_b200.autograd) against the reference's
differences, torch.autograd.gradcheck against central differences of the
GPU objective, and the mixed-precision adjoint against the FP64 one."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel

FIXTURE = os.path.join(GOLDEN, "meam200_grad10", "grad10.npz")
VARIANTS = ["raw", "inrange"]
GRAD_REF_FD = 1e-6   # FP64 adjoint vs the reference's differences, of max|g|
GRAD_MIX = 1e-4      # mixed-precision adjoint vs FP64 adjoint, of max|g|


def _err(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _database(variant, teacher_outputs):
    """PotentialFile and Database of the check; teacher_outputs(pot, db) ->
    (energy [ncells], stress [ncells, 6], forces [natoms, 3])."""
    from meamzilla_b200 import synth
    from meamzilla_b200.potential import Database, PotentialFile
    spec, cells = synth.grad10_workload(variant)
    pot = PotentialFile.from_spec(spec)
    e, s, f = teacher_outputs(pot, Database.from_cells(cells, pot))
    synth.set_teacher_targets(cells, e, s, f, synth.GRAD10["target_seed"])
    return pot, Database.from_cells(cells, pot)


def _oracle(pot, db):
    import oracle
    return oracle.CRestatement(db.view(), [pot.spline(s) for s in range(pot.nsplines)], pot.style, pot.ntypes,
                               1.0, 1.0)


@pytest.mark.parametrize("variant", VARIANTS)
def test_oracle_matches_reference_at_ten_points(variant):
    fx = np.load(FIXTURE)

    def teacher(pot, db):
        r = _oracle(pot, db).objective(pot.coeffs(), full=True)
        return r["energy"], r["stress"], r["forces"]

    pot, db = _database(variant, teacher)
    orc = _oracle(pot, db)
    X, F, G = fx["x_" + variant], fx["obj_" + variant], fx["fdgrad_" + variant]
    for i in range(len(X)):
        assert rel(orc.objective(X[i]), F[i]) <= 1e-12, (variant, i)
    # the oracle's own central differences at one point, on a spread of coefficients
    x = X[3]
    for j in (0, 11, 23, 31, 40, 55):
        xp, xm = x.copy(), x.copy()
        xp[j] += 1e-6
        xm[j] -= 1e-6
        g = (orc.objective(xp) - orc.objective(xm)) / 2e-6
        assert abs(g - G[3][j]) <= 1e-6 * np.max(np.abs(G[3])), (variant, j, g, G[3][j])


def _gpu_case(variant, ncand):
    from meamzilla_b200.potential import MZ_FP64, Evaluator

    def teacher(pot, db):
        ev = Evaluator(db, pot, 1.0, 1.0, 0, max_candidates=1)
        r = ev.objective(pot.coeffs()[None, :], MZ_FP64, forces=True, energy=True, stress=True)
        return r["energy"][0], r["stress"][0], r["forces"][0]

    pot, db = _database(variant, teacher)
    return Evaluator(db, pot, 1.0, 1.0, 0, max_candidates=ncand)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", VARIANTS)
def test_autograd_adjoint_vs_reference_differences(variant):
    import torch
    from meamzilla_b200.autograd import objective
    fx = np.load(FIXTURE)
    ev = _gpu_case(variant, 10)
    X, F, G = fx["x_" + variant], fx["obj_" + variant], fx["fdgrad_" + variant]
    dev = torch.device("cuda:0")
    for i in range(len(X)):
        x = torch.tensor(X[i], dtype=torch.float64, device=dev, requires_grad=True)
        obj = objective(x, ev)
        obj.backward()
        assert rel(float(obj.detach()), F[i]) <= 1e-12, (variant, i)
        assert _err(x.grad.cpu().numpy(), G[i]) <= GRAD_REF_FD, (variant, i, _err(x.grad.cpu().numpy(), G[i]))
    # all ten points in one batched call: the same objectives and gradients
    Xt = torch.tensor(X, dtype=torch.float64, device=dev, requires_grad=True)
    objective(Xt, ev).sum().backward()
    for i in range(len(X)):
        assert _err(Xt.grad[i].cpu().numpy(), G[i]) <= GRAD_REF_FD


@pytest.mark.gpu
@pytest.mark.parametrize("variant", VARIANTS)
def test_gradcheck_against_gpu_central_differences(variant):
    import torch
    from meamzilla_b200.autograd import objective
    from meamzilla_b200.potential import MZ_FP64, MZ_MIXED
    fx = np.load(FIXTURE)
    ev = _gpu_case(variant, 2)
    X = fx["x_" + variant]
    for i in (0, 9):
        x = torch.tensor(X[i], dtype=torch.float64, device="cuda:0", requires_grad=True)
        _, g = ev.objective_grad(X[i][None, :], MZ_FP64)
        scale = float(np.max(np.abs(g)))
        assert torch.autograd.gradcheck(lambda t: objective(t, ev), (x,), eps=1e-6, atol=1e-7 * scale, rtol=1e-7)
        _, gm = ev.objective_grad(X[i][None, :], MZ_MIXED)
        assert _err(gm[0], g[0]) <= GRAD_MIX, (variant, i, _err(gm[0], g[0]))
