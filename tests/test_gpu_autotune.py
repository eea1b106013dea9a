"""The launch autotuner (mz_tuning): the first objective call of a precision,
with and without the gradient, times the forward and the adjoint at three
atom-block sizes (the adjoint at two persistent-grid sizes, the mixed MEAM
forward with one and two candidates per CTA) and keeps the fastest.  FP64
results are bit-identical across variants; mixed results agree to rounding
of FP32 chunk sums; gradients to rounding.  MZ_TUNE=0 keeps the first
variant, MZ_TUNE=2 the first with two candidates per CTA."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _workload():
    from meamzilla_b200 import synth
    from meamzilla_b200.potential import Database, PotentialFile
    spec, cells = synth.make_workload("meam2k", seed=21, ncells=40)
    rng = np.random.default_rng(5)
    for c in cells:
        c.energy0 = float(rng.normal(-3.0, 0.1))
        c.force0 = rng.normal(0.0, 0.3, (c.natoms, 3))
        c.stress0 = rng.normal(0.0, 1e-3, 6)
    pot = PotentialFile.from_spec(synth.in_range_variant(spec))
    return pot, Database.from_cells(cells, pot)


def test_tuned_and_untuned_variants_agree(monkeypatch):
    from meamzilla_b200 import synth
    from meamzilla_b200.potential import MZ_FP64, MZ_MIXED, Evaluator
    pot, db = _workload()
    X = synth.perturbed(pot.coeffs(), 4, 0.01, seed=6)
    monkeypatch.setenv("MZ_TUNE", "0")
    fixed = Evaluator(db, pot, 1.0, 1.0, 0, max_candidates=4)
    monkeypatch.delenv("MZ_TUNE")
    tuned = Evaluator(db, pot, 1.0, 1.0, 0, max_candidates=4)
    for prec, gtol in ((MZ_FP64, 1e-11), (MZ_MIXED, 1e-5)):
        a = fixed.objective(X, prec, errvec=True, forces=True)
        b = tuned.objective(X, prec, errvec=True, forces=True)
        oa, ga = fixed.objective_grad(X, prec)
        ob, gb = tuned.objective_grad(X, prec)
        if prec == MZ_FP64:
            for k in ("obj", "errvec", "forces"):
                assert np.array_equal(a[k], b[k]), k
            assert np.array_equal(oa, ob)
        else:
            assert np.max(np.abs(a["obj"] - b["obj"]) / a["obj"]) <= 1e-6
            assert np.max(np.abs(a["forces"] - b["forces"])) <= 1e-5
            assert np.max(np.abs(oa - ob) / oa) <= 1e-6
        assert np.max(np.abs(ga - gb)) <= gtol * np.max(np.abs(ga)), prec
        t0, t1 = fixed.tuning(prec, True), tuned.tuning(prec, True)
        assert t0["forward_block_slots"] == 256 and t0["adjoint_block_slots"] == 256
        assert t1["forward_block_slots"] in (256, 192, 128) and t1["adjoint_block_slots"] in (256, 192, 128)
        assert t1["adjoint_ctas"] >= 1
    # the tuned choice is fixed for the context: a repeat is bit-identical
    oc, gc = tuned.objective_grad(X, MZ_MIXED)
    assert np.array_equal(gc, gb)


@pytest.mark.parametrize("name", ["meam_mix6", "meam2_edge", "meam_inrange_w"])
def test_two_candidates_per_cta_match_one(name, monkeypatch):
    """k_atoms2 / k_adj2 (two candidates per CTA, packed FP32 pairs) against
    k_atoms / k_adj: for an odd number of candidates (the last CTA holds
    one) both meet the mixed-precision bars against FP64 (objective 1e-6,
    forces 1e-5 eV/A, gradient 1e-4 of its largest component; their FP32
    roundings differ, so they are not bit-identical), and the FP64 path is
    untouched."""
    from conftest import load_case
    from meamzilla_b200.potential import MZ_FP64, MZ_MIXED, Evaluator
    case = load_case(name)
    g = case["gold"]
    rng = np.random.default_rng(8)
    X = g["coeff"][None, :] + rng.normal(0.0, 0.01, (5, g["coeff"].size))
    monkeypatch.setenv("MZ_TUNE", "0")
    one = Evaluator(case["db"], case["pot"], max_candidates=5, **case["weights"])
    monkeypatch.setenv("MZ_TUNE", "2")
    two = Evaluator(case["db"], case["pot"], max_candidates=5, **case["weights"])
    a = one.objective(X, MZ_MIXED, errvec=True, forces=True)
    b = two.objective(X, MZ_MIXED, errvec=True, forces=True)
    assert two.tuning(MZ_MIXED, False)["forward_candidates_per_cta"] == 2
    assert one.tuning(MZ_MIXED, False)["forward_candidates_per_cta"] == 1
    ref = one.objective(X, MZ_FP64, forces=True)
    for r in (a, b):
        assert np.max(np.abs(r["obj"] - ref["obj"]) / ref["obj"]) <= 1e-6
        assert np.max(np.abs(r["forces"] - ref["forces"])) <= 1e-5
    oa, ga = one.objective_grad(X, MZ_MIXED)
    ob, gb = two.objective_grad(X, MZ_MIXED)
    assert two.tuning(MZ_MIXED, True)["adjoint_candidates_per_cta"] == 2
    assert np.max(np.abs(oa - ob) / oa) <= 1e-6
    assert np.max(np.abs(ga - gb)) <= 1e-4 * np.max(np.abs(ga))
    _, g64 = one.objective_grad(X, MZ_FP64)
    assert np.max(np.abs(gb - g64)) <= 1e-4 * np.max(np.abs(g64))
    # repeated calls of the two-candidate adjoint are bit-identical
    assert np.array_equal(two.objective_grad(X, MZ_MIXED)[1], gb)
    assert np.array_equal(ref["obj"], two.objective(X, MZ_FP64))
