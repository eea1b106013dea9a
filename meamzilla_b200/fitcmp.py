"""Powell vs L-BFGS from the same start, on a seeded synthetic workload.

    python -m meamzilla_b200.fitcmp [--workload meam200] [--seed 0] [--powell-steps 20] [--rescale F]

Builds the workload (teacher potential, targets = teacher energies / forces /
stresses + noise), starts both fits from teacher + N(0, 0.1), runs Powell
(FP64, batched Jacobian) and then L-BFGS on the adjoint with Powell's final
objective as its target, and prints one JSON line: final objectives, wall
seconds, objective evaluations.  With --rescale F the start potential is first
rescaled as Meamzilla does at start-up (meamzilla.cpp:135-143: parameter
`rescale` 2 -> flag 0, rescale when the densities leave U's range; 3 -> flag 1)
and both fits start from the rescaled coefficients; Powell then runs with the
reference's rescale hooks on (its `rescale` parameter is F + 2, non-zero:
opt_powell.cpp:138-146, 262-292).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import synth
from .optimize import lbfgs_fit, powell_fit
from .potential import MZ_FP64, MZ_MIXED, Database, Evaluator, Potential, PotentialFile


def build(workload: str, seed: int, ncells=None, max_candidates=1, in_range=False):
    spec, cells = synth.make_workload(workload, seed=seed, ncells=ncells)
    if in_range:
        spec = synth.in_range_variant(spec)
    pot = PotentialFile.from_spec(spec)
    db = Database.from_cells(cells, pot)
    ev0 = Evaluator(db, pot, 1.0, 1.0, 0, max_candidates=1)
    out = ev0.objective(pot.coeffs()[None, :], MZ_FP64, forces=True, energy=True, stress=True)
    del ev0
    rng = np.random.default_rng(3000 + seed)
    nc = len(cells)
    e0 = out["energy"][0] + rng.normal(0.0, 1e-3, nc)
    s0 = out["stress"][0] + rng.normal(0.0, 0.01, (nc, 6)) / synth.GPA_PER_EV_A3
    f0 = out["forces"][0] + rng.normal(0.0, 0.01, out["forces"][0].shape)
    db.set_targets(e0, s0.ravel(), f0.ravel())
    ev = Evaluator(db, pot, 1.0, 1.0, 0, max_candidates=max_candidates)
    return pot, db, ev


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="meam200")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--ncells", type=int, default=None)
    ap.add_argument("--powell-steps", type=int, default=20)
    ap.add_argument("--start-sigma", type=float, default=0.1)
    ap.add_argument("--in-range", action="store_true",
                    help="supplementary variant with densities inside U's range (synth.in_range_variant)")
    ap.add_argument("--rescale", type=int, default=None, help="rescale flag applied to the start potential")
    args = ap.parse_args()
    pot, db, ev = build(args.workload, args.seed, args.ncells, max_candidates=1, in_range=args.in_range)
    P = pot.ncoeff
    pot, db, ev = build(args.workload, args.seed, args.ncells, max_candidates=P, in_range=args.in_range)
    rng = np.random.default_rng(77 + args.seed)
    x0 = pot.coeffs() + rng.normal(0.0, args.start_sigma, P)
    rescaled = None
    if args.rescale is not None:
        start = Potential(ev, x0)
        F_before = float(ev.objective(x0[None, :])[0])
        rescaled = dict(flag=args.rescale, changed=bool(start.rescale(args.rescale)), objective_before=F_before)
        ev, x0 = start.ev, start.x
        pot = ev.pot
    F0 = float(ev.objective(x0[None, :])[0])
    hooks = args.rescale + 2 if args.rescale is not None else 0
    # (a rescale inside Powell gives its potential a new evaluator, ip["evaluator"];
    # L-BFGS starts from the same start potential)
    xp, Fp, ip = powell_fit(ev, x0, max_steps=args.powell_steps, rescale=hooks)
    xl, Fl, il = lbfgs_fit(ev, x0, MZ_FP64, maxiter=20000, target=Fp)
    xm, Fm, im = lbfgs_fit(ev, x0, MZ_MIXED, maxiter=20000, target=Fp)
    st = db.stats()
    print(json.dumps({
        "workload": args.workload + (" (in-range variant)" if args.in_range else ""), "natoms": st["natoms"], "ntriplets": st["ntriplets"], "ncoeff": P,
        "start_objective": F0, "rescale": rescaled,
        "powell": {"objective": Fp, "seconds": ip["seconds"], "evals": ip["evals"], "outer": ip["outer"],
                   "rescales": ip["rescales"]},
        "lbfgs_fp64": {"objective": Fl, "seconds": il["seconds"], "evals": il["evals"],
                       "reached_powell": bool(Fl <= Fp)},
        "lbfgs_mixed": {"objective": Fm, "seconds": im["seconds"], "evals": im["evals"],
                        "reached_powell": bool(Fm <= Fp)},
    }))


if __name__ == "__main__":
    main()
