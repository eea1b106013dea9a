"""Generate the golden fixtures under tests/golden/ from the REFERENCE itself.

Each case directory holds the reference-format inputs (start.pot, db.conf,
param with relative file names) and golden.npz with what the compiled,
unmodified reference (oracle/_ref/mzref, built by oracle/Makefile) returns
through Potential::compute for two coefficient vectors:

    obj, errvec, force, energy, stress, dens, coeff       (file coefficients)
    obj2, errvec2, force2, energy2, stress2, coeff2      (perturbed vector)
    fdgrad (central differences of the objective, h = 1e-6; small cases)

Run here (needs the reference sources to build mzref):
    make -C oracle && python tests/golden/make_golden.py [--gmeam | --grad10 | --pair | --jmeam | --quintic
                                                          | --powell | --quintic-styles]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from meamzilla_b200 import synth  # noqa: E402
import oracle  # noqa: E402


def _targets(cells, seed):
    rng = np.random.default_rng(seed)
    for c in cells:
        c.energy0 = float(rng.normal(-3.0, 0.1))
        c.force0 = rng.normal(0.0, 0.3, (c.natoms, 3))
        c.stress0 = rng.normal(0.0, 1e-3, 6)


def _write(name, pot, cells, fd=False, perturb=0.02, **param_kw):
    d = os.path.join(HERE, name)
    os.makedirs(d, exist_ok=True)
    synth.write_pot(os.path.join(d, "start.pot"), pot)
    synth.write_config(os.path.join(d, "db.conf"), cells)
    lines = ["config db.conf", "startpot start.pot", "tempfile tempfile", "endpot endpot"]
    lines += ["energy_weight %s" % param_kw.get("energy_weight", 1.0),
              "stress_weight %s" % param_kw.get("stress_weight", 1.0), "rescale 0"]
    if param_kw.get("embed_extrap"):
        lines.append("embed_extrap %d" % param_kw["embed_extrap"])
    with open(os.path.join(d, "param"), "w") as fh:
        fh.write("\n".join(lines) + "\n")
    ref = oracle.run_reference("param", cwd=d, fd_h=1e-6 if fd else 0.0)
    out = dict(obj=ref["obj"], errvec=ref["errvec"], force=ref["force"], energy=ref["energy"], stress=ref["stress"],
               coeff=ref["coeff"])
    if "dens" in ref:
        out["dens"] = ref["dens"]
    if fd:
        out["fdgrad"] = ref["fdgrad"]
    rng = np.random.default_rng(99)
    x2 = ref["coeff"] + rng.normal(0.0, perturb, ref["coeff"].size)
    ref2 = oracle.run_reference("param", cwd=d, coeffs=x2)
    out.update(obj2=ref2["obj"], errvec2=ref2["errvec"], force2=ref2["force"], energy2=ref2["energy"],
               stress2=ref2["stress"], coeff2=x2)
    np.savez_compressed(os.path.join(d, "golden.npz"), **out)
    print(name, "obj", ref["obj"], "natoms", sum(c.natoms for c in cells), "esize", ref["errvec"].size)


def in_range_meam(pot):
    """Scale rho and f knots so densities fall inside U's [-1, 1] range (the
    teacher's densities lie far outside it)."""
    p = pot.copy()
    for s in p.groups[1]:
        s.y *= 0.02
        s.grad *= 0.02
    for s in p.groups[3]:
        s.y *= 0.12
        s.grad *= 0.12
    return p


def gmeam_goldens():
    """gmeam/spline: g indexed by (i; j, k) types, one f punishment per f spline."""
    # 6. two species, cells of the two-species rule, teacher as generated
    _, cells = synth.make_workload("meam2k", seed=8, ncells=3)
    cells = [c for c in cells if c.natoms <= 400][:3] or cells[:1]
    _targets(cells, 6)
    pot = synth.teacher_potential("gmeam/spline", 2, 5.5, seed=21)
    _write("gmeam_mix2", pot, cells, fd=True)
    # 7. one species in range (no density punishment), per-cell weights
    _, cells = synth.make_workload("meam200", seed=9, ncells=4)
    _targets(cells, 7)
    for i, c in enumerate(cells):
        c.weight = 1.0 + 0.25 * i
    pot = synth.teacher_potential("gmeam/spline", 1, 4.5, seed=22)
    _write("gmeam_inrange1", in_range_meam(pot), cells, fd=True, energy_weight=1.5, stress_weight=0.5)


def pair_goldens():
    """pair/spline: phi only, each pair once, self images at one half."""
    # 8. one species: three bcc cells of the eam54 rules and a one-atom cell
    #    whose only neighbours are its own images
    _, cells = synth.make_workload("eam54", seed=13, ncells=3)
    cells.append(synth.Cell(lattice=np.diag([2.9, 3.1, 3.3]), types=np.zeros(1, dtype=np.int64),
                            pos=np.array([[0.1, 0.2, 0.3]]), force0=np.zeros((1, 3))))
    _targets(cells, 8)
    pot = synth.teacher_potential("pair/spline", 1, 5.0, seed=23)
    _write("pair_bcc1", pot, cells, fd=True)
    # 9. two species, cells of the two-species rule; phi_AB's grid ends at
    #    4.6 A, so A-B pairs between 4.6 and 5.5 A are not in the list
    #    (check_pair drops them), phi_BB has a natural left end and two fixed knots
    _, cells = synth.make_workload("meam2k", seed=14, ncells=4)
    cells = [c for c in cells if c.natoms <= 300][:3] or cells[:1]
    _targets(cells, 9)
    pot = synth.teacher_potential("pair/spline", 2, 5.5, seed=24)
    ab = pot.groups[0][1]
    pot.groups[0][1] = synth.Spline(1.8, 4.6, np.interp(np.linspace(1.8, 4.6, 10), np.linspace(1.8, 5.5, 10), ab.y),
                                    ab.grad.copy())
    pot.groups[0][2].bc = (-1, 0)
    pot.groups[0][2].fixed = np.zeros(10, dtype=int)
    pot.groups[0][2].fixed[[2, 7]] = 1
    _write("pair_mix2", pot, cells, fd=True, energy_weight=2.0, stress_weight=0.5)


JMEAM_CASES = ["jmeam_inrange1", "jmeam_mix2", "jmeam2_mix2"]


def jmeam_goldens():
    """jmeam/spline and jmeam2/spline: MEAM + sum_{j<k} p_ij p_ik q_i(cos)
    (and a second such term) in the energy, f and p magnitude punishments."""
    # 10. one species, densities in range (rho and f scaled), per-cell weights
    _, cells = synth.make_workload("meam200", seed=15, ncells=4)
    _targets(cells, 10)
    for i, c in enumerate(cells):
        c.weight = 1.0 + 0.2 * i
    pot = synth.teacher_potential("jmeam/spline", 1, 4.5, seed=25)
    _write(JMEAM_CASES[0], in_range_meam(pot), cells, fd=True, energy_weight=1.5, stress_weight=0.8)
    # 11./12. two species, cells of the two-species rule, teacher as generated
    _, cells = synth.make_workload("meam2k", seed=16, ncells=4)
    cells = [c for c in cells if c.natoms <= 300][:3] or cells[:1]
    _targets(cells, 11)
    _write(JMEAM_CASES[1], synth.teacher_potential("jmeam/spline", 2, 5.5, seed=26), cells, fd=True)
    _write(JMEAM_CASES[2], synth.teacher_potential("jmeam2/spline", 2, 5.5, seed=27), cells, fd=True)


Q5_CASES = ["eam_q5", "meam_q5_inrange", "pair_q5"]


def quintic_goldens():
    """spline5eq bases (Spline5Eq, spline5eq.cpp): end y'' read and written,
    the 2n x 2n refresh, quadratic extrapolation of U, and the coefficient
    walk that visits slope and y'' of every free end while get_ncoeff counts
    one (spline5eq.cpp:81-85, 459-468)."""
    # 13. EAM, three bcc cells; phi with both ends free, rho with a natural right end
    _, cells = synth.make_workload("eam54", seed=17, ncells=3)
    _targets(cells, 13)
    pot = synth.quintic_variant(synth.teacher_potential("eam/spline", 1, 5.0, seed=28), seed=1)
    pot.groups[0][0].bc = (0, 0)
    pot.groups[1][0].bc = (0, -1)
    _write(Q5_CASES[0], pot, cells)
    # 14. MEAM in range (the start-up rescale runs), per-cell weights
    _, cells = synth.make_workload("meam200", seed=18, ncells=3)
    _targets(cells, 14)
    for i, c in enumerate(cells):
        c.weight = 1.0 + 0.3 * i
    pot = synth.quintic_variant(in_range_meam(synth.teacher_potential("meam/spline", 1, 4.5, seed=29)), seed=2)
    _write(Q5_CASES[1], pot, cells, energy_weight=1.2, stress_weight=0.6)
    # 15. pair/spline, two species, one natural end
    _, cells = synth.make_workload("meam2k", seed=19, ncells=4)
    cells = [c for c in cells if c.natoms <= 300][:2] or cells[:1]
    _targets(cells, 15)
    pot = synth.quintic_variant(synth.teacher_potential("pair/spline", 2, 5.5, seed=30), seed=3)
    pot.groups[0][1].bc = (-1, 0)
    _write(Q5_CASES[2], pot, cells)


Q5B_CASES = ["gmeam_q5", "gmeam_q5mix2", "jmeam_q5", "jmeam2_q5mix2", "meam_mixb2", "eam_mixb"]


def quintic_styles_goldens():
    """spline5eq in gmeam/spline and jmeam[2]/spline potentials, and
    potentials mixing spline3eq and spline5eq functions (the reference reads
    the basis per function, pot_fns.cpp:439-465, and evaluates a mixed
    potential through the virtual Spline path, pot_meam_spline.cpp:56-73)."""
    # 16. gmeam, one species in range, every function quintic, per-cell weights
    _, cells = synth.make_workload("meam200", seed=31, ncells=3)
    _targets(cells, 16)
    for i, c in enumerate(cells):
        c.weight = 1.0 + 0.25 * i
    pot = synth.quintic_variant(in_range_meam(synth.teacher_potential("gmeam/spline", 1, 4.5, seed=32)), seed=4)
    _write(Q5B_CASES[0], pot, cells, fd=True, energy_weight=1.3, stress_weight=0.7)
    # 17. gmeam, two species: phi and f quintic, the rest cubic
    _, cells = synth.make_workload("meam2k", seed=33, ncells=4)
    cells = [c for c in cells if c.natoms <= 300][:3] or cells[:1]
    _targets(cells, 17)
    pot = synth.quintic_variant(synth.teacher_potential("gmeam/spline", 2, 5.5, seed=34), seed=5, groups=(0, 3))
    _write(Q5B_CASES[1], pot, cells, fd=True)
    # 18. jmeam, one species in range, every function quintic
    _, cells = synth.make_workload("meam200", seed=35, ncells=3)
    _targets(cells, 18)
    pot = synth.quintic_variant(in_range_meam(synth.teacher_potential("jmeam/spline", 1, 4.5, seed=36)), seed=6)
    _write(Q5B_CASES[2], pot, cells, fd=True)
    # 19. jmeam2, two species: phi, g and q quintic, the rest cubic
    _, cells = synth.make_workload("meam2k", seed=37, ncells=4)
    cells = [c for c in cells if c.natoms <= 300][:3] or cells[:1]
    _targets(cells, 19)
    pot = synth.quintic_variant(synth.teacher_potential("jmeam2/spline", 2, 5.5, seed=38), seed=7, groups=(0, 4, 6))
    _write(Q5B_CASES[3], pot, cells, fd=True)
    # 20. meam, two species: U and g quintic, the rest cubic; in range
    _, cells = synth.make_workload("meam2k", seed=39, ncells=4)
    cells = [c for c in cells if c.natoms <= 300][:3] or cells[:1]
    _targets(cells, 20)
    pot = synth.quintic_variant(in_range_meam(synth.teacher_potential("meam/spline", 2, 5.5, seed=40)), seed=8,
                                groups=(2, 4))
    _write(Q5B_CASES[4], pot, cells, fd=True)
    # 21. eam: phi quintic, rho and U cubic
    _, cells = synth.make_workload("eam54", seed=41, ncells=3)
    _targets(cells, 21)
    pot = synth.quintic_variant(synth.teacher_potential("eam/spline", 1, 5.0, seed=42), seed=9, groups=(0,))
    _write(Q5B_CASES[5], pot, cells, fd=True)


def data_goldens(names=None):
    """ref.{rho,energy,stress,force,error,punish}: the text files the
    reference's Potential::write_data writes for the start potential."""
    for name in sorted(names or os.listdir(HERE)):
        d = os.path.join(HERE, name)
        if os.path.isfile(os.path.join(d, "param")):
            oracle.run_reference("param", cwd=d, write_prefix=os.path.join(d, "ref"))
            print(name, "data files written")


def rescale_goldens(names=None):
    """rescale.npz of every case: the reference's Potential::rescale with
    flag 0 (when needed) and 1 (always), run on the start potential, dumped
    spline by spline by the harness (oracle/ref_harness.cpp -rescale)."""
    for name in sorted(names or os.listdir(HERE)):
        d = os.path.join(HERE, name)
        if not os.path.isfile(os.path.join(d, "param")):
            continue
        out = {}
        for flag in (0, 1):
            r = oracle.run_reference("param", cwd=d, rescale=flag)
            out["flag%d" % flag] = r["rescale"]
            out["obj%d" % flag] = r["obj"]  # Potential::compute after the rescale
        np.savez_compressed(os.path.join(d, "rescale.npz"), **out)
        print(name, "rescale returns", out["flag0"][0], out["flag1"][0])


def grad10_goldens():
    """The reference's central differences (h = 1e-6, ref_harness -fd) of the
    objective at 10 seeded points on the 200-cell single-species MEAM
    workload, for the teacher as generated and its in-range variant; targets
    = the reference's teacher outputs + seeded noise (synth.GRAD10).  Only
    the points and the reference's results are stored: the database is
    regenerated from the seeds by synth.grad10_workload."""
    import shutil
    import tempfile
    from concurrent.futures import ThreadPoolExecutor
    out = {}
    tmp = tempfile.mkdtemp()
    try:
        for variant in ("raw", "inrange"):
            pot, cells = synth.grad10_workload(variant)
            d = os.path.join(tmp, variant)
            par = synth.write_case(d, pot, cells)
            t = oracle.run_reference(par, cwd=d)
            synth.set_teacher_targets(cells, t["energy"], t["stress"], t["force"], synth.GRAD10["target_seed"])
            synth.write_config(os.path.join(d, "db.conf"), cells)
            x0 = oracle.run_reference(par, cwd=d)["coeff"]
            X = synth.perturbed(x0, synth.GRAD10["npoints"], synth.GRAD10["sigma"][variant],
                                synth.GRAD10["point_seed"])
            with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as pool:
                res = list(pool.map(lambda x: oracle.run_reference(par, cwd=d, coeffs=x, fd_h=1e-6), X))
            out["x_" + variant] = X
            out["obj_" + variant] = np.array([r["obj"] for r in res])
            out["fdgrad_" + variant] = np.stack([r["fdgrad"] for r in res])
            print("grad10", variant, "natoms", sum(c.natoms for c in cells), "obj", out["obj_" + variant][:3])
    finally:
        shutil.rmtree(tmp)
    d = os.path.join(HERE, "meam200_grad10")
    os.makedirs(d, exist_ok=True)
    np.savez_compressed(os.path.join(d, "grad10.npz"), **out)


POWELL = dict(workload="eam54", seed=5, ncells=6, start_seed=9, start_sigma=0.01, steps=8)


def powell_case():
    """The Powell parity case: eam54 cells (seed 5, 6 cells), the in-range
    teacher; phi and rho free except knots 0-2, U fixed, both end slopes of
    every spline fixed -- 14 coefficients, a well-determined least-squares
    problem (with U free the exact-target problem is ill-conditioned and
    Powell's path is too sensitive to rounding to compare)."""
    pot, cells = synth.make_workload(POWELL["workload"], seed=POWELL["seed"], ncells=POWELL["ncells"])
    pot = synth.in_range_variant(pot)
    for gi, grp in enumerate(pot.groups):
        for sp in grp:
            fixed = np.zeros(sp.nknots, dtype=int)
            fixed[:3 if gi < 2 else sp.nknots] = 1
            sp.fixed = fixed
            sp.bc = (1, 1)
    return pot, cells


def powell_goldens():
    """eam_powell4/powell.npz: the reference's OptPowell::compute_pot
    (opt_powell.cpp:96-315) run for 1..4 outer steps by the harness
    (oracle/ref_harness.cpp -powell) from a seeded start, with targets = the
    reference's own teacher outputs.  F[k] and X[k] after outer step k+1."""
    name = "eam_powell4"
    d = os.path.join(HERE, name)
    os.makedirs(d, exist_ok=True)
    pot, cells = powell_case()
    synth.write_pot(os.path.join(d, "start.pot"), pot)
    synth.write_config(os.path.join(d, "db.conf"), cells)
    with open(os.path.join(d, "param"), "w") as fh:
        fh.write("config db.conf\nstartpot start.pot\ntempfile tempfile\nendpot endpot\n"
                 "energy_weight 1.0\nstress_weight 1.0\nrescale 0\n")
    t = oracle.run_reference("param", cwd=d)
    a0 = np.cumsum([0] + [c.natoms for c in cells])
    force = np.asarray(t["force"]).reshape(-1, 3)
    for i, c in enumerate(cells):
        c.energy0 = float(t["energy"][i])
        c.stress0 = np.asarray(t["stress"]).reshape(-1, 6)[i].copy()
        c.force0 = force[a0[i]:a0[i + 1]].copy()
    synth.write_config(os.path.join(d, "db.conf"), cells)
    x_teacher = t["coeff"]
    x0 = x_teacher + np.random.default_rng(POWELL["start_seed"]).normal(0.0, POWELL["start_sigma"], x_teacher.size)
    K = POWELL["steps"]
    r = oracle.run_reference("param", cwd=d, coeffs=x0, powell_steps=K)
    pw = np.asarray(r["powell"]).reshape(K, x0.size + 1)
    for f in os.listdir(d):  # the optimizer's temporary potentials
        if f.startswith("tempfile"):
            os.remove(os.path.join(d, f))
    np.savez_compressed(os.path.join(d, "powell.npz"), x0=x0, obj0=r["obj"], F=pw[:, 0], X=pw[:, 1:],
                        x_teacher=x_teacher)
    print(name, "P", x0.size, "F0", r["obj"], "F", pw[:, 0])


def main():
    # 1. EAM, 3 bcc cells (the eam54 rules)
    pot, cells = synth.make_workload("eam54", seed=3, ncells=3)
    _targets(cells, 1)
    _write("eam_bcc3", pot, cells, fd=True)

    # 2. MEAM, 6 cells of the meam200 mixture
    pot, cells = synth.make_workload("meam200", seed=3, ncells=6)
    _targets(cells, 2)
    _write("meam_mix6", pot, cells, fd=True)

    # 3. MEAM in range (no density punishment), embed_extrap, per-cell weights
    pot, cells = synth.make_workload("meam200", seed=4, ncells=4)
    _targets(cells, 3)
    for i, c in enumerate(cells):
        c.weight, c.eweight, c.sweight = 1.0 + 0.5 * i, 2.0 - 0.3 * i, 0.5 + 0.2 * i
    _write("meam_inrange_w", in_range_meam(pot), cells, fd=True, energy_weight=2.5, stress_weight=0.7)

    # 4. two-species MEAM (meam2k rules), natural and fixed ends, fixed knots,
    #    a g grid narrower than [-1, 1] (cos beyond it is not a triplet; below
    #    it the cubic is extrapolated), embed_extrap 1
    pot, cells = synth.make_workload("meam2k", seed=5, ncells=3)
    _targets(cells, 4)
    p = pot.copy()
    p.groups[0][1].bc = (-1, 1)                 # phi_AB: natural left, fixed right slope
    p.groups[1][0].bc = (1, -1)                 # rho_A: fixed left, natural right
    p.groups[3][2].fixed = np.zeros(10, dtype=int)
    p.groups[3][2].fixed[[0, 4, 9]] = 1         # f_BB: three fixed knots
    g = p.groups[4][1]
    p.groups[4][1] = synth.Spline(-0.5, 0.9, np.interp(np.linspace(-0.5, 0.9, 8), np.linspace(-1, 1, 8), g.y),
                                  g.grad.copy())
    _write("meam2_edge", p, cells, embed_extrap=1)

    # 5. isolated atoms: a sparse cell where some atoms have no neighbours,
    #    and a one-atom cell whose only neighbours are its own images
    lat = np.eye(3) * 12.0
    pos = np.array([[0.0, 0.0, 0.0], [2.6, 0.0, 0.0], [6.0, 6.0, 6.0], [9.0, 2.0, 5.0]])
    c1 = synth.Cell(lattice=lat, types=np.zeros(4, dtype=np.int64), pos=pos, force0=np.zeros((4, 3)))
    c2 = synth.Cell(lattice=np.diag([2.9, 3.1, 3.3]), types=np.zeros(1, dtype=np.int64),
                    pos=np.array([[0.1, 0.2, 0.3]]), force0=np.zeros((1, 3)))
    cells = [c1, c2]
    _targets(cells, 5)
    pot = synth.teacher_potential("meam/spline", 1, 4.5, seed=11)
    _write("meam_sparse", pot, cells, fd=True)
    pot = synth.teacher_potential("eam/spline", 1, 5.0, seed=12)
    _write("eam_sparse", pot, cells)


if __name__ == "__main__":
    import sys
    if "--powell" in sys.argv:
        powell_goldens()
        sys.exit(0)
    if "--quintic-styles" in sys.argv:
        quintic_styles_goldens()
        rescale_goldens(Q5B_CASES)
        data_goldens(Q5B_CASES)
        sys.exit(0)
    if "--grad10" in sys.argv:
        grad10_goldens()
        sys.exit(0)
    if "--jmeam" in sys.argv:
        jmeam_goldens()
        rescale_goldens(JMEAM_CASES)
        data_goldens(JMEAM_CASES)
        sys.exit(0)
    if "--quintic" in sys.argv:
        quintic_goldens()
        rescale_goldens(Q5_CASES)
        data_goldens(Q5_CASES)
        sys.exit(0)
    if "--pair" in sys.argv:
        pair_goldens()
        rescale_goldens(["pair_bcc1", "pair_mix2"])
        data_goldens(["pair_bcc1", "pair_mix2"])
        sys.exit(0)
    if "--gmeam" in sys.argv:
        gmeam_goldens()
    elif "--rescale-only" not in sys.argv and "--data-only" not in sys.argv:
        main()
    if "--data-only" not in sys.argv:
        rescale_goldens()
    data_goldens()
