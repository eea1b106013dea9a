"""Seeded synthetic databases and potentials in the reference file formats.

No public dataset is involved: every workload is generated here from a seed.
The generation rules follow the five workloads the evaluator is measured on:

  eam54    plain single-species spline EAM: 20 periodic 3x3x3 bcc supercells
           (54 atoms), lattice constant U[3.1, 3.4] A, jitter N(0, 0.08 A);
           phi and rho 10 knots on [1.8, 5.0], U 8 knots on [-1, 1].
  meam200  single-species spline MEAM: 200 cells, atom count U{32..250};
           50 % bcc, 25 % fcc or hcp strained U[-3 %, 3 %], 25 % liquid-like
           at 0.06 /A^3 with minimum distance 1.9 A; jitter N(0, 0.08 A).
           phi, rho, f 10 knots on [1.8, 4.5]; U and g 8 knots on [-1, 1].
  meam500  as meam200 with 500 cells, atom count log-uniform in [16, 512].
  meam2k   two-species MEAM: 2000 cells, atom count log-uniform [8, 1024],
           species 50/50, radial functions on [1.8, 5.5]; 12 splines,
           136 coefficients.

Teacher functions (knot values plus seeded N(0, 0.02), end slopes from the
analytic derivative): Morse phi (D=0.4 eV, a=1.4/A, r0=2.8 A),
rho = exp(-1.5(r-2.5)), U = -sqrt(n+1.1), f = exp(-(r-2.5)),
g = 1 + 0.3 cos^2.  Targets are the teacher's energy per atom, forces and
stress plus N(0, 1e-3 eV), N(0, 0.01 eV/A) and N(0, 0.01 GPa) noise; stress
is written in eV/A^3 (the reference applies no unit conversion).

File formats (written by write_pot / write_config / write_param) are the
reference's: potential file src/pot_list.cpp:101-142 + src/spline3eq.cpp:54-106,
configuration file src/cell.cpp:39-136, parameter file src/input.h:47-77.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Callable, List, Optional, Sequence

import numpy as np

GPA_PER_EV_A3 = 160.2177

# ----------------------------------------------------------------------------
# potential description
# ----------------------------------------------------------------------------


@dataclasses.dataclass
class Spline:
    """One equidistant spline: cubic (#B spline3eq block) or, with grad2 set
    (the y'' at the ends), quintic (#B spline5eq)."""

    left: float
    right: float
    y: np.ndarray                      # knot values
    grad: np.ndarray                   # end slopes [left, right]
    bc: Sequence[int] = (0, 0)         # -1 natural, 0 free slope, 1 fixed slope
    fixed: Optional[np.ndarray] = None  # per-knot 1 = fixed
    grad2: Optional[np.ndarray] = None  # spline5eq: y'' at the ends

    @property
    def nknots(self) -> int:
        return len(self.y)

    def copy(self) -> "Spline":
        return Spline(self.left, self.right, self.y.copy(), self.grad.copy(), tuple(self.bc),
                      None if self.fixed is None else self.fixed.copy(),
                      None if self.grad2 is None else self.grad2.copy())


@dataclasses.dataclass
class PotSpec:
    """A potential file: style, number of types, splines per function group."""

    style: str                  # "eam/spline" or "meam/spline"
    ntypes: int
    groups: List[List[Spline]]  # MEAM: phi, rho, U, f, g ; EAM: phi, rho, U

    def copy(self) -> "PotSpec":
        return PotSpec(self.style, self.ntypes, [[s.copy() for s in g] for g in self.groups])


def _spline_from_fn(fn, dfn, left, right, n, rng, noise=0.02):
    x = np.linspace(left, right, n)
    y = fn(x) + rng.normal(0.0, noise, n)
    return Spline(left, right, y, np.array([dfn(left), dfn(right)], dtype=np.float64))


def _morse(r):
    return 0.4 * (np.exp(-2 * 1.4 * (r - 2.8)) - 2 * np.exp(-1.4 * (r - 2.8)))


def _dmorse(r):
    return 0.4 * (-2 * 1.4 * np.exp(-2 * 1.4 * (r - 2.8)) + 2 * 1.4 * np.exp(-1.4 * (r - 2.8)))


TEACHER = {
    "phi": (_morse, _dmorse),
    "rho": (lambda r: np.exp(-1.5 * (r - 2.5)), lambda r: -1.5 * np.exp(-1.5 * (r - 2.5))),
    "U": (lambda n: -np.sqrt(n + 1.1), lambda n: -0.5 / np.sqrt(n + 1.1)),
    "f": (lambda r: np.exp(-(r - 2.5)), lambda r: -np.exp(-(r - 2.5))),
    "g": (lambda c: 1.0 + 0.3 * c * c, lambda c: 0.6 * c),
    # JMEAM's direct three-body terms p_ij p_ik q_i(cos) (and p2, q2)
    "p": (lambda r: np.exp(-1.2 * (r - 2.5)), lambda r: -1.2 * np.exp(-1.2 * (r - 2.5))),
    "q": (lambda c: 0.05 * (c + 0.3) ** 2, lambda c: 0.1 * (c + 0.3)),
    "p2": (lambda r: np.exp(-0.8 * (r - 2.5)), lambda r: -0.8 * np.exp(-0.8 * (r - 2.5))),
    "q2": (lambda c: -0.02 * (1.0 + c), lambda c: -0.02 + 0.0 * c),
}


def n_alloy(kind: str, ntypes: int, style: str = "meam/spline") -> int:
    """Number of alloy splines in a function group (src/pot_fns.cpp:403-433);
    gmeam/spline's g is Triplet_i_jk, n n (n + 1) / 2 splines (pot_gmeam.cpp:31-36)."""
    if kind in ("phi", "f", "p", "p2"):
        return ntypes * (ntypes + 1) // 2
    if kind == "g" and style == "gmeam/spline":
        return ntypes * ntypes * (ntypes + 1) // 2
    return ntypes


def teacher_potential(style: str, ntypes: int, rcut: float, seed: int) -> PotSpec:
    rng = np.random.default_rng(seed)
    kinds = (["phi"] if style == "pair/spline" else
             ["phi", "rho", "U"] + (["f", "g"] if style in ("meam/spline", "gmeam/spline", "jmeam/spline",
                                                           "jmeam2/spline") else []))
    kinds += {"jmeam/spline": ["p", "q"], "jmeam2/spline": ["p", "q", "p2", "q2"]}.get(style, [])
    groups = []
    for kind in kinds:
        fn, dfn = TEACHER[kind]
        if kind in ("U", "g", "q", "q2"):
            left, right, n = -1.0, 1.0, 8
        else:
            left, right, n = 1.8, rcut, 10
        groups.append([_spline_from_fn(fn, dfn, left, right, n, rng) for _ in range(n_alloy(kind, ntypes, style))])
    return PotSpec(style, ntypes, groups)


# ----------------------------------------------------------------------------
# configuration database
# ----------------------------------------------------------------------------


@dataclasses.dataclass
class Cell:
    lattice: np.ndarray          # rows are the #X, #Y, #Z box vectors
    types: np.ndarray            # (n,) int
    pos: np.ndarray              # (n, 3)
    force0: np.ndarray           # (n, 3)
    energy0: float = 0.0         # per atom
    stress0: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(6))
    weight: float = 1.0
    eweight: float = 1.0
    sweight: float = 1.0

    @property
    def natoms(self) -> int:
        return len(self.types)


def _bcc_basis():
    return np.array([[0, 0, 0], [0.5, 0.5, 0.5]])


def _fcc_basis():
    return np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])


def _supercell_dims(n_target, per_cell):
    """Smallest near-cubic n1*n2*n3 supercell holding at least n_target atoms."""
    best = None
    m = 1
    while True:
        for n1 in range(1, m + 1):
            for n2 in range(n1, m + 1):
                n3 = max(n2, int(math.ceil(n_target / (per_cell * n1 * n2))))
                cnt = per_cell * n1 * n2 * n3
                key = (cnt, n3 - n1)
                if best is None or key < best[0]:
                    best = (key, (n1, n2, n3))
        if best is not None and m ** 3 * per_cell >= n_target:
            return best[1]
        m += 1


def _crystal(kind, n_atoms, a_bcc, rng):
    rho = 2.0 / a_bcc ** 3
    if kind == "bcc":
        basis, a, cell = _bcc_basis(), a_bcc, None
        cell = np.eye(3) * a
    elif kind == "fcc":
        basis = _fcc_basis()
        a = (4.0 / rho) ** (1.0 / 3.0)
        cell = np.eye(3) * a
    else:  # hcp in its orthorhombic 4-atom cell
        ca = math.sqrt(8.0 / 3.0)
        a = (4.0 / (rho * math.sqrt(3.0) * ca)) ** (1.0 / 3.0)
        cell = np.diag([a, math.sqrt(3.0) * a, ca * a])
        basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 1.0 / 6.0, 0.5], [0.0, 2.0 / 3.0, 0.5]])
    per = len(basis)
    n1, n2, n3 = _supercell_dims(n_atoms, per)
    grid = np.array([[i, j, k] for i in range(n1) for j in range(n2) for k in range(n3)], dtype=np.float64)
    frac = (grid[:, None, :] + basis[None, :, :]).reshape(-1, 3) / np.array([n1, n2, n3])
    lattice = cell * np.array([n1, n2, n3])[:, None]
    keep = np.sort(rng.choice(len(frac), size=n_atoms, replace=False))  # vacancies down to n_atoms
    return lattice, frac[keep]


def _liquid(n_atoms, density, dmin, rng):
    L = (n_atoms / density) ** (1.0 / 3.0)
    lattice = np.eye(3) * L
    pts = np.empty((n_atoms, 3))
    m = 0
    tries = 0
    while m < n_atoms:
        cand = rng.random((64, 3)) * L
        for p in cand:
            d = pts[:m] - p
            d -= L * np.round(d / L)
            if m == 0 or np.einsum("ij,ij->i", d, d).min() >= dmin * dmin:
                pts[m] = p
                m += 1
                if m == n_atoms:
                    break
        tries += 64
        if tries > 5000 * n_atoms:
            raise RuntimeError("liquid packing failed")
    return lattice, pts / L


def _short_atoms(lattice, cart, floor):
    """Atoms with a neighbour (periodic images included) closer than floor."""
    from scipy.spatial import cKDTree
    n = len(cart)
    shifts = np.array([[i, j, k] for i in (-1, 0, 1) for j in (-1, 0, 1) for k in (-1, 0, 1)], dtype=np.float64)
    img = (cart[None, :, :] + (shifts @ lattice)[:, None, :]).reshape(-1, 3)
    cnt = cKDTree(img).query_ball_point(cart, floor, return_length=True)
    return np.nonzero(cnt > 1)[0]  # the atom itself is always within reach


def _jitter(lattice, frac, sigma, rng, floor):
    """Gaussian displacements; atoms that end up closer than floor to a
    neighbour are re-drawn (kept at the lattice site after 50 tries)."""
    base = frac @ lattice
    cart = base + rng.normal(0.0, sigma, base.shape)
    for _ in range(50):
        bad = _short_atoms(lattice, cart, floor)
        if bad.size == 0:
            return cart
        cart[bad] = base[bad] + rng.normal(0.0, sigma, (bad.size, 3))
    bad = _short_atoms(lattice, cart, floor)
    cart[bad] = base[bad]
    return cart


def make_cells(n_cells, count_rule, rng, ntypes=1, mix="meam", dmin_floor=1.85):
    """Generate cell geometries (no targets yet).

    count_rule(rng) -> atom count; mix "bcc" = all bcc (eam54), "meam" = the
    50/25/25 bcc / strained fcc-hcp / liquid mixture.
    """
    cells = []
    for c in range(n_cells):
        n = int(count_rule(rng))
        a_bcc = rng.uniform(3.1, 3.4)
        u = rng.random()
        if mix == "bcc" or u < 0.5:
            lattice, frac = _crystal("bcc", n, a_bcc, rng)
        elif u < 0.75:
            lattice, frac = _crystal("fcc" if rng.random() < 0.5 else "hcp", n, a_bcc, rng)
            eps = rng.uniform(-0.03, 0.03, (3, 3))
            eps = 0.5 * (eps + eps.T)
            lattice = lattice @ (np.eye(3) + eps)
        else:
            lattice, frac = _liquid(n, 0.06, 1.9, rng)
        pos = _jitter(lattice, frac, 0.08, rng, dmin_floor)
        types = rng.integers(0, ntypes, n) if ntypes > 1 else np.zeros(n, dtype=np.int64)
        cells.append(Cell(lattice=lattice, types=types.astype(np.int64), pos=pos, force0=np.zeros((n, 3))))
    return cells


def add_targets(cells, energy, stress, forces, rng):
    """Set targets = teacher values + noise (energy per atom, stress eV/A^3)."""
    for i, c in enumerate(cells):
        c.energy0 = float(energy[i] + rng.normal(0.0, 1e-3))
        c.stress0 = np.asarray(stress[i], dtype=np.float64) + rng.normal(0.0, 0.01, 6) / GPA_PER_EV_A3
        c.force0 = np.asarray(forces[i], dtype=np.float64) + rng.normal(0.0, 0.01, (c.natoms, 3))


def set_teacher_targets(cells, energy, stress, forces, seed: int):
    """Targets = teacher outputs (energy per atom [ncells], stress [ncells, 6]
    in eV/A^3, forces [natoms, 3]) + the noise of add_targets, seeded."""
    a0 = np.cumsum([0] + [c.natoms for c in cells])
    forces = np.asarray(forces, dtype=np.float64).reshape(-1, 3)
    stress = np.asarray(stress, dtype=np.float64).reshape(-1, 6)
    add_targets(cells, np.asarray(energy, dtype=np.float64).ravel(), stress,
                [forces[a0[i]:a0[i + 1]] for i in range(len(cells))], np.random.default_rng(seed))


# ----------------------------------------------------------------------------
# workloads
# ----------------------------------------------------------------------------

WORKLOADS = {
    # name: (style, ntypes, rcut, ncells, count rule, mix, seeds)
    "eam54": ("eam/spline", 1, 5.0, 20, lambda r: 54, "bcc"),
    "meam200": ("meam/spline", 1, 4.5, 200, lambda r: r.integers(32, 251), "meam"),
    "meam500": ("meam/spline", 1, 4.5, 500, lambda r: int(round(math.exp(r.uniform(math.log(16), math.log(512))))), "meam"),
    "meam2k": ("meam/spline", 2, 5.5, 2000, lambda r: int(round(math.exp(r.uniform(math.log(8), math.log(1024))))), "meam"),
}


def make_workload(name: str, seed: int = 0, ncells: Optional[int] = None):
    """Return (teacher PotSpec, cells without targets) for a named workload."""
    style, ntypes, rcut, n_cells, rule, mix = WORKLOADS[name]
    if ncells is not None:
        n_cells = ncells
    pot = teacher_potential(style, ntypes, rcut, seed=1000 + seed)
    rng = np.random.default_rng(2000 + seed)
    cells = make_cells(n_cells, rule, rng, ntypes=ntypes, mix=mix)
    return pot, cells


# The gradient check of the single-species MEAM workload (200 cells): the
# teacher as generated or its in-range variant, targets = teacher outputs +
# noise (seed below), 10 parameter points = teacher + N(0, sigma).
GRAD10 = {"workload": "meam200", "seed": 0, "target_seed": 3100, "point_seed": 3200, "npoints": 10,
          "sigma": {"raw": 0.05, "inrange": 0.005}}


def grad10_workload(variant: str):
    """(teacher PotSpec, cells without targets) of the gradient check;
    variant "raw" (the teacher as generated) or "inrange"."""
    pot, cells = make_workload(GRAD10["workload"], seed=GRAD10["seed"])
    return (in_range_variant(pot) if variant == "inrange" else pot), cells


def quintic_variant(pot: PotSpec, seed: int = 0, groups=None) -> PotSpec:
    """The same knots as spline5eq splines (Spline5Eq, spline5eq.cpp), with
    end second derivatives from the knots' second differences.  `groups`
    (function group indices, default all) picks the groups made quintic; the
    others keep spline3eq (a mixed-basis potential)."""
    p = pot.copy()
    rng = np.random.default_rng(seed)
    for gi, group in enumerate(p.groups):
        if groups is not None and gi not in groups:
            continue
        for s in group:
            h = (s.right - s.left) / (s.nknots - 1)
            d2 = np.diff(s.y, 2) / (h * h)
            s.grad2 = np.array([d2[0], d2[-1]]) * (1.0 + 0.05 * rng.normal(size=2))
    return p


def in_range_variant(pot: PotSpec, rho_scale: float = 0.01, g_scale: float = 0.0025) -> PotSpec:
    """Supplementary variant (labelled as such wherever used): the teacher's
    rho and g scaled so that every embedding density of the MEAM workloads
    falls inside U's knot range [-1, 1].  With the teacher as generated the
    densities lie far outside it (20-150), the objective is almost all
    density punishment and U's interior knots do not affect it."""
    p = pot.copy()
    for s in p.groups[1]:
        s.y = s.y * rho_scale
        s.grad = s.grad * rho_scale
    if len(p.groups) > 4:
        for s in p.groups[4]:
            s.y = s.y * g_scale
            s.grad = s.grad * g_scale
    return p


def perturbed(pot_coeffs: np.ndarray, n: int, sigma: float, seed: int) -> np.ndarray:
    """n candidate parameter vectors: coeffs + N(0, sigma) (GA population)."""
    rng = np.random.default_rng(seed)
    return pot_coeffs[None, :] + rng.normal(0.0, sigma, (n, pot_coeffs.size))


# ----------------------------------------------------------------------------
# writers (reference formats)
# ----------------------------------------------------------------------------


def _f(x):
    return "%.17g" % float(x)


def write_pot(path: str, pot: PotSpec, comment: str = "synthetic teacher potential"):
    lines = [comment, "#T %s %d" % (pot.style, pot.ntypes), "#P"]
    for group in pot.groups:
        for s in group:
            lines.append("#B spline5eq" if s.grad2 is not None else "#B spline3eq")
            lines.append("%s %s %d" % (_f(s.left), _f(s.right), s.nknots))
            lines.append("%d %d" % tuple(s.bc))
            lines.append("%s %s" % (_f(s.grad[0]), _f(s.grad[1])))
            if s.grad2 is not None:
                lines.append("%s %s" % (_f(s.grad2[0]), _f(s.grad2[1])))
            fixed = s.fixed if s.fixed is not None else np.zeros(s.nknots, dtype=int)
            for k in range(s.nknots):
                lines.append("%d %s" % (int(fixed[k]), _f(s.y[k])))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def write_config(path: str, cells: Sequence[Cell]):
    out = []
    for c in cells:
        out.append("#N %d 1" % c.natoms)
        for lab, v in zip(("#X", "#Y", "#Z"), c.lattice):
            out.append("%s %s %s %s" % (lab, _f(v[0]), _f(v[1]), _f(v[2])))
        out.append("#E %s" % _f(c.energy0))
        out.append("#S " + " ".join(_f(v) for v in c.stress0))
        out.append("#W %s" % _f(c.weight))
        if c.eweight != 1.0:
            out.append("#EW %s" % _f(c.eweight))
        if c.sweight != 1.0:
            out.append("#SW %s" % _f(c.sweight))
        out.append("#F")
        for t, p, f in zip(c.types, c.pos, c.force0):
            out.append("%d %s %s %s %s %s %s" % (int(t), _f(p[0]), _f(p[1]), _f(p[2]), _f(f[0]), _f(f[1]), _f(f[2])))
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")


def write_param(path: str, config: str, startpot: str, energy_weight=1.0, stress_weight=1.0,
                rescale=0, embed_extrap=0, extra: Optional[dict] = None):
    d = os.path.dirname(os.path.abspath(path))
    lines = [
        "config %s" % config,
        "startpot %s" % startpot,
        "tempfile %s" % os.path.join(d, "tempfile"),
        "endpot %s" % os.path.join(d, "endpot"),
        "energy_weight %s" % _f(energy_weight),
        "stress_weight %s" % _f(stress_weight),
        "rescale %d" % rescale,
    ]
    if embed_extrap:
        lines.append("embed_extrap %d" % embed_extrap)
    for k, v in (extra or {}).items():
        lines.append("%s %s" % (k, v))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def write_case(dirname: str, pot: PotSpec, cells: Sequence[Cell], **param_kw) -> str:
    """Write pot/config/param files for a case; returns the param path."""
    os.makedirs(dirname, exist_ok=True)
    pot_path = os.path.join(dirname, "start.pot")
    conf_path = os.path.join(dirname, "db.conf")
    par_path = os.path.join(dirname, "param")
    write_pot(pot_path, pot)
    write_config(conf_path, cells)
    write_param(par_path, conf_path, pot_path, **param_kw)
    return par_path
