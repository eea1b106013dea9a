"""Host-side mirror of the reference's Potential interface over the C ABI.

The reference's optimizers see one object, Potential (src/potential.h:35-109):

    double compute(const Comm&, ErrorVec* = nullptr)     potential.h:67
    int get_ncoeff(); double& coeff(int); void modify_coeff(int, double, double)
    void set_dir(dir, x); double compute_dir(comm, ErrorVec*, dir, x)
    Potential* clone(); double get_error(); write_pot / write_data

`Potential` below keeps those names, argument meanings and error behaviour
(compute never fails on numbers; NaN propagates), and evaluates through the
CUDA evaluator.  `Evaluator` is the batched interface (many candidate
parameter vectors per call) that the reference has no counterpart for.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import MZ_FP64, MZ_MIXED, MzError, check, lib, ptr

__all__ = ["PotentialFile", "Database", "Evaluator", "Potential", "read_param", "from_param_file",
           "MZ_FP64", "MZ_MIXED", "MzError"]


def _release(obj, fn: str) -> None:
    """Free a handle; silent during interpreter shutdown."""
    h = getattr(obj, "_h", None)
    obj._h = None
    if h and _lib._lib is not None:
        try:
            getattr(_lib._lib, fn)(h)
        except Exception:
            pass


def style_npen(style: int, ntypes: int) -> int:
    """Punishment entries after the per-cell constraints: MEAM the f
    magnitude, GMEAM one per f spline, JMEAM / JMEAM2 f and p (p2)
    magnitudes, EAM U'(mid) per type, pair/spline none."""
    return {_lib.MZ_STYLE_MEAM_SPLINE: 1, _lib.MZ_STYLE_GMEAM_SPLINE: ntypes * (ntypes + 1) // 2,
            _lib.MZ_STYLE_JMEAM_SPLINE: 2, _lib.MZ_STYLE_JMEAM2_SPLINE: 3, _lib.MZ_STYLE_PAIR_SPLINE: 0}.get(
        style, ntypes)


def read_param(path: str) -> Dict[str, List[str]]:
    """Parameter file as key -> tokens (Input::parse, src/input.h:47-77: the
    first line whose first token is the key wins; blank lines are dropped)."""
    out: Dict[str, List[str]] = {}
    with open(path) as fh:
        for line in fh:
            toks = line.replace("\r", "").split()
            if toks and toks[0] not in out:
                out[toks[0]] = toks[1:]
    return out


class PotentialFile:
    """A potential file (#T/#P/#B spline3eq blocks) and its coefficient layout."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle

    @classmethod
    def read(cls, path: str) -> "PotentialFile":
        h = C.c_void_p()
        check(lib().mz_pot_read(path.encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def parse(cls, text: str) -> "PotentialFile":
        h = C.c_void_p()
        check(lib().mz_pot_parse(text.encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def from_spec(cls, spec) -> "PotentialFile":
        """From a synth.PotSpec."""
        import tempfile
        from . import synth
        with tempfile.TemporaryDirectory() as d:
            p = os.path.join(d, "pot")
            synth.write_pot(p, spec)
            return cls.read(p)

    def __del__(self):
        _release(self, "mz_pot_free")

    @property
    def handle(self):
        return self._h

    def info(self):
        st, nt, ns = C.c_int(), C.c_int(), C.c_int()
        check(lib().mz_pot_info(self._h, C.byref(st), C.byref(nt), C.byref(ns)))
        return st.value, nt.value, ns.value

    @property
    def style(self) -> int:
        return self.info()[0]

    @property
    def ntypes(self) -> int:
        return self.info()[1]

    @property
    def nsplines(self) -> int:
        return self.info()[2]

    @property
    def ncoeff(self) -> int:
        n = C.c_int()
        check(lib().mz_pot_ncoeff(self._h, C.byref(n)))
        return n.value

    def coeffs(self) -> np.ndarray:
        x = np.zeros(self.ncoeff)
        check(lib().mz_pot_get_coeffs(self._h, ptr(x)))
        return x

    def set_coeffs(self, x) -> None:
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.size != self.ncoeff:
            raise ValueError("expected %d coefficients" % self.ncoeff)
        check(lib().mz_pot_set_coeffs(self._h, ptr(x)))

    def copy(self) -> "PotentialFile":
        """An independent copy (Potential::clone, potential.h:43)."""
        h = C.c_void_p()
        check(lib().mz_pot_clone(self._h, C.byref(h)))
        return PotentialFile(h)

    def rescale(self, db: "Database", densities, flag: int = 1):
        """Potential::rescale in place (PotMEAM::rescale pot_meam.cpp:281-375,
        PotEAM::rescale pot_eam.cpp:257-389) from the per-atom densities of
        the current coefficients.  Returns (rescaled, a, b): the reference's
        return value, the embedding scale factor and the MEAM f scale (0 when
        not applied); the JMEAM p (p2) scales (pot_jmeam.cpp:375-401) are
        left in self.jmeam_factors.  Evaluators built before must be
        re-created."""
        d = np.ascontiguousarray(densities, dtype=np.float64)
        if d.size != db.stats()["natoms"]:
            raise ValueError("one density per atom expected")
        r = C.c_int()
        f = np.zeros(4)
        check(lib().mz_pot_rescale(self._h, db.handle, ptr(d), int(flag), C.byref(r), ptr(f)))
        self.jmeam_factors = (float(f[2]), float(f[3]))
        return bool(r.value), float(f[0]), float(f[1])

    def write(self, path: str) -> None:
        check(lib().mz_pot_write(self._h, path.encode()))

    def spline(self, s: int) -> dict:
        v = _lib.SplineView()
        check(lib().mz_pot_get_spline(self._h, s, C.byref(v)))
        n = v.nknots
        return dict(group=v.group, alloy=v.alloy, nknots=n, left=v.left, right=v.right,
                    nat=(v.nat[0], v.nat[1]), grad_fixed=(v.grad_fixed[0], v.grad_fixed[1]),
                    grad=np.array([v.grad[0], v.grad[1]]),
                    y_fixed=_lib.as_array(v.y_fixed, n, np.int32), y=_lib.as_array(v.y, n, np.float64),
                    x=_lib.as_array(v.x, n, np.float64), step=v.step, quintic=v.quintic,
                    grad2=np.array([v.grad2[0], v.grad2[1]]))

    def spline_eval(self, s: int, x: float):
        val, grad = C.c_double(), C.c_double()
        check(lib().mz_pot_spline_eval(self._h, s, float(x), C.byref(val), C.byref(grad)))
        return val.value, grad.value


class Database:
    """Configuration database with its neighbour lists, built for a potential."""

    def __init__(self, handle: C.c_void_p, pot: PotentialFile):
        self._h = handle
        self.pot = pot

    @classmethod
    def read(cls, config_path: str, pot: PotentialFile, device: Optional[int] = None) -> "Database":
        """Read a configuration file; with `device`, the neighbour lists are
        built on that GPU (identical result)."""
        h = C.c_void_p()
        if device is None:
            check(lib().mz_db_read(config_path.encode(), pot.handle, C.byref(h)))
        else:
            check(lib().mz_db_read_device(config_path.encode(), pot.handle, int(device), C.byref(h)))
        return cls(h, pot)

    @classmethod
    def from_cells(cls, cells: Sequence, pot: PotentialFile, device: Optional[int] = None) -> "Database":
        """From a list of synth.Cell (lattice rows, types, positions, targets);
        with `device`, the neighbour lists are built on that GPU."""
        nat = np.array([c.natoms for c in cells], dtype=np.int32)
        lat = np.ascontiguousarray(np.stack([np.asarray(c.lattice, dtype=np.float64) for c in cells]))
        e0 = np.array([c.energy0 for c in cells], dtype=np.float64)
        s0 = np.ascontiguousarray(np.stack([np.asarray(c.stress0, dtype=np.float64) for c in cells]))
        w = np.array([c.weight for c in cells], dtype=np.float64)
        ew = np.array([c.eweight for c in cells], dtype=np.float64)
        sw = np.array([c.sweight for c in cells], dtype=np.float64)
        types = np.ascontiguousarray(np.concatenate([np.asarray(c.types) for c in cells]).astype(np.int32))
        pos = np.ascontiguousarray(np.concatenate([np.asarray(c.pos, dtype=np.float64) for c in cells]))
        f0 = np.ascontiguousarray(np.concatenate([np.asarray(c.force0, dtype=np.float64) for c in cells]))
        d = _lib.CellsDesc()
        d.ncells = len(cells)
        d.natoms = int(nat.sum())
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        d.cell_natoms = nat.ctypes.data_as(ip)
        d.cell_lattice = lat.ctypes.data_as(dp)
        d.cell_energy0 = e0.ctypes.data_as(dp)
        d.cell_stress0 = s0.ctypes.data_as(dp)
        d.cell_weight = w.ctypes.data_as(dp)
        d.cell_eweight = ew.ctypes.data_as(dp)
        d.cell_sweight = sw.ctypes.data_as(dp)
        d.atom_type = types.ctypes.data_as(ip)
        d.atom_pos = pos.ctypes.data_as(dp)
        d.atom_force0 = f0.ctypes.data_as(dp)
        h = C.c_void_p()
        if device is None:
            check(lib().mz_db_build(C.byref(d), pot.handle, C.byref(h)))
        else:
            check(lib().mz_db_build_device(C.byref(d), pot.handle, int(device), C.byref(h)))
        return cls(h, pot)

    def __del__(self):
        _release(self, "mz_db_free")

    @property
    def handle(self):
        return self._h

    def stats(self) -> dict:
        s = _lib.DbStats()
        check(lib().mz_db_info(self._h, C.byref(s)))
        return dict(ncells=s.ncells, natoms=s.natoms, npairs=s.npairs, ntriplets=s.ntriplets,
                    max_row=s.max_row, esize_cells=s.esize)

    def view(self) -> dict:
        """Copies of the built arrays (CSR rows in the reference's pair order)."""
        v = _lib.DbView()
        check(lib().mz_db_get_view(self._h, C.byref(v)))
        N, NC, Np, nf = v.natoms, v.ncells, v.npairs, v.nfun
        a = _lib.as_array
        return dict(
            ncells=NC, natoms=N, npairs=Np,
            cell_atom0=a(v.cell_atom0, NC + 1, np.int32), cell_vol=a(v.cell_vol, NC, np.float64),
            cell_weight=a(v.cell_weight, NC, np.float64), cell_eweight=a(v.cell_eweight, NC, np.float64),
            cell_sweight=a(v.cell_sweight, NC, np.float64), cell_energy0=a(v.cell_energy0, NC, np.float64),
            cell_stress0=a(v.cell_stress0, 6 * NC, np.float64), cell_lattice=a(v.cell_lattice, 9 * NC, np.float64),
            atom_type=a(v.atom_type, N, np.int32), atom_cell=a(v.atom_cell, N, np.int32),
            atom_pos=a(v.atom_pos, 3 * N, np.float64), atom_force0=a(v.atom_force0, 3 * N, np.float64),
            pair_off=a(v.pair_off, N + 1, np.int64), pair_nbr=a(v.pair_nbr, Np, np.int32),
            pair_r=a(v.pair_r, Np, np.float64), pair_u=a(v.pair_u, 3 * Np, np.float64),
            pair_knot=a(v.pair_knot, nf * Np, np.int8), pair_shift=a(v.pair_shift, nf * Np, np.float64), nfun=nf,
            in_off=a(v.in_off, N + 1, np.int64), in_slot=a(v.in_slot, Np, np.int64),
        )

    def set_targets(self, energy0=None, stress0=None, force0=None) -> None:
        arrs = [None if x is None else np.ascontiguousarray(x, dtype=np.float64) for x in (energy0, stress0, force0)]
        check(lib().mz_db_set_targets(self._h, *[ptr(x) for x in arrs]))


class Evaluator:
    """Device-resident evaluator of a database and a potential's structure.

    Candidates are coefficient vectors in the reference's Potential::coeff
    order; many of them are evaluated per launch."""

    def __init__(self, db: Database, pot: PotentialFile, energy_weight=0.0, stress_weight=0.0,
                 embed_extrap=0, device=0, max_candidates=1, omit_punishments=False):
        s = _lib.Settings(float(energy_weight), float(stress_weight), int(embed_extrap), int(device),
                          int(max_candidates), 1 if omit_punishments else 0)
        h = C.c_void_p()
        check(lib().mz_create(db.handle, pot.handle, C.byref(s), C.byref(h)))
        self._h = h
        self.db = db
        self.pot = pot
        self.energy_weight, self.stress_weight, self.embed_extrap = float(energy_weight), float(stress_weight), int(embed_extrap)
        self.device, self.max_candidates, self.omit_punishments = int(device), int(max_candidates), bool(omit_punishments)
        st = db.stats()
        self.natoms, self.ncells = st["natoms"], st["ncells"]
        self.ncoeff = pot.ncoeff
        self.npen = style_npen(pot.style, pot.ntypes)
        self.esize = st["esize_cells"] + self.npen

    def __del__(self):
        _release(self, "mz_destroy")

    @property
    def handle(self):
        return self._h

    def objective(self, params, precision=MZ_FP64, errvec=False, forces=False, energy=False, stress=False):
        """Objective of each row of params; optional per-candidate outputs."""
        x = np.ascontiguousarray(np.atleast_2d(params), dtype=np.float64)
        n = x.shape[0]
        if x.shape[1] != self.ncoeff:
            raise ValueError("expected %d coefficients per candidate" % self.ncoeff)
        obj = np.zeros(n)
        ev = np.zeros((n, self.esize)) if errvec else None
        fo = np.zeros((n, self.natoms, 3)) if forces else None
        en = np.zeros((n, self.ncells)) if energy else None
        sg = np.zeros((n, self.ncells, 6)) if stress else None
        check(lib().mz_objective(self._h, n, ptr(x), int(precision), ptr(obj), ptr(ev), ptr(fo), ptr(en), ptr(sg)))
        if not (errvec or forces or energy or stress):
            return obj
        out = dict(obj=obj)
        for k, v in (("errvec", ev), ("forces", fo), ("energy", en), ("stress", sg)):
            if v is not None:
                out[k] = v
        return out

    def objective_grad(self, params, precision=MZ_FP64):
        x = np.ascontiguousarray(np.atleast_2d(params), dtype=np.float64)
        n = x.shape[0]
        obj = np.zeros(n)
        g = np.zeros((n, self.ncoeff))
        check(lib().mz_objective_grad(self._h, n, ptr(x), int(precision), ptr(obj), ptr(g)))
        return obj, g

    def densities(self, params) -> np.ndarray:
        x = np.ascontiguousarray(params, dtype=np.float64)
        d = np.zeros(self.natoms)
        check(lib().mz_densities(self._h, ptr(x), ptr(d)))
        return d

    def tensor_core_forward(self) -> bool:
        """True when the mixed MEAM forward runs its triplet sums on the
        tensor cores (opt-in: MZ_TC=1 in the environment at construction)."""
        on = C.c_int()
        check(lib().mz_tensor_core_forward(self._h, C.byref(on)))
        return bool(on.value)

    def tuning(self, precision=MZ_MIXED, grad=True) -> dict:
        """The autotuner's launch variant for (precision, gradient): forward
        and adjoint pair slots per atom block, adjoint CTAs, forward and
        adjoint candidates per CTA (zeros before the first such call)."""
        c = np.zeros(5, dtype=np.int32)
        check(lib().mz_tuning(self._h, int(precision), 1 if grad else 0, ptr(c)))
        on = C.c_int()
        check(lib().mz_moment_path(self._h, int(precision), 1 if grad else 0, C.byref(on)))
        return dict(forward_block_slots=int(c[0]), adjoint_block_slots=int(c[1]), adjoint_ctas=int(c[2]),
                    forward_candidates_per_cta=int(c[3]), adjoint_candidates_per_cta=int(c[4]),
                    triplet_moments=bool(on.value), moment_forward_tensor_cores=on.value >= 2,
                    moment_adjoint_tensor_cores=on.value == 3)

    def moment_path(self, precision=MZ_MIXED, grad=True) -> int:
        """Non-zero when the tuned (precision, gradient) launches run the
        triplet-moment path (mixed-precision meam/spline): 1 with the
        contractions on the CUDA cores, 2 with the forward one on the tensor
        cores, 3 with both."""
        on = C.c_int()
        check(lib().mz_moment_path(self._h, int(precision), 1 if grad else 0, C.byref(on)))
        return int(on.value)

    def launches(self) -> int:
        n = C.c_int64()
        check(lib().mz_launch_count(self._h, C.byref(n)))
        return n.value

    # --- device-pointer interface (torch CUDA tensors), enqueued on stream()
    def stream(self) -> int:
        """The context's CUDA stream (cudaStream_t as an integer)."""
        return lib().mz_stream(self._h) or 0

    @staticmethod
    def _after_torch(t) -> None:
        """The evaluator runs on its own stream: finish the work torch queued
        on its current stream (e.g. the copy that produced `t`) first."""
        import torch
        torch.cuda.current_stream(t.device).synchronize()

    def objective_device(self, params, obj, precision=MZ_MIXED, errvec=None, forces=None) -> None:
        """params: (n, ncoeff) float64 CUDA tensor; obj: (n,) float64 CUDA tensor;
        optional errvec (n, esize) and forces (n, natoms, 3) CUDA tensors.
        Enqueued on stream(); call sync() before reading the outputs."""
        self._after_torch(params)
        n = params.shape[0]
        ev = None if errvec is None else C.c_void_p(errvec.data_ptr())
        fo = None if forces is None else C.c_void_p(forces.data_ptr())
        check(lib().mz_objective_device(self._h, n, C.c_void_p(params.data_ptr()), int(precision),
                                        C.c_void_p(obj.data_ptr()), ev, fo))

    def objective_grad_device(self, params, obj, grad, precision=MZ_MIXED) -> None:
        """As objective_device, with grad an (n, ncoeff) float64 CUDA tensor."""
        self._after_torch(params)
        n = params.shape[0]
        check(lib().mz_objective_grad_device(self._h, n, C.c_void_p(params.data_ptr()), int(precision),
                                             C.c_void_p(obj.data_ptr()), C.c_void_p(grad.data_ptr())))

    def gram_device(self, A, B, out) -> None:
        """out[i, j] = sum_k A[i, k] * B[j, k] in FP64 on this evaluator's
        stream (mz_gram_device): A (na, n), B (nb, n), out (na, nb) float64
        CUDA tensors with unit stride along k.  Call sync() before reading
        out."""
        for t in (A, B, out):
            if not t.is_cuda or t.dtype.itemsize != 8 or not t.dtype.is_floating_point:
                raise TypeError("gram_device takes float64 CUDA tensors")
        if A.dim() != 2 or B.dim() != 2 or A.stride(1) != 1 or B.stride(1) != 1 or not out.is_contiguous():
            raise ValueError("rows with unit stride and a contiguous output are required")
        if A.shape[1] != B.shape[1] or tuple(out.shape) != (A.shape[0], B.shape[0]):
            raise ValueError("shapes do not match")
        self._after_torch(A)
        check(lib().mz_gram_device(self._h, A.shape[0], C.c_void_p(A.data_ptr()), A.stride(0), B.shape[0],
                                   C.c_void_p(B.data_ptr()), B.stride(0), A.shape[1], C.c_void_p(out.data_ptr())))

    def sync(self) -> None:
        check(lib().mz_sync(self._h))

    def profile(self, on: bool = True) -> None:
        check(lib().mz_profile(self._h, 1 if on else 0))

    def kernel_times(self) -> dict:
        """{kernel name: (total ms, launches)} since the last call."""
        ms = np.zeros(_lib.MZ_NKERNELS)
        cnt = np.zeros(_lib.MZ_NKERNELS, dtype=np.int64)
        check(lib().mz_kernel_times(self._h, ptr(ms), ptr(cnt)))
        return {lib().mz_kernel_name(k).decode(): (float(ms[k]), int(cnt[k])) for k in range(_lib.MZ_NKERNELS)
                if cnt[k] > 0}


def alu_peak(device: int = 0, precision=MZ_MIXED) -> float:
    """Measured FMA throughput of the device in TFLOP/s (FP64 or FP32)."""
    t = C.c_double()
    check(lib().mz_alu_peak(int(device), int(precision), C.byref(t)))
    return t.value


class Potential:
    """The reference's Potential object, evaluated on the GPU.

    Shares one Evaluator between clones (the reference shares its Config)."""

    ncalls = 0  # Potential::ncalls_ (potential.cpp:30): objective evaluations

    def __init__(self, evaluator: Evaluator, coeffs: Optional[np.ndarray] = None, precision=MZ_FP64):
        self.ev = evaluator
        self.x = np.array(evaluator.pot.coeffs() if coeffs is None else coeffs, dtype=np.float64)
        self.precision = precision
        self.error_sum = 0.0

    # --- Potential::clone (potential.h:43)
    def clone(self) -> "Potential":
        p = Potential(self.ev, self.x.copy(), self.precision)
        p.error_sum = self.error_sum
        return p

    # --- parameter access (potential.h:59-61)
    def get_ncoeff(self) -> int:
        return self.x.size

    def coeff(self, i: int) -> float:
        return float(self.x[i])

    def set_coeff(self, i: int, v: float) -> None:
        self.x[i] = v

    def modify_coeff(self, idx: int, height: float, width: float) -> None:
        """Gaussian bump of knot values, or a shift of an end slope
        (Spline::modify_coeff, spline.cpp:120-149; potential.cpp:212-226)."""
        pot = self.ev.pot
        base = 0
        for s in range(pot.nsplines):
            sp = pot.spline(s)
            free = [k for k in range(sp["nknots"]) if not sp["y_fixed"][k]]
            ends = [e for e in range(2) if not sp["grad_fixed"][e] and not sp["nat"][e]]
            nco = len(free) + len(ends)
            if idx < base + nco:
                local = idx - base
                if local < len(free):
                    kk = free[local]
                    w = int(4 * width)
                    pos = {k: base + free.index(k) for k in free}
                    for i in range(-w, w + 1):
                        k = kk + i
                        if 0 <= k < sp["nknots"] and k in pos:
                            self.x[pos[k]] += 0.3989422804014326779 * np.exp(-i * i * 0.5 / (width * width)) * height
                else:
                    self.x[idx] += height
                return
            base += nco

    # --- Potential::compute (potential.h:67)
    def compute(self, error_vec: Optional[list] = None) -> float:
        if error_vec is not None:
            out = self.ev.objective(self.x[None, :], self.precision, errvec=True)
            error_vec[:] = list(out["errvec"][0])
            val = float(out["obj"][0])
        else:
            val = float(self.ev.objective(self.x[None, :], self.precision)[0])
        self.error_sum = val
        Potential.ncalls += 1
        return val

    def get_error(self) -> float:
        return self.error_sum

    # --- Potential::set_dir / compute_dir (potential.cpp:268-292)
    def set_dir(self, dir_vec, x: float) -> None:
        self.x += x * np.asarray(dir_vec, dtype=np.float64)

    def compute_dir(self, error_vec: Optional[list], dir_vec, x: float) -> float:
        tmp = self.clone()
        tmp.set_dir(dir_vec, x)
        return tmp.compute(error_vec)

    def compute_densities(self) -> np.ndarray:
        return self.ev.densities(self.x)

    # --- Potential::rescale (potential.h:68)
    def rescale(self, flag: int = 1, out=None) -> int:
        """Rescale this potential (PotMEAM::rescale / PotEAM::rescale) from its
        GPU densities.  The reference rescales only the potential it is
        called on, so a copy of the potential file is rescaled and this
        object gets its own evaluator when anything changed."""
        ev = self.ev
        if ev.pot.style == _lib.MZ_STYLE_PAIR_SPLINE:
            return 0  # Potential::rescale (potential.cpp:258-261)
        dens = ev.densities(self.x)
        pot = ev.pot.copy()
        pot.set_coeffs(self.x)
        changed, a, b = pot.rescale(ev.db, dens, flag)
        if changed:
            if out is not None:
                if b:
                    out.write("MEAM potential scaling factor %f\n" % b)
                for name, bp in zip(("JMEAM", "JMEAM2"), pot.jmeam_factors):
                    if bp:
                        out.write("%s potential scaling factor %f\n" % (name, bp))
                out.write("Embedding function scaling factor %f\n" % a)
            self.ev = Evaluator(ev.db, pot, ev.energy_weight, ev.stress_weight, ev.embed_extrap, device=ev.device,
                                max_candidates=ev.max_candidates, omit_punishments=ev.omit_punishments)
            self.x = pot.coeffs()
        return int(changed)

    # --- output
    def write_pot(self, path: str, num: int = -1) -> None:
        pot = self.ev.pot
        keep = pot.coeffs()
        pot.set_coeffs(self.x)
        try:
            pot.write(path if num < 0 else "%s.%d" % (path, num))
        finally:
            pot.set_coeffs(keep)

    def write_data(self, prefix: str, num: int = -1) -> None:
        """Potential::write_data (potential.cpp:325-342): .rho .energy .stress
        .force .error .punish files from one FP64 evaluation on the GPU
        (pair/spline: no .rho or .punish)."""
        ev = self.ev
        out = ev.objective(self.x[None, :], MZ_FP64, errvec=True, forces=True, energy=True, stress=True)
        dens = (None if ev.pot.style == _lib.MZ_STYLE_PAIR_SPLINE else
                np.ascontiguousarray(ev.densities(self.x), dtype=np.float64))
        pot = ev.pot.copy()
        pot.set_coeffs(self.x)
        write_data_arrays(ev.db, pot, ev.energy_weight, ev.stress_weight, out["errvec"][0], out["energy"][0],
                          out["stress"][0], out["forces"][0], dens, prefix, num)

    def error_breakdown(self) -> dict:
        """Force / energy / stress / punish sums as the .error file reports them
        (Potential::write_errors, potential.cpp:634-707)."""
        ev: list = []
        total = self.compute(ev)
        e = np.asarray(ev)
        view = self.ev.db.view()
        a0 = view["cell_atom0"]
        sums = dict(energy=0.0, stress=0.0, forces=0.0)
        idx = 0
        for c in range(view["ncells"]):
            na = a0[c + 1] - a0[c]
            sums["energy"] += e[idx] ** 2
            sums["stress"] += float(np.sum(e[idx + 1: idx + 7] ** 2))
            sums["forces"] += float(np.sum(e[idx + 7: idx + 7 + 3 * na] ** 2))
            idx += 7 + 3 * na
        sums["punish"] = float(np.sum(e[idx:] ** 2))
        sums["total"] = total
        return sums


def from_param_file(path: str, device: int = 0, max_candidates: int = 1, precision=MZ_FP64) -> Potential:
    """Build everything from a reference parameter file (config, startpot,
    energy_weight, stress_weight, embed_extrap keys)."""
    p = read_param(path)

    def resolve(f):  # the reference opens file names as given (relative to the working directory)
        return f

    if "config" not in p:
        raise MzError(3, 'ERROR: Parameter not found in file: "config"')
    if "startpot" not in p:
        raise MzError(3, 'ERROR: Parameter not found in file: "startpot"')
    pot = PotentialFile.read(resolve(p["startpot"][0]))
    db = Database.read(resolve(p["config"][0]), pot)
    ew = float(p.get("energy_weight", ["0"])[0])
    sw = float(p.get("stress_weight", ["0"])[0])
    ee = int(p.get("embed_extrap", ["0"])[0])
    ev = Evaluator(db, pot, ew, sw, ee, device=device, max_candidates=max_candidates)
    return Potential(ev, precision=precision)


def write_data_arrays(db: Database, pot: PotentialFile, energy_weight: float, stress_weight: float, errvec, energy,
                      stress, forces, densities, prefix: str, num: int = -1) -> None:
    """The reference's data files from evaluated arrays (mz_write_data);
    densities None for pair/spline."""
    arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).ravel()
            for a in (errvec, energy, stress, forces, densities)]
    check(lib().mz_write_data(db.handle, pot.handle, float(energy_weight), float(stress_weight),
                              *[ptr(a) for a in arrs], prefix.encode(), int(num)))
