"""TEST ORACLE (test infrastructure, never part of the product).

Two checkers for the CUDA evaluator, both CPU-only and FP64:

* ``CRestatement`` -- oracle/mz_oracle.c, a plain-C restatement of the
  reference objective (PotMEAMSpline / PotEAMSpline ::fast_compute and
  Potential::accumulate_error) over the evaluator builder's neighbour lists.
* ``run_reference`` -- the UNMODIFIED reference program compiled from its own
  sources by oracle/Makefile (oracle/_ref/mzref) and driven through its own
  Potential::compute by oracle/ref_harness.cpp.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
MZREF = os.path.join(REF_DIR, "mzref")
MZREF_FAST = os.path.join(REF_DIR, "mzref_fast")
LIBORACLE = os.path.join(REF_DIR, "libmzoracle.so")


def build(reference_dir: str = "/root/reference") -> None:
    """make -C oracle (the reference binaries only where its sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE, "-j8", "REF=%s" % reference_dir], check=True)


class _Spline(C.Structure):
    _fields_ = [("nknots", C.c_int), ("left", C.c_double), ("right", C.c_double), ("nat", C.c_int * 2),
                ("grad_fixed", C.c_int * 2), ("grad", C.c_double * 2), ("y_fixed", C.POINTER(C.c_int)),
                ("y", C.POINTER(C.c_double)), ("quintic", C.c_int), ("grad2", C.c_double * 2)]


class _Pot(C.Structure):
    _fields_ = [("style", C.c_int), ("ntypes", C.c_int), ("nsplines", C.c_int), ("splines", C.POINTER(_Spline)),
                ("embed_extrap", C.c_int), ("energy_weight", C.c_double), ("stress_weight", C.c_double),
                ("omit_punishments", C.c_int)]


class _Db(C.Structure):
    _fields_ = [("ncells", C.c_int), ("natoms", C.c_int), ("npairs", C.c_int64),
                ("cell_atom0", C.POINTER(C.c_int)), ("cell_vol", C.POINTER(C.c_double)),
                ("cell_weight", C.POINTER(C.c_double)), ("cell_eweight", C.POINTER(C.c_double)),
                ("cell_sweight", C.POINTER(C.c_double)), ("cell_energy0", C.POINTER(C.c_double)),
                ("cell_stress0", C.POINTER(C.c_double)), ("atom_type", C.POINTER(C.c_int)),
                ("atom_cell", C.POINTER(C.c_int)), ("atom_force0", C.POINTER(C.c_double)),
                ("pair_off", C.POINTER(C.c_int64)), ("pair_nbr", C.POINTER(C.c_int)),
                ("pair_r", C.POINTER(C.c_double)), ("pair_u", C.POINTER(C.c_double)),
                ("pair_knot", C.POINTER(C.c_int8)), ("pair_shift", C.POINTER(C.c_double)), ("nfun", C.c_int)]


_liboracle = None


def _lib():
    global _liboracle
    if _liboracle is None:
        if not os.path.exists(LIBORACLE):
            subprocess.run(["make", "-s", "-C", HERE, "_ref/libmzoracle.so"], check=True)
        L = C.CDLL(LIBORACLE)
        L.mzo_objective.restype = C.c_double
        L.mzo_objective.argtypes = [C.POINTER(_Db), C.POINTER(_Pot), C.c_void_p] + [C.c_void_p] * 5
        L.mzo_objective_tangent.restype = C.c_double
        L.mzo_objective_tangent.argtypes = [C.POINTER(_Db), C.POINTER(_Pot), C.c_void_p, C.c_void_p,
                                            C.POINTER(C.c_double)]
        L.mzo_esize.restype = C.c_int
        L.mzo_esize.argtypes = [C.POINTER(_Db), C.POINTER(_Pot)]
        _liboracle = L
    return _liboracle


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class CRestatement:
    """The C restatement bound to one database view and potential structure.

    `view` is meamzilla_b200.Database.view(); `splines` is the list of
    PotentialFile.spline(s) dicts."""

    def __init__(self, view: dict, splines: list, style: int, ntypes: int, energy_weight=0.0, stress_weight=0.0,
                 embed_extrap=0, omit_punishments=0):
        self._keep = []
        arr = []
        for s in splines:
            yf = np.ascontiguousarray(s["y_fixed"], dtype=np.int32)
            y = np.ascontiguousarray(s["y"], dtype=np.float64)
            self._keep += [yf, y]
            sp = _Spline()
            sp.nknots = s["nknots"]
            sp.left, sp.right = s["left"], s["right"]
            sp.nat[0], sp.nat[1] = s["nat"]
            sp.grad_fixed[0], sp.grad_fixed[1] = s["grad_fixed"]
            sp.grad[0], sp.grad[1] = float(s["grad"][0]), float(s["grad"][1])
            sp.y_fixed = _p(yf, C.c_int)
            sp.y = _p(y, C.c_double)
            sp.quintic = int(s.get("quintic", 0))
            g2 = s.get("grad2", (0.0, 0.0))
            sp.grad2[0], sp.grad2[1] = float(g2[0]), float(g2[1])
            arr.append(sp)
        self._splines = (_Spline * len(arr))(*arr)
        self.pot = _Pot(style, ntypes, len(arr), C.cast(self._splines, C.POINTER(_Spline)), embed_extrap,
                        energy_weight, stress_weight, int(omit_punishments))
        v = {k: (np.ascontiguousarray(x) if isinstance(x, np.ndarray) else x) for k, x in view.items()}
        self._v = v
        d = _Db()
        d.ncells, d.natoms, d.npairs = v["ncells"], v["natoms"], v["npairs"]
        d.nfun = v.get("nfun", 3)
        for name, t in (("cell_atom0", C.c_int), ("cell_vol", C.c_double), ("cell_weight", C.c_double),
                        ("cell_eweight", C.c_double), ("cell_sweight", C.c_double), ("cell_energy0", C.c_double),
                        ("cell_stress0", C.c_double), ("atom_type", C.c_int), ("atom_cell", C.c_int),
                        ("atom_force0", C.c_double), ("pair_off", C.c_int64), ("pair_nbr", C.c_int),
                        ("pair_r", C.c_double), ("pair_u", C.c_double), ("pair_knot", C.c_int8),
                        ("pair_shift", C.c_double)):
            setattr(d, name, _p(v[name], t))
        self.db = d
        self.natoms, self.ncells = v["natoms"], v["ncells"]
        self.esize = _lib().mzo_esize(C.byref(self.db), C.byref(self.pot))

    @classmethod
    def for_evaluator(cls, ev):
        """Bound to the same database / potential / weights as an Evaluator."""
        pot = ev.pot
        splines = [pot.spline(s) for s in range(pot.nsplines)]
        return cls(ev.db.view(), splines, pot.style, pot.ntypes, ev.energy_weight, ev.stress_weight,
                   ev.embed_extrap)

    def objective(self, coeffs, full=False):
        x = np.ascontiguousarray(coeffs, dtype=np.float64)
        if not full:
            return _lib().mzo_objective(C.byref(self.db), C.byref(self.pot), x.ctypes.data, None, None, None, None,
                                        None)
        ev = np.zeros(self.esize)
        fo = np.zeros((self.natoms, 3))
        en = np.zeros(self.ncells)
        st = np.zeros((self.ncells, 6))
        de = np.zeros(self.natoms)
        obj = _lib().mzo_objective(C.byref(self.db), C.byref(self.pot), x.ctypes.data, ev.ctypes.data,
                                   fo.ctypes.data, en.ctypes.data, st.ctypes.data, de.ctypes.data)
        return dict(obj=obj, errvec=ev, forces=fo, energy=en, stress=st, dens=de)


    def tangent(self, coeffs, direction):
        """(objective, exact derivative along `direction`): the tangent-linear
        restatement, forward-mode differentiation of the objective."""
        x = np.ascontiguousarray(coeffs, dtype=np.float64)
        d = np.ascontiguousarray(direction, dtype=np.float64)
        out = C.c_double(0.0)
        obj = _lib().mzo_objective_tangent(C.byref(self.db), C.byref(self.pot), x.ctypes.data, d.ctypes.data,
                                           C.byref(out))
        return obj, out.value

    def gradient(self, coeffs):
        """Exact gradient: one tangent evaluation per coefficient direction."""
        x = np.ascontiguousarray(coeffs, dtype=np.float64)
        g = np.zeros(x.size)
        e = np.zeros(x.size)
        for i in range(x.size):
            e[:] = 0.0
            e[i] = 1.0
            g[i] = self.tangent(x, e)[1]
        return g


def run_reference(param_path: str, coeffs=None, fd_h: float = 0.0, reps: int = 0, fast: bool = False,
                  timeout: float = 600.0, cwd=None, rescale=None, write_prefix=None, powell_steps: int = 0) -> dict:
    """Run the compiled reference on a parameter file; returns its outputs."""
    exe = MZREF_FAST if fast else MZREF
    if not os.path.exists(exe):
        raise FileNotFoundError("reference oracle binary missing: %s (run make -C oracle)" % exe)
    with tempfile.TemporaryDirectory() as d:
        prefix = os.path.join(d, "out")
        cmd = [exe, "-p", param_path, "-o", prefix, "-q"]
        if coeffs is not None:
            xf = os.path.join(d, "x.bin")
            np.asarray(coeffs, dtype=np.float64).tofile(xf)
            cmd += ["-x", xf]
        if fd_h > 0:
            cmd += ["-fd", repr(float(fd_h))]
        if reps > 0:
            cmd += ["-reps", str(reps)]
        if rescale is not None:
            cmd += ["-rescale", str(int(rescale))]
        if write_prefix is not None:
            cmd += ["-write", os.path.abspath(write_prefix)]
        if powell_steps > 0:
            cmd += ["-powell", str(int(powell_steps))]
        res = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, cwd=cwd)
        if res.returncode != 0:
            raise RuntimeError("mzref failed (%d): %s %s" % (res.returncode, res.stdout[-2000:], res.stderr[-2000:]))
        out = {}
        for k in ("obj", "errvec", "energy", "stress", "force", "dens", "coeff", "fdgrad", "rescale", "powell"):
            f = "%s.%s.bin" % (prefix, k)
            if os.path.exists(f):
                out[k] = np.fromfile(f, dtype=np.float64)
        out["obj"] = float(out["obj"][0])
        for line in res.stdout.splitlines():
            if line.startswith("seconds_per_eval"):
                out["seconds_per_eval"] = float(line.split()[1])
        return out
