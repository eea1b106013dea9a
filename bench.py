#!/usr/bin/env python
"""Benchmark of the B200 MEAM objective evaluator.

Metric: MEAM objective+gradient evaluations per second, batched in mixed
precision (FP32 spline and triplet arithmetic, FP64 sums), on the
two-species 2000-cell spline MEAM database (seeded synthetic data with the
generation rules of meamzilla_b200/synth.py, 136 coefficients), 64 candidate
coefficient vectors per step.  The FP64 plain objective rate (one candidate
per launch) is reported beside it, with the ratio.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]

One step = one objective+gradient launch sequence over all 64 candidates,
inputs resident on the device, timed with CUDA events on the evaluator's
stream.  `e2e` measures the same through the host API (host coefficient
vectors in, host objectives and gradients out).  Under torchrun each rank
evaluates its own 64 candidates (weak scaling, no collective on the data
path); the time is the maximum over ranks.

`--impl reference` times the reference program (compiled from its own
sources, oracle/_ref/mzref_fast) on the host cores: independent processes on
disjoint samples of the same database, its objective+gradient being the
objective plus one forward difference per coefficient as its Powell
optimizer forms it (opt_powell.cpp:363-384).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MEAM objective+gradient evals/s, mixed-batched vs FP64 plain GPU, rel err≤1e-6"
WORKLOAD = ("meam2k: two-species spline MEAM (meam/spline 2), 2000 periodic cells, atom count log-uniform "
            "in [8, 1024], 50/50 species, radial functions on [1.8, 5.5] A, 12 splines, 136 coefficients")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--ncand", type=int, default=64)
    ap.add_argument("--ncells", type=int, default=2000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--only-step", action="store_true",
                    help="run only the metric's step (warm-up + steps, no FP64, accuracy, end-to-end or CPU legs) "
                         "and print its time: the launch sequence the profiles capture")
    ap.add_argument("--cpu-configs", action="store_true",
                    help="time the compiled reference's objective on the smaller workloads (one JSON line each) "
                         "and exit")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers

def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    smax.append(float(p[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, p[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return d.get("hbm_gbs", 6650.0), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback: 6650 GB/s, an earlier copy measurement on this GPU type (MEASURED_PEAKS.json absent)"


def build_workload(args, device):
    """Teacher potential, database with teacher targets + noise, evaluator."""
    from meamzilla_b200 import synth
    from meamzilla_b200.potential import MZ_FP64, Database, Evaluator, PotentialFile
    spec, cells = synth.make_workload("meam2k", seed=args.seed, ncells=args.ncells)
    pot = PotentialFile.from_spec(spec)
    db = Database.from_cells(cells, pot)
    ev0 = Evaluator(db, pot, 1.0, 1.0, 0, device=device, max_candidates=1)
    out = ev0.objective(pot.coeffs()[None, :], MZ_FP64, forces=True, energy=True, stress=True)
    del ev0
    rng = np.random.default_rng(3000 + args.seed)
    nc = len(cells)
    e0 = out["energy"][0] + rng.normal(0.0, 1e-3, nc)
    s0 = out["stress"][0] + rng.normal(0.0, 0.01, (nc, 6)) / synth.GPA_PER_EV_A3
    f0 = out["forces"][0] + rng.normal(0.0, 0.01, out["forces"][0].shape)
    db.set_targets(e0, s0.ravel(), f0.ravel())
    a0 = np.cumsum([0] + [c.natoms for c in cells])
    for i, c in enumerate(cells):  # keep the python copy consistent for the CPU baseline files
        c.energy0, c.stress0, c.force0 = float(e0[i]), s0[i], f0[a0[i]:a0[i + 1]]
    ev = Evaluator(db, pot, 1.0, 1.0, 0, device=device, max_candidates=args.ncand)
    return spec, cells, pot, db, ev


def algorithmic(stats, ncand, P):
    """Fixed algorithmic work of one batched objective+gradient step, counted
    from the reference's expressions (splint_comb, spline3eq.h:110-122;
    fast_compute, pot_meam_spline.cpp:152-269): bytes
    B32 = 20 Np + 4 Nt + 48 N + 112 ncells + ncand (8 + 16 P) (FP32 pair and
    cosine streams, per-atom forces, per-cell targets and outputs, the
    candidates' coefficients and gradients) and forward flops
    145 Np + 111 Nt + 40 N per candidate (pairs: three cubic pieces with
    slopes and the force terms; triplets: the cosine, one g piece and the
    density and force terms; atoms: the embedding); the gradient costs two
    forward passes more."""
    Np, Nt, N, nc = stats["npairs"], stats["ntriplets"], stats["natoms"], stats["ncells"]
    b32 = 20 * Np + 4 * Nt + 48 * N + 112 * nc + ncand * (8 + 8 * P + 8 * P)
    fwd = 145 * Np + 111 * Nt + 40 * N
    return b32, fwd


def kernel_algorithmic_flops(name, stats, ncand):
    """The share of the step's algorithmic flops a kernel carries: the row
    kernels' forward (k_atoms) and adjoint (k_adj); on the triplet-moment path
    the contractions carry the triplet terms (forward 111 Nt, adjoint twice
    that) and the epilogues the pair and atom terms."""
    Np, Nt, N = stats["npairs"], stats["ntriplets"], stats["natoms"]
    fwd = 145 * Np + 111 * Nt + 40 * N
    table = {"k_atoms": fwd, "k_adj": 2 * fwd, "k_fm_fwd": 111 * Nt, "k_fm_adj": 2 * 111 * Nt,
             "k_fm_epi": 145 * Np + 40 * N, "k_fm_pre": 2 * (145 * Np + 40 * N)}
    return table.get(name, 0) * ncand


def executed_flops(name, stats, ncand, fm_dpad):
    """Flops a moment contraction executes (one FMA = 2): 2 x 3 Dpad x slots x
    candidates; None for the other kernels."""
    if name in ("k_fm_fwd", "k_fm_adj") and fm_dpad:
        return 2 * 3 * fm_dpad * stats["npairs"] * ncand
    return None


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def row_counts(cell, rcut):
    """Neighbours of every atom of a periodic cell within rcut over its
    images (the reference's full list, config.cpp:186-228), counted with a
    k-d tree -- the reference arm's own count, independent of the evaluator
    library."""
    from scipy.spatial import cKDTree
    L = np.asarray(cell.lattice, dtype=float)
    pos = np.asarray(cell.pos, dtype=float)
    vol = abs(np.linalg.det(L))
    m = [int(math.ceil(rcut / (vol / np.linalg.norm(np.cross(L[(k + 1) % 3], L[(k + 2) % 3]))))) for k in range(3)]
    shifts = np.array([[i, j, k] for i in range(-m[0], m[0] + 1) for j in range(-m[1], m[1] + 1)
                       for k in range(-m[2], m[2] + 1)], dtype=float) @ L
    images = (pos[None, :, :] + shifts[:, None, :]).reshape(-1, 3)
    return cKDTree(images).query_ball_point(pos, rcut, return_length=True) - 1


# Features per kind of the triplet-moment path on this workload: 2 partner
# types x 12 B-spline coefficients of f (10 knots) x 10 of g (8 knots) = 240.
FM_DPAD_MEAM2K = 240

# Algorithmic bytes per launch of the moment contractions: the moments read
# once (FP32, or four 8-bit digits of 256 padded features per kind when the
# forward runs on the tensor cores) and the per-slot sums written (FP64 Y) or
# read (FP32 dL/dY).
FM8_BYTES_PER_SLOT = 3 * 256 * 4
KERNEL_BYTES = {
    "k_fm_fwd": lambda st, nc: 4 * 3 * FM_DPAD_MEAM2K * st["npairs"] + 8 * 3 * st["npairs"] * nc,
    "k_fm_adj": lambda st, nc: 4 * 3 * FM_DPAD_MEAM2K * st["npairs"] + 4 * 3 * st["npairs"] * nc,
}
# The epilogues' per-slot, per-candidate streams: k_fm_epi reads Y (FP64 x 3)
# and writes V (FP64 x 3); k_fm_pre reads Y, the neighbours' lambda (FP32 x 3)
# and writes dL/dY (FP32 x 3).
KERNEL_BYTES["k_fm_epi"] = lambda st, nc: (24 + 24) * st["npairs"] * nc
KERNEL_BYTES["k_fm_pre"] = lambda st, nc: (24 + 12 + 12) * st["npairs"] * nc


def int8_mma_ops(stats, ncand):
    """Integer operations one moment contraction on the tensor cores
    executes: ten digit-pair MMAs over 3 kinds x 256 features per slot and
    64 candidates (2 ops per multiply-add), slots padded to 128-slot tiles."""
    slots = stats["npairs"]
    groups = (ncand + 63) // 64
    return 2 * 10 * 3 * 256 * slots * 64 * groups


KERNEL_BYTES_TC = {
    "k_fm_fwd": lambda st, nc: FM8_BYTES_PER_SLOT * st["npairs"] + 8 * 3 * st["npairs"] * nc,
    "k_fm_adj": lambda st, nc: FM8_BYTES_PER_SLOT * st["npairs"] + 4 * 3 * st["npairs"] * nc,
}
# DRAM bytes per launch measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum) on a smaller
# case of this workload, scaled by the units a full launch processes (profiles/ holds the captures).
KERNEL_TRAFFIC = {
    "k_adj": lambda st, nc: 2480.3e6 / 15.8433e6 * st["npairs"] * nc,
    "k_atoms": lambda st, nc: 496.0e6 / 3.9608e6 * st["npairs"] * nc,
    # 200-cell case, 1,980,412 pair slots x 64 candidates (profiles/k_fm_epilogues_small.md)
    "k_fm_adj_pre": lambda st, nc: 7605.1e6 / 126.746e6 * st["npairs"] * nc,
    "k_fm_epi": lambda st, nc: 7058.5e6 / 126.746e6 * st["npairs"] * nc,
}
KERNEL_TRAFFIC["k_fm_pre"] = KERNEL_TRAFFIC["k_fm_adj_pre"]


# --------------------------------------------------------- CPU reference arm

def cpu_reference(spec, cells, stats, P, reps, target_triplets=1.0e7, max_procs=64):
    """Time the compiled reference (oracle/_ref/mzref_fast) on disjoint samples
    of the database, one single-threaded process per host core (the
    reference's MPI atom decomposition without its communication).  Returns
    objective evals/s of the full database, extrapolated by triplet count."""
    import oracle
    from meamzilla_b200 import synth
    exe = oracle.MZREF_FAST
    if not os.path.exists(exe):
        return None, "oracle/_ref/mzref_fast not built"
    try:
        import psutil
        avail_gb = psutil.virtual_memory().available / 2 ** 30
    except Exception:
        avail_gb = 16.0
    ncores = os.cpu_count() or 1
    nproc = int(max(1, min(ncores, max_procs, avail_gb // 3)))
    # triplets per cell (j<k pairs of every row, the reference's triplet count)
    rows = stats["rows_per_cell"]
    trip = [int(sum(n * (n - 1) // 2 for n in r)) for r in rows]
    samples, i = [], 0
    while len(samples) < nproc and i < len(cells):
        lo, t = i, 0
        while i < len(cells) and t < target_triplets:
            t += trip[i]
            i += 1
        samples.append((lo, i, t))
    tmp = tempfile.mkdtemp(prefix="mzref_")
    procs = []
    for k, (lo, hi, t) in enumerate(samples):
        d = os.path.join(tmp, "s%d" % k)
        par = synth.write_case(d, spec, cells[lo:hi])
        procs.append((subprocess.Popen([exe, "-p", par, "-reps", str(reps), "-q"], stdout=subprocess.PIPE,
                                       stderr=subprocess.DEVNULL, text=True), t))
    rate = 0.0
    sample_trip = 0
    for pr, t in procs:
        out, _ = pr.communicate(timeout=1800)
        sec = None
        for line in out.splitlines():
            if line.startswith("seconds_per_eval"):
                sec = float(line.split()[1])
        if sec is None or pr.returncode != 0:
            return None, "reference run failed"
        rate += t / sec
        sample_trip += t
    subprocess.run(["rm", "-rf", tmp])
    obj_evals = rate / stats["ntriplets"]
    desc = ("%d concurrent single-thread processes of the reference (-Ofast -march=x86-64-v3) on %s, each on a "
            "disjoint run of cells (%d cells, %.3g triplets in all), %d timed compute() calls each after one "
            "warm-up; objective evals/s of the full database extrapolated by triplet count; objective+gradient = "
            "objective + %d forward differences" % (len(procs), cpu_model(), samples[-1][1] - samples[0][0],
                                                     sample_trip, reps, P))
    return {"obj_evals_per_s": obj_evals, "objgrad_evals_per_s": obj_evals / (P + 1), "cores": len(procs),
            "sample": desc, "cpu": cpu_model()}, None


def cpu_configs(reps=3):
    """The reference's objective on the three smaller workloads, on the host
    cores: the EAM database of 20 bcc cells (54 atoms), the single-species
    MEAM database of 200 cells (its 10 gradient points and the L-BFGS /
    Powell comparison use the same database) and the 500-cell MEAM
    population database.  One single-threaded process on the whole database,
    and the whole-core decomposition of cpu_reference.  Rows counted without
    the evaluator library."""
    from meamzilla_b200 import synth
    out = []
    for name in ("eam54", "meam200", "meam500"):
        spec, cells = synth.make_workload(name, seed=0)
        rcut = synth.WORKLOADS[name][2]
        rows = [row_counts(c, rcut) for c in cells]
        ntrip = int(sum(int((r * (r - 1) // 2).sum()) for r in rows)) if spec.style != "eam/spline" else 0
        stats = {"ntriplets": max(ntrip, 1), "rows_per_cell": rows, "natoms": sum(c.natoms for c in cells),
                 "npairs": int(sum(int(r.sum()) for r in rows))}
        # one process, the whole database (-np 1)
        import oracle
        tmp = tempfile.mkdtemp(prefix="mzcfg_")
        par = synth.write_case(os.path.join(tmp, name), spec, cells)
        t0 = time.perf_counter()
        r1 = subprocess.run([oracle.MZREF_FAST, "-p", par, "-reps", str(reps), "-q"], capture_output=True,
                            text=True, timeout=1800)
        sec1 = None
        for line in r1.stdout.splitlines():
            if line.startswith("seconds_per_eval"):
                sec1 = float(line.split()[1])
        subprocess.run(["rm", "-rf", tmp])
        line = {"workload": name, "ncells": len(cells), "natoms": stats["natoms"], "npairs": stats["npairs"],
                "ntriplets": ntrip, "ncoeff": spec_ncoeff(spec), "cpu": cpu_model(),
                "one_process": {"objective_evals_per_s": (1.0 / sec1) if sec1 else None, "cores": 1,
                                "reps": reps},
                "wall_s": time.perf_counter() - t0}
        if spec.style != "eam/spline":
            stats["rows_per_cell"] = rows
            # one disjoint run of cells per host core
            target = max(1.0e5, ntrip / float(os.cpu_count() or 1))
            res, err = cpu_reference(spec, cells, stats, spec_ncoeff(spec), reps, target_triplets=target)
            line["all_cores"] = ({"objective_evals_per_s": res["obj_evals_per_s"], "cores": res["cores"],
                                  "sample": res["sample"]} if res else {"unavailable": err})
        out.append(line)
        print(json.dumps(line), flush=True)
    return out


# ------------------------------------------------------------------- arms

def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    from meamzilla_b200 import synth  # the generator only: numpy, no evaluator library
    spec, cells = synth.make_workload("meam2k", seed=args.seed, ncells=args.ncells)
    rcut = synth.WORKLOADS["meam2k"][2]
    rows = [row_counts(c, rcut) for c in cells]
    stats = {"ncells": len(cells), "natoms": int(sum(c.natoms for c in cells)),
             "npairs": int(sum(int(r.sum()) for r in rows)),
             "ntriplets": int(sum(int((r * (r - 1) // 2).sum()) for r in rows)), "rows_per_cell": rows}
    P = spec_ncoeff(spec)
    t0 = time.time()
    res, err = cpu_reference(spec, cells, stats, P, reps=max(1, args.steps))
    wall = time.time() - t0
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return
    line = {
        "impl": "reference", "metric": METRIC, "value": res["objgrad_evals_per_s"], "unit": "evals/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 / res["objgrad_evals_per_s"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "ncells": stats["ncells"], "natoms": stats["natoms"],
                   "npairs": stats["npairs"], "ntriplets": stats["ntriplets"], "ncoeff": P},
        "objective_evals_per_s": res["obj_evals_per_s"],
        "cpu_baseline": {"value": res["objgrad_evals_per_s"], "unit": "evals/s", "cores": res["cores"],
                         "kind": "reference", "sample": res["sample"]},
        "e2e": {"value": res["objgrad_evals_per_s"], "unit": "evals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "wall_s": wall,
    }
    print(json.dumps(line))


def spec_ncoeff(spec):
    """Adjustable coefficients of a generated potential: free knots and free
    end slopes (Potential::get_ncoeff)."""
    n = 0
    for grp in spec.groups:
        for s in grp:
            fixed = s.fixed if s.fixed is not None else np.zeros(s.nknots, dtype=int)
            n += int(np.sum(np.asarray(fixed) == 0)) + sum(1 for e in s.bc if e == 0)
    return n


def _rows_per_cell(v):
    off = v["pair_off"]
    n = np.diff(off)
    a0 = v["cell_atom0"]
    return [n[a0[c]:a0[c + 1]] for c in range(v["ncells"])]


def run_mine(args, world, rank, local):
    import torch
    from meamzilla_b200 import synth
    from meamzilla_b200.potential import MZ_FP64, MZ_MIXED, alu_peak
    if not torch.cuda.is_available():
        raise RuntimeError("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    spec, cells, pot, db, ev = build_workload(args, local)
    stats = db.stats()
    P = pot.ncoeff
    x0 = pot.coeffs()
    X = synth.perturbed(x0, args.ncand, 0.05, seed=1 + rank)
    dev = torch.device("cuda", local)
    Xd = torch.tensor(X, dtype=torch.float64, device=dev)
    obj = torch.empty(args.ncand, dtype=torch.float64, device=dev)
    grad = torch.empty((args.ncand, P), dtype=torch.float64, device=dev)
    stream = torch.cuda.ExternalStream(ev.stream())

    # the autotuner picks its launch variant on the first call of each kind:
    # the metric's own call (64 candidates, mixed, with gradient) comes first
    ev.objective_grad_device(Xd, obj, grad, MZ_MIXED)
    ev.sync()
    if args.only_step:
        for _ in range(args.warmup + args.steps):
            ev.objective_grad_device(Xd, obj, grad, MZ_MIXED)
        ev.sync()
        if rank == 0:
            print(json.dumps({"only_step": True, "steps": args.warmup + args.steps, "ncand": args.ncand,
                              "ncells": args.ncells, "moment_path": ev.moment_path(MZ_MIXED, True)}))
        return

    # accuracy of the mixed path against FP64: objectives of all candidates,
    # forces and gradients of ACC_SAMPLE of them (every 64 / ACC_SAMPLE-th)
    ACC_SAMPLE = 8
    o64 = ev.objective(X, MZ_FP64)
    o32 = ev.objective(X, MZ_MIXED)
    pick = np.arange(0, args.ncand, max(1, args.ncand // ACC_SAMPLE))[:ACC_SAMPLE]
    ferr, gerr = [], []
    for c in pick:
        f64 = ev.objective(X[c:c + 1], MZ_FP64, forces=True)["forces"][0]
        f32 = ev.objective(X[c:c + 1], MZ_MIXED, forces=True)["forces"][0]
        ferr.append(float(np.max(np.abs(f32 - f64))))
    _, g64 = ev.objective_grad(X[pick], MZ_FP64)
    _, g32 = ev.objective_grad(X[pick], MZ_MIXED)
    for k in range(len(pick)):
        gerr.append(float(np.max(np.abs(g32[k] - g64[k])) / np.max(np.abs(g64[k]))))
    accuracy = {"obj_rel_err_max": float(np.max(np.abs(o32 - o64) / np.abs(o64))),
                "obj_candidates": int(args.ncand),
                "force_err_max_eV_per_A": float(max(ferr)),
                "grad_err_max_rel_to_max": float(max(gerr)),
                "force_grad_candidates": [int(c) for c in pick],
                "reference": "the GPU's own FP64 path, itself pinned to the reference at 1e-12"}

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    # ---- batched mixed objective + gradient (the metric)
    for _ in range(args.warmup):
        ev.objective_grad_device(Xd, obj, grad, MZ_MIXED)
    ev.sync()
    barrier()
    torch.cuda.synchronize()
    ev.sync()
    ev.kernel_times()
    ev.profile(True)
    l0 = ev.launches()
    clocks = ClockSampler(local)
    clocks.start()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        ev.objective_grad_device(Xd, obj, grad, MZ_MIXED)
    end.record(stream)
    end.synchronize()
    ev.sync()
    clk = clocks.stop()
    launches = ev.launches() - l0
    kt = ev.kernel_times()
    ev.profile(False)
    barrier()
    torch.cuda.synchronize()
    ms = max_over_ranks(start.elapsed_time(end))
    value = world * args.ncand * args.steps / (ms * 1e-3)

    # ---- FP64 plain objective, one candidate per launch
    x1 = Xd[:1].contiguous()
    o1 = torch.empty(1, dtype=torch.float64, device=dev)
    for _ in range(max(3, args.warmup)):
        ev.objective_device(x1, o1, MZ_FP64)
    ev.sync()
    barrier()
    k64 = max(5, 4 * args.steps)
    s2 = torch.cuda.Event(enable_timing=True)
    e2 = torch.cuda.Event(enable_timing=True)
    s2.record(stream)
    for _ in range(k64):
        ev.objective_device(x1, o1, MZ_FP64)
    e2.record(stream)
    e2.synchronize()
    ms64 = max_over_ranks(s2.elapsed_time(e2))
    fp64_rate = world * k64 / (ms64 * 1e-3)

    # ---- objective only, all candidates per launch (a GA population or annealing chains)
    batched = {}
    for name, prec in (("mixed", MZ_MIXED), ("fp64", MZ_FP64)):
        for _ in range(2):
            ev.objective_device(Xd, obj, prec)
        ev.sync()
        barrier()
        s3 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        s3.record(stream)
        for _ in range(3):
            ev.objective_device(Xd, obj, prec)
        e3.record(stream)
        e3.synchronize()
        batched[name + "_evals_per_s"] = world * 3 * args.ncand / (max_over_ranks(s3.elapsed_time(e3)) * 1e-3)
    batched["candidates_per_launch"] = args.ncand

    # ---- end to end through the host API (pinned host buffers)
    ph = torch.tensor(X, dtype=torch.float64).pin_memory()
    oh = torch.empty(args.ncand, dtype=torch.float64).pin_memory()
    gh = torch.empty((args.ncand, P), dtype=torch.float64).pin_memory()
    from meamzilla_b200._lib import check, lib
    import ctypes as C

    def host_step():
        check(lib().mz_objective_grad(ev.handle, args.ncand, C.c_void_p(ph.data_ptr()), MZ_MIXED,
                                      C.c_void_p(oh.data_ptr()), C.c_void_p(gh.data_ptr())))
    host_step()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        host_step()
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    e2e = world * args.ncand * args.steps / t_e2e

    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    tuned = ev.tuning(MZ_MIXED, True)

    # ---- roofline of the dominant kernel, on the bound that binds it: the
    # FP32 pipe for a CUDA-core contraction (the flops it executes; the row
    # formulation's algorithmic flops beside); HBM for the integer
    # tensor-core contractions (their digits and operands are read once;
    # the int8 MMA rate beside, against the nominal dense int8 peak) and for
    # the epilogues (their per-slot, per-candidate streams).  HBM is always
    # reported beside (roofline_hbm).
    hbm, hbm_src = measured_peaks()
    fp32_peak = alu_peak(local, MZ_MIXED)
    fp64_peak = alu_peak(local, MZ_FP64)
    b32, fwd = algorithmic(stats, args.ncand, P)
    dom = max(kt, key=lambda k: kt[k][0])
    dom_ms = kt[dom][0] / kt[dom][1]
    kflops = kernel_algorithmic_flops(dom, stats, args.ncand)
    fm_dpad = FM_DPAD_MEAM2K if tuned.get("triplet_moments") else None
    tc_fwd = bool(tuned.get("moment_forward_tensor_cores"))
    tc_adj = bool(tuned.get("moment_adjoint_tensor_cores"))
    on_tc = (dom == "k_fm_fwd" and tc_fwd) or (dom == "k_fm_adj" and tc_adj)
    table = dict(KERNEL_BYTES)
    if tc_fwd:
        table["k_fm_fwd"] = KERNEL_BYTES_TC["k_fm_fwd"]
        table["k_fm_adj"] = KERNEL_BYTES_TC["k_fm_adj"]
    kbytes = table.get(dom, lambda st, nc: None)(stats, args.ncand)
    roof_hbm = {"bound": "hbm", "kernel": dom, "algorithmic_bytes": kbytes,
                "achieved": kbytes / (dom_ms * 1e-3) / 1e9 if kbytes else None, "peak": hbm, "unit": "GB/s",
                "frac": kbytes / (dom_ms * 1e-3) / 1e9 / hbm if kbytes else None, "peak_source": hbm_src,
                "ms_per_launch": dom_ms}
    xflops = None if on_tc else executed_flops(dom, stats, args.ncand, fm_dpad)
    if on_tc or dom in ("k_fm_epi", "k_fm_pre"):
        roof = dict(roof_hbm, traffic=KERNEL_TRAFFIC.get(dom, lambda st, nc: None)(stats, args.ncand))
        if on_tc:
            ops = int8_mma_ops(stats, args.ncand)
            roof["int8_mma_ops"] = ops
            roof["int8_tops"] = ops / (dom_ms * 1e-3) / 1e12
            roof["int8_frac_of_nominal_4500"] = ops / (dom_ms * 1e-3) / 1e12 / 4500.0
    else:
        rflops = xflops if xflops else kflops
        roof = {"bound": "fp32", "kernel": dom, "achieved": rflops / (dom_ms * 1e-3) / 1e12, "peak": fp32_peak,
                "unit": "TFLOP/s", "frac": rflops / (dom_ms * 1e-3) / 1e12 / fp32_peak,
                "flops_per_launch": rflops, "flops_counted": "executed" if xflops else "algorithmic",
                "algorithmic_flops": kflops,
                "algorithmic_tflops": kflops / (dom_ms * 1e-3) / 1e12,
                "traffic": KERNEL_TRAFFIC.get(dom, lambda st, nc: None)(stats, args.ncand),
                "peak_source": "measured FMA stream on this GPU, FP32 (FP64: %.1f TFLOP/s)" % fp64_peak,
                "ms_per_launch": dom_ms}
    step_flops = 3 * fwd * args.ncand
    roof_step = {"algorithmic_flops": step_flops, "achieved_tflops": step_flops / (ms / args.steps * 1e-3) / 1e12,
                 "frac_fp32": step_flops / (ms / args.steps * 1e-3) / 1e12 / fp32_peak,
                 "algorithmic_bytes": b32,
                 "note": "flops of the per-triplet formulation (forward + 2x adjoint); the triplet-moment path "
                         "runs the triplet sums as integer tensor-core contractions instead, so this rate can "
                         "exceed the FP32 FMA peak" if tuned.get("triplet_moments") else
                         "flops of the per-triplet formulation (forward + 2x adjoint)"}
    roof_fp64 = {"bound": "fp64", "achieved": fwd / (ms64 / k64 * 1e-3) / 1e12, "peak": fp64_peak,
                 "unit": "TFLOP/s", "frac": fwd / (ms64 / k64 * 1e-3) / 1e12 / fp64_peak,
                 "algorithmic_flops": fwd}

    line = {
        "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded generator, meamzilla_b200/synth.py)",
        "config": {"workload": WORKLOAD, "ncells": stats["ncells"], "natoms": stats["natoms"],
                   "npairs": stats["npairs"], "ntriplets": stats["ntriplets"], "ncoeff": P,
                   "candidates_per_step_per_gpu": args.ncand, "precision": "mixed (FP32 splines, FP64 sums)",
                   "l2": "inputs larger than L2: pair streams %.2f GB" % (stats["npairs"] * 36 / 1e9),
                   "autotuned": tuned},
        "fp64_plain": {"value": fp64_rate, "unit": "objective evals/s", "ms_per_eval": ms64 / k64,
                       "candidates_per_launch": 1},
        "ratio_vs_fp64_plain": value / fp64_rate,
        "objective_only_batched": batched,
        "accuracy_vs_fp64": accuracy,
        "kernels_ms_per_step": {k: kt[k][0] / args.steps for k in kt},
        "roofline": roof,
        "roofline_hbm": roof_hbm,
        "roofline_step": roof_step,
        "roofline_fp64_plain": roof_fp64,
        "e2e": {"value": e2e, "unit": "evals/s", "h2d_bytes_per_step": args.ncand * P * 8,
                "d2h_bytes_per_step": args.ncand * (P + 1) * 8},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if world == 1 and not args.no_cpu_baseline:
        stats["rows_per_cell"] = _rows_per_cell(db.view())
        res, err = cpu_reference(spec, cells, stats, P, reps=3)
        if res is not None:
            line["cpu_baseline"] = {"value": res["objgrad_evals_per_s"], "unit": "evals/s", "cores": res["cores"],
                                    "kind": "reference", "sample": res["sample"], "cpu": res["cpu"],
                                    "objective_evals_per_s": res["obj_evals_per_s"]}
            # measured against measured: objective evaluations, FP64 GPU (one candidate per launch)
            # and mixed batched, over the reference's objective on the host cores
            line["vs_reference_objective"] = {
                "fp64_plain_over_cpu": fp64_rate / res["obj_evals_per_s"],
                "mixed_batched_over_cpu": batched["mixed_evals_per_s"] / res["obj_evals_per_s"],
                "objgrad_over_modelled_cpu_objgrad": value / res["objgrad_evals_per_s"]}
        else:
            line["cpu_baseline"] = {"value": None, "unavailable": err}
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    args = parse_args()
    world, rank, local = dist_setup(args)
    if args.cpu_configs:
        if rank == 0:
            cpu_configs()
        return
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
    else:
        run_mine(args, world, rank, local)


if __name__ == "__main__":
    main()
