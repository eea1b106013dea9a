"""The sharded multi-rank objective on CPU ranks (gloo, world size 2).

Each rank builds its shard with parallel.gpu_shard -- the real cell split and
the punishment left out on rank 1 -- with an evaluator factory that puts the
CPU oracle where the GPU Evaluator would be (objective from the C
restatement, gradient from its tangent-linear restatement, both honouring
omit_punishments).  The all-reduced objective and gradient must equal the
whole database's, on every rank.  The NCCL path (device buffers, one GPU per
rank) is the same code with the Evaluator; it is not measured on hardware."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class OracleEvaluator:
    """CPU stand-in with the Evaluator's constructor and objective /
    objective_grad calls."""

    def __init__(self, db, pot, energy_weight, stress_weight, embed_extrap, device=None, max_candidates=1,
                 omit_punishments=False):
        import oracle
        self.db, self.pot = db, pot
        self.orc = oracle.CRestatement(db.view(), [pot.spline(s) for s in range(pot.nsplines)], pot.style,
                                       pot.ntypes, energy_weight, stress_weight, embed_extrap,
                                       omit_punishments=int(omit_punishments))

    def objective(self, x, precision=None):
        return np.array([self.orc.objective(r) for r in np.atleast_2d(x)])

    def objective_grad(self, x, precision=None):
        x = np.atleast_2d(x)
        return self.objective(x), np.stack([self.orc.gradient(r) for r in x])


def _rank_main(rank, world, port, q):
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        import oracle
        from test_parallel_gloo import OracleEvaluator
        from meamzilla_b200 import synth
        from meamzilla_b200.parallel import ShardedObjective, gpu_shard
        from meamzilla_b200.potential import Database, PotentialFile
        spec, cells = synth.make_workload("meam2k", seed=7, ncells=6)
        rng = np.random.default_rng(1)
        for c in cells:
            c.energy0 = rng.normal(-3, 0.1)
            c.force0 = rng.normal(0, 0.3, (c.natoms, 3))
        ev, local, (lo, hi) = gpu_shard(cells, spec, rank, world, 5.5, make_evaluator=OracleEvaluator)
        sharded = ShardedObjective(local)
        assert sharded.device is None  # gloo reduces host buffers
        pot = PotentialFile.from_spec(spec)
        x0 = pot.coeffs()
        X = np.stack([x0, x0 + rng.normal(0, 0.02, x0.size)])
        total = sharded(X)
        tobj, tgrad = sharded(X, grad=True)
        if rank == 0:
            dbf = Database.from_cells(cells, pot)
            full = oracle.CRestatement(dbf.view(), [pot.spline(s) for s in range(pot.nsplines)], pot.style,
                                       pot.ntypes, 1.0, 1.0)
            ref = np.array([full.objective(r) for r in X])
            gref = np.stack([full.gradient(r) for r in X])
            q.put(("ok", list(total), list(ref), (lo, hi), list(tobj), tgrad.tolist(), gref.tolist()))
        else:
            q.put(("rank1", list(total), None, (lo, hi), list(tobj), tgrad.tolist(), None))
    except Exception as e:  # report, do not hang the other rank
        q.put(("error", repr(e), None, None, None, None, None))
        raise
    finally:
        dist.destroy_process_group()


def test_sharded_objective_and_gradient_two_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    errs = [r for r in res if r[0] == "error"]
    assert not errs, errs
    r0 = next(r for r in res if r[0] == "ok")
    r1 = next(r for r in res if r[0] == "rank1")
    assert r0[3][1] == r1[3][0]  # contiguous shards
    np.testing.assert_allclose(r0[1], r0[2], rtol=1e-12)
    np.testing.assert_allclose(r1[1], r0[1], rtol=0, atol=0)  # identical on every rank
    np.testing.assert_allclose(r0[4], r0[2], rtol=1e-12)
    g, gref = np.array(r0[5]), np.array(r0[6])
    assert np.max(np.abs(g - gref)) <= 1e-10 * np.max(np.abs(gref))
    np.testing.assert_array_equal(np.array(r1[5]), g)


def test_shard_cells_balances_and_covers():
    from meamzilla_b200.parallel import shard_cells
    work = [5, 1, 1, 1, 8, 2, 2, 3, 9, 1]
    for world in (1, 2, 3, 4):
        parts = shard_cells(work, world)
        assert parts[0][0] == 0 and parts[-1][1] == len(work)
        assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
        assert all(hi > lo for lo, hi in parts)
    with pytest.raises(ValueError):
        shard_cells([1, 2], 3)
