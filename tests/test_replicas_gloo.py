"""The multi-GPU path on CPUs: replicas as two gloo ranks.

The hot path does not shard (each GPU runs its own simulation), so the
N-rank job is N independent runs, seeded by rank, whose time is the
maximum over ranks and whose work is the sum, reduced once after the timed
region (picopic_b200.replicas, what bench.py uses with NCCL).  Each rank
here runs a small oracle simulation on the CPU: its result equals the same
run done alone (no data crosses between replicas), seeds differ by rank,
and the reductions give max and sum over ranks.
"""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _simulate(seed):
    from oracle.harness import OracleSim
    from tests.cases import ELECTRONS, IONS, particles, small_grid
    grid = small_grid(pml=False)
    sim = OracleSim(grid, "borisrel", "vb", quirks="fixed")
    for sp in (ELECTRONS, IONS):
        sim.add(sp)
    for i, sp in enumerate((ELECTRONS, IONS)):
        sim.set_particles(i, *particles(grid, 500, seed + i, mass=sp.mass))
    assert sim.step(3) == 0
    return sim.get_field("e_z"), 3 * 1000


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from picopic_b200.replicas import Replicas
    rep = Replicas("gloo", timeout_s=60)
    seed = rep.seed(1234)
    ez, work = _simulate(seed)
    rep.barrier()
    elapsed = 1.0 + rank  # a stand-in for each rank's device time
    out[rank] = {"seed": seed, "ez_sum": float(np.abs(ez).sum()), "max": rep.allmax(elapsed),
                 "sum": rep.allsum(work)}
    rep.close()


def test_two_gloo_replicas():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0]["seed"] != res[1]["seed"]
    for r in range(world):
        assert res[r]["max"] == 2.0          # the slowest rank's time
        assert res[r]["sum"] == 2 * 3000     # the work of both ranks
        ez, _ = _simulate(res[r]["seed"])    # the same run, alone
        assert res[r]["ez_sum"] == float(np.abs(ez).sum())
