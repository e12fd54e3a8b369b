"""A run split along z into slabs (picopic_b200/slabs.py) against the same
run undivided, on the CPU oracle as the slabs' engine.

Every slab is an ordinary domain over its cells plus ghost cells; after each
step the owners hand over the particles that left their cells, and the
ghost cells' fields and particles come from the slabs that own them.  The slabs' own cells must then hold what the undivided run holds:
the twelve field arrays within 1e-10 of each array's largest value (the
deposit sums the same currents in another particle order) and the same
particles.  With one slab per process the strips go through
torch.distributed point-to-point messages of a gloo group (two and three
ranks on 127.0.0.1).
"""
import os
import socket

import numpy as np
import pytest

from oracle.harness import OracleSim
from picopic_b200 import slabs as S
from tests.cases import ELECTRONS, IONS, beam_spec, particles, random_fields, small_grid

RTOL = 1e-10
STEPS = 6


def _species(grid):
    return [ELECTRONS, IONS, beam_spec(grid)]


def _plain(sp):
    """The beam without its injection (slabs after the first)."""
    from oracle.harness import SpeciesSpec
    return SpeciesSpec(sp.name, sp.charge, sp.mass, id=sp.id)


def _engine_factory(grid, quirks):
    species = _species(grid)

    def make(geometry, slab):
        o = OracleSim(geometry, "borisrel", "vb", quirks=quirks)
        for sp in species:
            o.add(sp if (slab.first or sp.beam is None) else _plain(sp))
        o.set_rng("philox", 7)
        return o
    return make, species


def _inputs(grid):
    species = _species(grid)
    parts = {}
    for i, sp in enumerate(species):
        if sp.beam is None:
            parts[i] = particles(grid, 2500, 30 + i, mass=sp.mass, boost=30.0 if sp.mass == 1 else 150.0)
    return parts, random_fields(grid, 5)


def _whole(grid, quirks):
    o = OracleSim(grid, "borisrel", "vb", quirks=quirks)
    for sp in _species(grid):
        o.add(sp)
    o.set_rng("philox", 7)
    parts, fields = _inputs(grid)
    for i, p in parts.items():
        o.set_particles(i, *p)
    for k, a in fields.items():
        o.set_field(k, a)
    assert o.step(STEPS) == 0
    return o


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _sorted(p):
    order = np.lexsort((p["r"], p["z"]))
    return {k: np.asarray(p[k])[order] for k in S.PARTICLE_KEYS}


def _compare(fields, particles_by_slot, whole, nsp):
    for k in S.FIELDS:
        assert _rel(fields[k], whole.get_field(k)) <= RTOL, k
    for t in range(nsp):
        a, b = _sorted(particles_by_slot[t]), _sorted(whole.get_particles(t))
        assert a["r"].size == b["r"].size, t
        for k in S.PARTICLE_KEYS:
            assert _rel(a[k], b[k]) <= RTOL, (t, k)


def test_plan_covers_the_grid():
    for nz, count in ((96, 2), (97, 3), (160, 5)):
        sl = S.plan(nz, count, ghost=6)
        assert sl[0].k0 == 0 and sl[-1].k1 == nz
        for a, b in zip(sl, sl[1:]):
            assert a.k1 == b.k0 and a.e1 == min(nz, a.k1 + 6) and b.e0 == b.k0 - 6
    with pytest.raises(ValueError):
        S.plan(96, 2, ghost=2)
    with pytest.raises(ValueError):
        S.plan(20, 4, ghost=6)


@pytest.mark.parametrize("count,quirks", [(2, "fixed"), (3, "reference")])
def test_slabs_equal_the_undivided_run(count, quirks):
    grid = small_grid(nr=16, nz=96)
    make, species = _engine_factory(grid, quirks)
    nsp = len(species)
    g = S.SlabGroup(grid, count, make, species)
    parts, fields = _inputs(grid)
    for i, p in parts.items():
        g.set_particles(i, *p)
    for k, a in fields.items():
        g.set_field(k, a)
    g.step(STEPS)
    whole = _whole(grid, quirks)
    _compare({k: g.get_field(k) for k in S.FIELDS}, [g.get_particles(t) for t in range(nsp)], whole, nsp)
    assert g.get_particles(2)["r"].size > 0, "the beam was injected"


def _rank_main(rank, world, port, out_dir, quirks):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        grid = small_grid(nr=16, nz=96)
        make, species = _engine_factory(grid, quirks)
        nsp = len(species)
        r = S.SlabRank(grid, make, species)
        parts, fields = _inputs(grid)
        for i, p in parts.items():
            r.set_particles(i, *p)
        for k, a in fields.items():
            r.set_field(k, a)
        r.step(STEPS)
        cols = {k: r.own_field_columns(k) for k in S.FIELDS}
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"),
                 **{f"f_{k}": v[1] for k, v in cols.items()}, lo=cols["e_r"][0],
                 **{f"p{t}_{k}": v for t in range(nsp) for k, v in r.own_particles(t).items()})
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_one_slab_per_gloo_rank(world, tmp_path):
    import torch.multiprocessing as mp
    quirks = "fixed"
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path), quirks), nprocs=world,
                       start_method="spawn")
    grid = small_grid(nr=16, nz=96)
    nsp = len(_species(grid))
    fields = {k: np.zeros(grid.shape) for k in S.FIELDS}
    parts = [[] for _ in range(nsp)]
    for rank in range(world):
        d = np.load(tmp_path / f"rank{rank}.npz")
        lo = int(d["lo"])
        for k in S.FIELDS:
            a = d[f"f_{k}"]
            fields[k][:, lo + 2:lo + 2 + a.shape[1]] = a
        for t in range(nsp):
            parts[t].append({k: d[f"p{t}_{k}"] for k in S.PARTICLE_KEYS})
    merged = [{k: np.concatenate([p[k] for p in parts[t]]) for k in S.PARTICLE_KEYS} for t in range(nsp)]
    _compare(fields, merged, _whole(grid, quirks), nsp)


def test_particles_at_slab_boundaries_are_handed_over_once():
    """Particles on and within a few ulp of the slab boundaries, crossing them
    both ways: after every step each is owned by exactly one slab, and the
    run ends as the undivided one does."""
    grid = small_grid(nr=16, nz=96)
    species = [ELECTRONS]
    make = lambda geometry, slab: _single(geometry)
    g = S.SlabGroup(grid, 3, make, species)
    rng = np.random.default_rng(3)
    faces = np.array([sl.k0 for sl in g.slabs[1:]], dtype=float) * grid.dz
    z = np.concatenate([[np.nextafter(f, -np.inf), f, np.nextafter(f, np.inf)] for f in faces] +
                       [f + grid.dz * np.array([-1e-9, 1e-9, -0.3, 0.3]) for f in faces])
    n = z.size * 20
    z = np.repeat(z, 20)
    r = grid.dr * (1.5 + rng.random(n) * (grid.nr - 3))
    vz = rng.choice([-1.0, 1.0], size=n) * (0.02 + 0.9 * rng.random(n)) * grid.dz / grid.dt
    p = (r, z, rng.normal(size=n) * 1e5, rng.normal(size=n) * 1e5, vz, np.full(n, 1e5))
    g.set_particles(0, *p)
    whole = _single(grid)
    whole.set_particles(0, *p)
    for _ in range(STEPS):
        g.step(1)
        whole.step(1)
        own = g.get_particles(0)
        assert own["r"].size == whole.count(0) == n
    b = _sorted(whole.get_particles(0))
    a = _sorted(g.get_particles(0))
    for k in S.PARTICLE_KEYS:
        assert _rel(a[k], b[k]) <= RTOL, k


def _single(geometry):
    o = OracleSim(geometry, "borisrel", "vb", quirks="fixed")
    o.add(ELECTRONS)
    o.set_rng("philox", 7)
    return o


def test_beam_crosses_slab_boundaries():
    """The injected bunch runs from the first slab through a boundary into the
    next (as plain particles there): 120 steps on a 48-cell grid in 2 slabs,
    against the undivided run (fields within 1e-8 of each array's largest
    value: rounding differences grow over the longer run)."""
    grid = small_grid(nr=16, nz=48)
    make, species = _engine_factory(grid, "fixed")
    g = S.SlabGroup(grid, 2, make, species)
    parts, fields = _inputs(grid)
    for i, p in parts.items():
        g.set_particles(i, *p)
    for k, a in fields.items():
        g.set_field(k, a)
    whole = OracleSim(grid, "borisrel", "vb", quirks="fixed")
    for sp in species:
        whole.add(sp)
    whole.set_rng("philox", 7)
    for i, p in parts.items():
        whole.set_particles(i, *p)
    for k, a in fields.items():
        whole.set_field(k, a)
    steps = 120
    g.step(steps)
    assert whole.step(steps) == 0
    beam = g.get_particles(2)
    boundary = g.slabs[1].k0 * grid.dz
    assert (beam["z"] >= boundary).sum() > 0, "the bunch reached the second slab"
    assert g.parts[1].own(2)["r"].size > 0
    for k in S.FIELDS:
        assert _rel(g.get_field(k), whole.get_field(k)) <= 1e-8, k
    for t in range(len(species)):
        a, b = _sorted(g.get_particles(t)), _sorted(whole.get_particles(t))
        assert a["r"].size == b["r"].size, t
        for k in S.PARTICLE_KEYS:
            assert _rel(a[k], b[k]) <= 1e-8, (t, k)
