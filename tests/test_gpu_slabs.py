"""A run split along z into slabs of GPU domains (picopic_b200/slabs.py,
several domains on one GPU in one process) against the undivided run on the
same GPU, with the strips exchanged through the host and device to device
(pcg_transfer_species_range, pcg_copy_field_columns): the FP64 layout within 1e-9 of each field array's largest value
and of each particle quantity after 10 steps (the deposit adds the same
currents in another order), the float layout within 1e-4 (fields) and 1e-5
(particles), as the float path is checked against the oracle."""
import numpy as np
import pytest

from oracle.harness import SpeciesSpec
from picopic_b200 import slabs as S
from tests.cases import ELECTRONS, IONS, beam_spec, particles, random_fields, small_grid

pytestmark = pytest.mark.gpu

STEPS = 10


def _species(grid):
    return [ELECTRONS, IONS, beam_spec(grid)]


def _domain(geometry, precision, quirks, species):
    from picopic_b200 import Domain
    d = Domain(geometry, pusher="borisrel", current="vb", precision=precision, quirks=quirks, seed=7)
    for sp in species:
        d.add(sp, capacity=40000)
    return d


def _inputs(grid):
    parts = {}
    for i, sp in enumerate(_species(grid)):
        if sp.beam is None:
            parts[i] = particles(grid, 3000, 30 + i, mass=sp.mass, boost=30.0 if sp.mass == 1 else 150.0)
    return parts, random_fields(grid, 5)


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _sorted(p):
    order = np.lexsort((p["r"], p["z"]))
    return {k: np.asarray(p[k])[order] for k in S.PARTICLE_KEYS}


@pytest.mark.parametrize("precision,quirks,count,on_device", [
    ("f64", "reference", 2, False), ("f64", "reference", 2, True), ("f64", "fixed", 3, True),
    ("f32", "fixed", 2, False), ("f32", "fixed", 3, True)])
def test_gpu_slabs_equal_the_undivided_run(precision, quirks, count, on_device):
    grid = small_grid(nr=16, nz=96)
    species = _species(grid)

    def make(geometry, slab):
        sp = [s if (slab.first or s.beam is None) else SpeciesSpec(s.name, s.charge, s.mass, id=s.id)
              for s in species]
        return _domain(geometry, precision, quirks, sp)

    g = S.SlabGroup(grid, count, make, species, on_device=on_device)
    assert g.on_device == on_device
    whole = _domain(grid, precision, quirks, species)
    parts, fields = _inputs(grid)
    for i, p in parts.items():
        g.set_particles(i, *p)
        whole.set_particles(i, *p)
    for k, a in fields.items():
        g.set_field(k, a)
        whole.set_field(k, a)
    g.step(STEPS)
    whole.step(STEPS)
    tol_f, tol_p = (1e-9, 1e-9) if precision == "f64" else (1e-4, 1e-5)
    for k in S.FIELDS:
        assert _rel(g.get_field(k), whole.get_field(k)) <= tol_f, k
    for t in range(len(species)):
        a, b = _sorted(g.get_particles(t)), _sorted(whole.get_particles(t))
        assert a["r"].size == b["r"].size, t
        for k in S.PARTICLE_KEYS:
            assert _rel(a[k], b[k]) <= tol_p, (t, k)
    assert g.get_particles(2)["r"].size > 0, "the beam was injected"


def test_gpu_beam_crosses_slab_boundaries():
    """The bunch injected in the first slab runs into the second (120 steps,
    48 cells, 2 slabs, device exchange, FP64) as in the undivided run."""
    grid = small_grid(nr=16, nz=48)
    species = _species(grid)

    def make(geometry, slab):
        sp = [s if (slab.first or s.beam is None) else SpeciesSpec(s.name, s.charge, s.mass, id=s.id)
              for s in species]
        return _domain(geometry, "f64", "fixed", sp)

    g = S.SlabGroup(grid, 2, make, species, on_device=True)
    whole = _domain(grid, "f64", "fixed", species)
    parts, fields = _inputs(grid)
    for i, p in parts.items():
        g.set_particles(i, *p)
        whole.set_particles(i, *p)
    for k, a in fields.items():
        g.set_field(k, a)
        whole.set_field(k, a)
    g.step(120)
    whole.step(120)
    assert g.parts[1].own(2)["r"].size > 0, "the bunch reached the second slab"
    for k in S.FIELDS:
        assert _rel(g.get_field(k), whole.get_field(k)) <= 1e-8, k
    for t in range(len(species)):
        a, b = _sorted(g.get_particles(t)), _sorted(whole.get_particles(t))
        assert a["r"].size == b["r"].size, t
        for k in S.PARTICLE_KEYS:
            assert _rel(a[k], b[k]) <= 1e-8, (t, k)
