"""SpecieP's diagnostic maps (pcg_species_map) against the oracle.

The oracle's maps equal the reference's bit for bit
(tests/test_oracle_vs_reference.py); the GPU sums each node with FP64
atomics in another order, so maps agree to RTOL_MAP = 1e-12 of each map's
largest value, and the temperature (a difference of two squared sums) to
RTOL_TEMP = 1e-8 of its largest value.  The float layout is checked on the
positions and velocities it stores (exported exactly as doubles).
"""
import numpy as np
import pytest

from oracle.harness import OracleSim
from tests.cases import ELECTRONS, IONS, map_particles, small_grid

pytestmark = pytest.mark.gpu

RTOL_MAP = 1e-12
RTOL_TEMP = 1e-8
ORDER = ("density", "energy", "temperature", "momentum")


@pytest.mark.parametrize("precision,quirks,counts", [
    ("f64", "reference", (4000, 3000)), ("f64", "fixed", (4000, 3000)), ("f32", "reference", (4000, 3000)),
    ("f64", "reference", (60, 25)), ("f32", "fixed", (60, 25))])
def test_species_maps_match_oracle(precision, quirks, counts):
    """Dense, and with most nodes empty (their maps hold zeros)."""
    from picopic_b200 import Domain
    grid = small_grid(nr=12, nz=24, pml=False)
    d = Domain(grid, precision=precision, quirks=quirks, seed=5)
    d.add(ELECTRONS, capacity=5000)
    d.add(IONS, capacity=5000)
    d.set_particles(0, *map_particles(grid, counts[0], 3))
    d.set_particles(1, *map_particles(grid, counts[1], 4, mass=1836.0))
    o = OracleSim(grid, quirks=quirks)
    o.add(ELECTRONS)
    o.add(IONS)
    for sid in (0, 1):
        p = d.get_particles(sid)
        o.set_particles(sid, p["r"], p["z"], p["vr"], p["vphi"], p["vz"], p["w"])
    for which in ORDER:
        for sid in (0, 1):
            a, b = d.species_map(sid, which), o.species_map(sid, which)
            scale = np.abs(b).max()
            assert scale > 0, which
            tol = RTOL_TEMP if which == "temperature" else RTOL_MAP
            assert np.abs(a - b).max() <= tol * scale, f"{which} species {sid}"


def test_density_map_integrates_to_the_particle_count():
    """sum over nodes of density x node volume = the real particles, for
    particles away from the axis and the walls (weight_cylindrical
    normalises each node's share by its CELL_VOLUME; with the reference's
    macro expansion node i + 1 takes 2i + 2 where its volume is 2i + 3, so
    this holds to the ratio of the two, here within 5 %)."""
    from picopic_b200 import Domain
    grid = small_grid(nr=24, nz=32, pml=False)
    d = Domain(grid, precision="f64", seed=5)
    d.add(ELECTRONS, capacity=5000)
    rng = np.random.default_rng(2)
    n = 4000
    r = (8 + rng.random(n) * 8) * grid.dr
    z = (4 + rng.random(n) * 24) * grid.dz
    w = rng.random(n) * 1e6 + 1e5
    zero = np.zeros(n)
    d.set_particles(0, r, z, zero, zero, zero, w)
    dens = d.species_map(0, "density")
    i = np.arange(-2, grid.nr + 2)[:, None]
    vol = np.pi * grid.dz * grid.dr ** 2 * np.where(i >= 0, 2 * i + 1, 0)
    total = np.sum(dens * vol)
    assert abs(total / w.sum() - 1) < 0.05
