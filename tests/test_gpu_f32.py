"""The single-precision production path against the double-precision oracle.

The float path keeps positions as (cell, offset) and rewrites the
reference formulas in those coordinates; it is compared with the oracle on
the same seeded inputs.  Tolerances (stated relative to the array maximum):
fields after one step within RTOL_FIELD_1 = 2e-4 (float rounding in the
deposit of ~1e4 particles), particle positions within 1e-6 and velocities
within 1e-5; per-cell particle counts may differ only for particles within
float rounding of a cell boundary.
"""
import numpy as np
import pytest

from oracle.harness import FIELDS, OracleSim
from tests.cases import ELECTRONS, IONS, beam_spec, particles, random_fields, small_grid

pytestmark = pytest.mark.gpu

RTOL_FIELD_1 = 2e-4
RTOL_POS = 1e-6
RTOL_VEL = 1e-5
COMBOS = [(p, c) for p in ("borisrel", "boris", "vay", "hc") for c in ("vb", "zigzag")]


def _pair(grid, pusher, current, species, n, seed):
    from picopic_b200 import Domain
    gpu = Domain(grid, pusher=pusher, current=current, precision="f32", seed=7)
    orc = OracleSim(grid, pusher, current)
    for sp in species:
        gpu.add(sp, capacity=20000)
        orc.add(sp)
    for i, sp in enumerate(species):
        if sp.beam is None:
            p = particles(grid, n, seed + i, mass=sp.mass, boost=30.0 if sp.mass == 1 else 150.0)
            gpu.set_particles(i, *p)
            orc.set_particles(i, *p)
    for name, a in random_fields(grid, seed).items():
        gpu.set_field(name, a)
        orc.set_field(name, a)
    orc.set_rng("philox", 7)
    return gpu, orc


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300) if a.size else 0.0


@pytest.mark.parametrize("pusher,current", COMBOS)
def test_f32_one_step(pusher, current):
    grid = small_grid()
    species = [ELECTRONS, IONS, beam_spec(grid)]
    gpu, orc = _pair(grid, pusher, current, species, 3000, seed=3)
    gpu.step(1)
    assert orc.step(1) == 0
    for k in FIELDS:
        assert _rel(gpu.get_field(k), orc.get_field(k)) <= RTOL_FIELD_1, k
    for sid in range(len(species)):
        pg, po = gpu.get_particles(sid), orc.get_particles(sid)
        assert pg["r"].size == po["r"].size
        assert _rel(pg["r"], po["r"]) <= RTOL_POS and _rel(pg["z"], po["z"]) <= RTOL_POS
        for k in ("vr", "vphi", "vz"):
            assert _rel(pg[k], po[k]) <= RTOL_VEL, (sid, k)
        assert np.mean(pg["cell_r"] != po["cell_r"]) < 1e-3
        assert np.mean(pg["cell_z"] != po["cell_z"]) < 1e-3


def test_f32_ten_steps_field_energy():
    """Ten steps of the float path keep the field energy within 1e-3 of the
    double oracle on a small noisy case."""
    grid = small_grid()
    species = [ELECTRONS, IONS]
    gpu, orc = _pair(grid, "borisrel", "vb", species, 3000, seed=5)
    gpu.step(10)
    assert orc.step(10) == 0
    def energy(fields):
        return sum(float(np.sum(fields[k][2:-2, 2:-2] ** 2)) for k in ("e_r", "e_phi", "e_z"))
    eg = energy({k: gpu.get_field(k) for k in ("e_r", "e_phi", "e_z")})
    eo = energy({k: orc.get_field(k) for k in ("e_r", "e_phi", "e_z")})
    assert abs(eg - eo) / eo < 1e-3


def test_f32_removal_counts_and_launches():
    """A beam crossing z = L loses particles to the runaway collector over
    many steps, with tile sorts in between: the live count in the
    diagnostics matches the slot count after compaction, and the step
    reports the kernels it launched."""
    from picopic_b200 import Domain
    grid = small_grid()
    spec = beam_spec(grid, macro_amount=4000)
    gpu = Domain(grid, pusher="borisrel", current="vb", precision="f32", seed=7)
    gpu.add(ELECTRONS, capacity=20000)
    gpu.add(spec, capacity=200000)
    gpu.set_particles(0, *particles(grid, 3000, 11))
    d0 = gpu.diag()
    removed = 0
    for _ in range(12):
        gpu.step(20)
        d = gpu.diag()
        assert d.particles == gpu.count(0) + gpu.count(1)
        removed = d.removed
    assert removed > 0, "the case must push beam particles through z = L"
    assert gpu.diag().kernel_launches - d0.kernel_launches >= 3 * 240


def test_import_binds_cells_as_the_reference():
    """The float layout's cell of an imported particle is the reference's
    CELL_NUMBER (floor(pos / cell size) in double, geometry.hpp:198) of the
    same double position, also exactly on cell boundaries and one ulp below
    them."""
    from picopic_b200 import Domain
    grid = small_grid(nr=24, nz=160, pml=False)
    d = Domain(grid, precision="f32", seed=7)
    d.add(ELECTRONS, capacity=40000)
    rng = np.random.default_rng(12)
    n = 30000
    r = rng.uniform(0.5, grid.nr - 0.5, n) * grid.dr
    z = rng.uniform(0.5, grid.nz - 0.5, n) * grid.dz
    kr = rng.integers(1, grid.nr - 1, 2000)
    kz = rng.integers(1, grid.nz - 1, 2000)
    r[:1000], z[:1000] = kr[:1000] * grid.dr, kz[:1000] * grid.dz
    r[1000:2000] = np.nextafter(kr[1000:] * grid.dr, 0.0)
    z[1000:2000] = np.nextafter(kz[1000:] * grid.dz, 0.0)
    zero = np.zeros(n)
    d.set_particles(0, r, z, zero, zero, zero, np.ones(n))
    p = d.get_particles(0)
    np.testing.assert_array_equal(p["cell_r"], np.floor(r / grid.dr).astype(np.int64))
    np.testing.assert_array_equal(p["cell_z"], np.floor(z / grid.dz).astype(np.int64))


def test_tile_sort_groups_cells_exactly():
    """The float step's tile sort (pcg_tile_sort, the sort a step runs when
    particles drift): no particle outside its tile, and the per-cell counts
    the sorted tiles hold equal, bit for bit, those of the particles' cells
    and those the FP64 oracle binds (floor(r / dr), floor(z / dz)) from the
    same positions.  3 x 5 tiles of 8 x 32 cells; after 3 steps of moving
    particles."""
    from picopic_b200 import Domain
    grid = small_grid(nr=24, nz=160, pml=False)
    d = Domain(grid, precision="f32", seed=7)
    species = (ELECTRONS, IONS)
    for sp in species:
        d.add(sp, capacity=30000)
    for i, sp in enumerate(species):
        d.set_particles(i, *particles(grid, 20000, 40 + i, mass=sp.mass,
                                      boost=30.0 if sp.mass == 1 else 150.0))
    d.step(3)
    orc = OracleSim(grid)
    for sp in species:
        orc.add(sp)
    for sid in range(len(species)):
        counts, misplaced = d.tile_sort(sid)
        assert misplaced == 0
        p = d.get_particles(sid)
        assert counts.sum() == len(p["r"])
        mine = np.zeros((grid.nr, grid.nz), dtype=np.int64)
        np.add.at(mine, (p["cell_r"], p["cell_z"]), 1)
        assert np.array_equal(counts, mine)
        orc.set_particles(sid, p["r"], p["z"], p["vr"], p["vphi"], p["vz"], p["w"])
        po = orc.get_particles(sid)
        theirs = np.zeros((grid.nr, grid.nz), dtype=np.int64)
        np.add.at(theirs, (po["cell_r"], po["cell_z"]), 1)
        assert np.array_equal(counts, theirs)
