"""Edge cases through the C ABI: empty species, one particle per species,
a one-run ensemble, and the errors a caller gets for a bad slot, a bad map
or an import beyond capacity."""
import numpy as np
import pytest

from tests.cases import ELECTRONS, IONS, particles, small_grid, thermal_plasma

pytestmark = pytest.mark.gpu


def _domain(precision, n=0, seed=3, cap=0):
    from picopic_b200 import Domain
    grid = small_grid(nr=16, nz=64, pml=False)
    d = Domain(grid, precision=precision, quirks="fixed", seed=seed)
    d.add(ELECTRONS, capacity=max(n, cap, 1) + 16)
    d.add(IONS, capacity=max(n, cap, 1) + 16)
    if n:
        for i, sp in enumerate((ELECTRONS, IONS)):
            d.set_particles(i, *particles(grid, n, seed + i, mass=sp.mass))
    return d, grid


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_empty_species_step_map_sort_collide(precision):
    d, grid = _domain(precision)
    d.step(3)
    dg = d.diag()
    assert dg.particles == 0 and dg.particle_steps == 0
    for which in ("density", "energy", "temperature", "momentum"):
        assert not np.any(d.species_map(0, which))
    if precision == "f32":
        counts, misplaced = d.tile_sort(0)
        assert counts.sum() == 0 and misplaced == 0
    assert d.collide() == 0
    assert np.all(np.isfinite(d.get_field("e_z")))


@pytest.mark.parametrize("scheme", ["p12", "ta77s"])
def test_one_electron_one_ion_per_cell(scheme):
    """The pairing sequence with one particle of each list per cell: one
    electron-ion pair per cell (and no like-particle pairs)."""
    from picopic_b200 import Domain
    grid = small_grid(nr=4, nz=8, pml=False)
    cells = grid.nr * grid.nz
    i, k = np.meshgrid(np.arange(grid.nr), np.arange(grid.nz), indexing="ij")
    r = (i.ravel() + 0.5) * grid.dr
    z = (k.ravel() + 0.5) * grid.dz
    d = Domain(grid, precision="f64", quirks="fixed", seed=5)
    d.add(ELECTRONS, capacity=cells)
    d.add(IONS, capacity=cells)
    _, _, vr, vphi, vz, _ = thermal_plasma(grid, cells, 1, 1.0, 1.0, 1e20)
    w = np.full(cells, 1e8)
    d.set_particles(0, r, z, vr, vphi, vz, w)
    d.set_particles(1, r, z, vr / 40, vphi / 40, vz / 40, w)
    d.set_collision_scheme(scheme)
    assert d.collide() == cells


def test_one_run_ensemble():
    from picopic_b200.ensemble import Ensemble
    d, _ = _domain("f32", n=2000)
    ens = Ensemble([d], threads=4)
    assert ens.step(3) > 0
    assert d.diag().particle_steps == 3 * 4000


def test_errors_for_bad_arguments():
    from picopic_b200._ffi import PcgError
    d, grid = _domain("f64", n=100)
    with pytest.raises(PcgError):
        d.species_map(7, "density")          # no such slot
    with pytest.raises(KeyError):
        d.species_map(0, "pressure")         # no such map
    with pytest.raises(PcgError):
        d.tile_sort(0)                       # the double layout has no tiles
    with pytest.raises(PcgError):
        d.set_particles(0, *particles(grid, 500, 9))  # capacity 116


def _with(grid, p, extra):
    """Particle arrays p with the particles of `extra` (r, z, vr, vphi, vz, w tuples) appended."""
    return [np.concatenate([np.asarray(a, float), np.array([e[q] for e in extra], float)])
            for q, a in enumerate(p)]


def test_float_import_drops_positions_outside_the_grid():
    """The float layout has no cell for a position outside the grid: such a
    particle is dropped at import and counted as removed, as the runaway
    collector removes it (a position within a cell of the grid raises no
    error; one farther out raises the out-of-grid error the double path
    raises, a position that is not a number the NaN error)."""
    from picopic_b200._ffi import PcgError
    d, grid = _domain("f32", cap=200)
    p = particles(grid, 100, 5)
    R, L = grid.radius, grid.longitude
    near = [(R + 0.5 * grid.dr, L / 2, 0, 0, 0, 1e5), (R / 2, -0.5 * grid.dz, 0, 0, 0, 1e5),
            (R / 2, L, 0, 0, 0, 1e5)]
    d.set_particles(0, *_with(grid, p, near))
    assert d.count(0) == 100
    assert d.diag().removed == 3
    d.step(2)
    d.synchronize()
    for bad, code in (((5 * R, L / 2, 0, 0, 0, 1e5), -4), ((float("nan"), L / 2, 0, 0, 0, 1e5), -10)):
        e, _ = _domain("f32", cap=200)
        e.set_particles(0, *_with(grid, p, [bad]))
        with pytest.raises(PcgError) as err:
            e.synchronize()
        assert err.value.code == code


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_superluminal_particle_stops_the_step(precision):
    """A particle faster than light ends the step with PCG_ERR_SUPERLUMINAL,
    the reference's fatal error (rel.cpp:33-34)."""
    from picopic_b200._ffi import PcgError
    d, grid = _domain(precision, cap=300)
    p = particles(grid, 200, 6)
    d.set_particles(0, *_with(grid, p, [(grid.radius / 2, grid.longitude / 2, 0, 0, 3.2e8, 1e5)]))
    d.step(1)
    with pytest.raises(PcgError) as err:
        d.synchronize()
    assert err.value.code == -11
