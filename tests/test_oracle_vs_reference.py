"""The CPU oracle against the reference's own sources, stage by stage.

oracle/Makefile.ref compiles the unmodified reference hot path into
oracle/_ref/; these tests run the same seeded inputs through both and demand
bit-identical fields, particles, cell indices and status codes after every
stage of the reference step order (PiCoPiC.cpp:326-347, SMB.cpp:1231-1306).
"""
import numpy as np
import pytest

from oracle.harness import FIELDS, STAGES, OracleSim, RefSim, reference_available
from tests.cases import ELECTRONS, IONS, beam_spec, load, small_grid, thermal_plasma

COMBOS = [(p, c) for p in ("borisrel", "boris", "vay", "hc") for c in ("vb", "zigzag")]


def _assert_same(o, r, nsp, where):
    fo, fr = o.fields(), r.fields()
    for k in FIELDS:
        np.testing.assert_array_equal(fo[k], fr[k], err_msg=f"{where}: field {k}")
    for sid in range(nsp):
        po, pr = o.get_particles(sid), r.get_particles(sid)
        for k in po:
            np.testing.assert_array_equal(po[k], pr[k], err_msg=f"{where}: species {sid} {k}")


@pytest.mark.parametrize("pusher,current", COMBOS)
def test_stagewise_bit_exact(pusher, current):
    if not reference_available(pusher, current):
        pytest.skip("compiled reference not built (oracle/Makefile.ref)")
    grid = small_grid()
    species = [ELECTRONS, IONS, beam_spec(grid)]
    o, r = OracleSim(grid, pusher, current), RefSim(grid, pusher, current)
    load(o, grid, species, 2000, seed=11)
    load(r, grid, species, 2000, seed=11)
    o.set_rng("mt19937", 42)
    r.seed(42)
    for step in range(3):
        for st in STAGES:
            assert o.stage(st) == r.stage(st) == 0, st
            if step == 0:
                _assert_same(o, r, len(species), f"step {step} after {st}")
        _assert_same(o, r, len(species), f"after step {step}")
    assert o.count(2) > 0, "beam was injected"
    assert o.errors == r.errors


def test_fatal_nan_position():
    """A NaN position is FATAL in the pusher (pusherBoris.cpp:51-57).

    The reference aborts there (and reads out of bounds if it went on), so
    only the oracle's error status is checked.
    """
    grid = small_grid(pml=False)
    o = OracleSim(grid)
    o.add(ELECTRONS)
    o.set_particles(0, [np.nan, 5e-4], [5e-4, 5e-4], [0, 0], [0, 0], [0, 0], [1, 1])
    assert o.stage("push") == -10


def test_long_run_removal_and_reflection():
    """20 full steps with fast particles: reflections and removals agree."""
    if not reference_available():
        pytest.skip("compiled reference not built")
    grid = small_grid(nr=16, nz=32)
    species = [ELECTRONS, IONS]
    o, r = OracleSim(grid), RefSim(grid)
    load(o, grid, species, 3000, seed=5)
    load(r, grid, species, 3000, seed=5)
    assert o.step(20) == r.step(20) == 0
    _assert_same(o, r, 2, "after 20 steps")


@pytest.mark.parametrize("ppc", [1, 2, 3, 10])
def test_p12_collisions_bit_exact(ppc):
    """One Perez-2012 collision pass (cells from the binding, no shuffle,
    the reference's mt19937 draws): velocities bit-identical."""
    if not reference_available():
        pytest.skip("compiled reference not built (oracle/Makefile.ref)")
    grid = small_grid(nr=8, nz=16, pml=False)
    n = grid.nr * grid.nz * ppc
    o, r = OracleSim(grid, quirks="reference"), RefSim(grid)
    for sim in (o, r):
        sim.add(ELECTRONS)
        sim.add(IONS)
        sim.set_particles(0, *thermal_plasma(grid, n, 1, 1.0, 1.0, 1e20, t_par_ratio=2.0))
        sim.set_particles(1, *thermal_plasma(grid, n + 7, 2, 1836.0, 0.5, 1e20))
    o.set_rng("mt19937", 123)
    r.seed(123)
    before = o.get_particles(0)["vz"].copy()
    # the oracle counts pair calls, the reference (collisionsP12.cpp:287)
    # only those that passed the early returns
    assert o.collide() >= r.collide() > 0 or ppc == 1
    for sid in (0, 1):
        po, pr = o.get_particles(sid), r.get_particles(sid)
        for k in ("vr", "vphi", "vz"):
            np.testing.assert_array_equal(po[k], pr[k], err_msg=f"species {sid} {k}")
    # one per cell: a row stops at its first cell without both species
    # (collisionsP12.cpp:351-354), so the pass may change nothing there
    assert ppc == 1 or np.abs(o.get_particles(0)["vz"] - before).max() > 0


@pytest.mark.parametrize("ppc", [1, 2, 3, 10])
def test_ta77s_collisions_bit_exact(ppc):
    """One Takizuka-Abe pass with the weighted correction (collisionsTA77S.cpp:
    pairs, then correct_velocities; no shuffle, the reference's mt19937
    draws: normal by the polar method, angle, dzeta): velocities
    bit-identical, with unequal electron and ion weights."""
    if not reference_available():
        pytest.skip("compiled reference not built (oracle/Makefile.ref)")
    grid = small_grid(nr=8, nz=16, pml=False)
    n = grid.nr * grid.nz * ppc
    o, r = OracleSim(grid, quirks="reference"), RefSim(grid)
    for sim in (o, r):
        sim.add(ELECTRONS)
        sim.add(IONS)
        sim.set_particles(0, *thermal_plasma(grid, n, 1, 1.0, 1.0, 1e20, t_par_ratio=2.0))
        sim.set_particles(1, *thermal_plasma(grid, n + 7, 2, 1836.0, 0.5, 1e20))
    o.set_rng("mt19937", 321)
    r.seed(321)
    before = o.get_particles(0)["vz"].copy()
    assert o.collide(scheme="ta77s") >= 0
    assert r.collide(scheme="ta77s") == 0
    for sid in (0, 1):
        po, pr = o.get_particles(sid), r.get_particles(sid)
        for k in ("vr", "vphi", "vz"):
            np.testing.assert_array_equal(po[k], pr[k], err_msg=f"species {sid} {k}")
    assert ppc == 1 or np.abs(o.get_particles(0)["vz"] - before).max() > 0


@pytest.mark.parametrize("ppc", [1, 2, 3, 10])
def test_sk98_collisions_bit_exact(ppc):
    """One CollisionsSK98 pass (collisionsSK98.cpp: relativistic CM-frame
    scattering, no rejection, no correction; no shuffle, the reference's
    mt19937 draws: normal by the polar method, uniform angle): velocities
    bit-identical, with unequal electron and ion weights."""
    if not reference_available():
        pytest.skip("compiled reference not built (oracle/Makefile.ref)")
    grid = small_grid(nr=8, nz=16, pml=False)
    n = grid.nr * grid.nz * ppc
    o, r = OracleSim(grid, quirks="reference"), RefSim(grid)
    for sim in (o, r):
        sim.add(ELECTRONS)
        sim.add(IONS)
        sim.set_particles(0, *thermal_plasma(grid, n, 1, 1.0, 1.0, 1e20, t_par_ratio=2.0))
        sim.set_particles(1, *thermal_plasma(grid, n + 7, 2, 1836.0, 0.5, 1e20))
    o.set_rng("mt19937", 99)
    r.seed(99)
    before = o.get_particles(0)["vz"].copy()
    assert o.collide(scheme="sk98") >= 0
    assert r.collide(scheme="sk98") == 0
    for sid in (0, 1):
        po, pr = o.get_particles(sid), r.get_particles(sid)
        for k in ("vr", "vphi", "vz"):
            np.testing.assert_array_equal(po[k], pr[k], err_msg=f"species {sid} {k}")
    assert ppc == 1 or np.abs(o.get_particles(0)["vz"] - before).max() > 0


@pytest.mark.parametrize("counts", [(4000, 3000), (60, 25)])
def test_species_maps_bit_exact(counts):
    """SpecieP::calc_density / calc_energy / calc_temperature / calc_momentum
    over weight_cylindrical: bit-identical grids, dense and with most cells
    empty (0/0 temperatures compare as NaN == NaN).  The temperature reads
    the absolute-momentum map the last energy map left; before any, the
    reference reads a grid it never initialised (undefined, not compared)."""
    if not reference_available():
        pytest.skip("compiled reference not built (oracle/Makefile.ref)")
    from tests.cases import map_particles
    grid = small_grid(nr=12, nz=24, pml=False)
    o, r = OracleSim(grid, quirks="reference"), RefSim(grid)
    for sim in (o, r):
        sim.add(ELECTRONS)
        sim.add(IONS)
        sim.set_particles(0, *map_particles(grid, counts[0], 3))
        sim.set_particles(1, *map_particles(grid, counts[1], 4, mass=1836.0))
    for which in ("density", "energy", "temperature", "momentum"):
        for sid in (0, 1):
            a, b = o.species_map(sid, which), r.species_map(sid, which)
            assert np.abs(a).max() > 0, which
            np.testing.assert_array_equal(a, b, err_msg=f"{which} species {sid}")


def test_sk98_conserves_momentum_and_energy_at_equal_weights():
    """Each SK98 pair rotates its CM-frame momentum and boosts back, so at
    equal weights the relativistic momentum sum(gamma m v) and energy
    sum(gamma m c^2) of the whole plasma are kept to rounding."""
    grid = small_grid(nr=8, nz=16, pml=False)
    n = grid.nr * grid.nz * 10
    o = OracleSim(grid, quirks="reference")
    o.add(ELECTRONS)
    o.add(IONS)
    masses = (9.1e-31, 1836 * 9.1e-31)
    for sid, (m, seed, T) in enumerate(((1.0, 1, 1.0), (1836.0, 2, 0.5))):
        r, z, vr, vphi, vz, w = thermal_plasma(grid, n, seed, m, T, 1e20)
        o.set_particles(sid, r, z, vr * 30, vphi * 30, vz * 30, np.full_like(w, 1e6))

    def totals():
        p_sum, e_sum = np.zeros(3), 0.0
        for sid, m in enumerate(masses):
            p = o.get_particles(sid)
            v = np.stack([p["vr"], p["vphi"], p["vz"]])
            g = 1 / np.sqrt(1 - (v ** 2).sum(0) / 9e16)
            p_sum += (g * m * v).sum(1)
            e_sum += (g * m * 9e16).sum()
        return p_sum, e_sum

    p0, e0 = totals()
    before = o.get_particles(0)["vz"].copy()
    o.set_rng("mt19937", 5)
    assert o.collide(scheme="sk98") > 0
    p1, e1 = totals()
    assert np.abs(o.get_particles(0)["vz"] - before).max() > 0
    # rounding against the sum of the momenta's magnitudes
    scale = sum(m * np.abs(np.stack([o.get_particles(sid)[k] for k in ("vr", "vphi", "vz")])).sum()
                for sid, m in enumerate(masses))
    assert np.abs(p1 - p0).max() <= 1e-13 * scale
    assert abs(e1 / e0 - 1) < 1e-14
