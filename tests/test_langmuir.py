"""Langmuir oscillation: a cold, exactly neutral plasma given a small
sinusoidal v_z must oscillate at the plasma frequency
omega_p = sqrt(n e^2 / (eps0 m_e)).

Set-up (tests/cases.quiet_plasma): 16 x 64 cells of 1e-4 m, n = 1e22 m^-3
(omega_p = 5.64e12 s^-1, c k / omega_p ~ 0.1 for the grid's longest modes,
so the electromagnetic modes the conducting wall mixes in sit within 0.5 %
of omega_p), dt = 0.05 of the Courant limit (omega_p dt = 0.066), 4 x 4
lattice points per cell, v0 = 1e5 m/s.  E_z is sampled every step at the
nodes (i, 16) for 400 steps (4.2 plasma periods) and its dominant frequency
found per radius.

With PCG_QUIRKS_FIXED the interior rows 2..12 oscillate within
FREQ_RTOL = 1 % of omega_p.  The reference's gather normalises its ring
weights by cell volumes (maxwellSolver.hpp:101-316), so a uniform field
reaches a particle at row i scaled by about 1 - 1/(2i); its interior
frequency is low by half that (row 8: ~3 %), which the reference-mode case
records.  The axis row (plasma starts at the reflecting wall r = dr/2) and
the row next to the outer wall are left out: their frequencies are set by
the boundaries, not by the bulk plasma.
"""
import numpy as np
import pytest

from oracle.harness import OracleSim
from tests.cases import (ELECTRONS, IONS, dominant_frequency, plasma_frequency, quiet_plasma,
                         small_grid)

DENSITY = 1e22
STEPS = 400
ROWS = range(2, 13)
Z_NODE = 16
FREQ_RTOL = 0.01


def _grid():
    dt = 0.05 * 1e-4 / (3e8 * np.sqrt(2))
    return small_grid(16, 64, pml=False, dt=dt)


def _row_frequencies(samples, grid):
    wp = plasma_frequency(DENSITY)
    e = np.array(samples)
    return np.array([dominant_frequency(e[:, i], grid.dt, 0.7 * wp, 1.3 * wp) for i in ROWS]) / wp


def _run_oracle(quirks):
    grid = _grid()
    sim = OracleSim(grid, "borisrel", "vb", quirks=quirks)
    sim.add(ELECTRONS)
    sim.add(IONS)
    el, io = quiet_plasma(grid, DENSITY, 4, 1e5)
    sim.set_particles(0, *el)
    sim.set_particles(1, *io)
    samples = []
    for _ in range(STEPS):
        assert sim.step(1) == 0
        samples.append(sim.get_field("e_z")[2:grid.nr + 2, 2 + Z_NODE].copy())
    return _row_frequencies(samples, grid)


def test_oracle_langmuir_frequency_fixed():
    f = _run_oracle("fixed")
    assert np.abs(f - 1).max() <= FREQ_RTOL, f


def test_oracle_langmuir_frequency_reference_gather_bias():
    f = _run_oracle("reference")
    # row 8 sees a uniform E_z weighted by ~1 - 1/16: omega ~ 0.97 omega_p
    assert 0.95 <= f[ROWS.index(8)] <= 0.985, f


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_langmuir_frequency(precision):
    from picopic_b200 import Domain
    grid = _grid()
    d = Domain(grid, pusher="borisrel", current="vb", precision=precision, quirks="fixed", seed=7)
    el, io = quiet_plasma(grid, DENSITY, 4, 1e5)
    d.add(ELECTRONS, capacity=len(el[0]))
    d.add(IONS, capacity=len(io[0]))
    d.set_particles(0, *el)
    d.set_particles(1, *io)
    samples = []
    for _ in range(STEPS):
        d.step(1)
        samples.append(d.get_field("e_z")[2:grid.nr + 2, 2 + Z_NODE].copy())
    f = _row_frequencies(samples, grid)
    assert np.abs(f - 1).max() <= FREQ_RTOL, f
