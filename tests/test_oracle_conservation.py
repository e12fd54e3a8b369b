"""The conservation identities behind pcg_node_charge / pcg_divergence,
checked on the CPU oracle (which reproduces the reference bit for bit).

Charge continuity: with the node shape of the Villasenor-Buneman deposit
(radial share 1/2 + i(i+1)/(2x) - x/2 of node i for a particle at x = r/dr
in cell i, linear axial shares) and the Yee face areas A(i) = 2 pi (i+1/2)
dr dz, S(i) = 2 pi i dr^2 (pi dr^2/4 on the axis), Q(n+1) - Q(n) +
dt div J = 0 on every real node to double rounding.  Gauss: eps0 div E - Q
keeps its value on interior nodes (the reference leaves the outer walls and
the axis-wall corner out of its E update).
"""
import numpy as np
import pytest

from oracle.harness import OracleSim
from tests.cases import ELECTRONS, IONS, near_axial, particles, small_grid

PI = 3.1415926535897932
EPS0 = 8.85e-12


def node_charge(grid, sim, species):
    q = np.zeros(grid.shape)
    for sid, sp in enumerate(species):
        p = sim.get_particles(sid)
        x, y = p["r"] / grid.dr, p["z"] / grid.dz
        i, k = np.floor(x).astype(int), np.floor(y).astype(int)
        fi = 0.5 + i * (i + 1) / (2 * x) - 0.5 * x
        b = y - k
        qw = sp.charge * 1.6e-19 * p["w"]
        for di, fr in ((0, fi), (1, 1 - fi)):
            for dk, fz in ((0, 1 - b), (1, b)):
                np.add.at(q, (i + di + 2, k + dk + 2), qw * fr * fz)
    return q


def divergence(grid, fr, fz):
    i = np.arange(-2, grid.nr + 2)[:, None].astype(float)
    a = 2 * PI * (i + 0.5) * grid.dr * grid.dz
    s = np.where(i > 0, 2 * PI * i * grid.dr ** 2, np.where(i == 0, PI * grid.dr ** 2 / 4, 0.0))
    d = np.zeros(grid.shape)
    d[1:, :] += fr[1:, :] * a[1:] - fr[:-1, :] * a[:-1]
    d[:, 1:] += (fz[:, 1:] - fz[:, :-1]) * s
    return d


def _sim(quirks):
    grid = small_grid(pml=False)
    sim = OracleSim(grid, "borisrel", "vb", quirks=quirks)
    species = [ELECTRONS, IONS]
    for sp in species:
        sim.add(sp)
    for i, sp in enumerate(species):
        sim.set_particles(i, *particles(grid, 3000, 21 + i, mass=sp.mass,
                                        boost=30.0 if sp.mass == 1 else 150.0))
    return grid, sim, species


@pytest.mark.parametrize("quirks", ["fixed", "reference"])
def test_oracle_charge_continuity(quirks):
    grid, sim, species = _sim(quirks)
    for _ in range(3):
        q0 = node_charge(grid, sim, species)
        assert sim.step(1) == 0
        q1 = node_charge(grid, sim, species)
        r = q1 - q0 + grid.dt * divergence(grid, sim.get_field("j_r"), sim.get_field("j_z"))
        assert np.abs(r[2:-2, 2:-2]).max() <= 1e-13 * np.abs(q1).max()
        assert np.abs(q1 - q0).max() > 1e-3 * np.abs(q1).max(), "the case must move charge"


def test_oracle_gauss_law_is_kept():
    grid, sim, species = _sim("fixed")
    g, q_prev = [], node_charge(grid, sim, species)
    for _ in range(4):
        assert sim.step(1) == 0
        g.append(EPS0 * divergence(grid, sim.get_field("e_r"), sim.get_field("e_z")) - q_prev)
        q_prev = node_charge(grid, sim, species)
    inner = np.s_[3:-3, 3:-3]
    for a, b in zip(g, g[1:]):
        assert np.abs(b - a)[inner].max() <= 1e-13 * np.abs(q_prev).max()


@pytest.mark.parametrize("quirks", ["fixed", "reference"])
def test_oracle_near_axial_face_crossing(quirks):
    """A nearly axial particle that crosses a z face: the reference drops the
    sub-segment behind the face when it moves less than 1e-15 m radially
    (currentVB.cpp:45-46), J_z included; the fixed mode's form of the segment
    integrals has no such threshold and closes continuity to rounding."""
    grid = small_grid(pml=False)
    sim = OracleSim(grid, "borisrel", "vb", quirks=quirks)
    sim.add(ELECTRONS)
    sim.set_particles(0, *near_axial(grid, 2000, 5))
    q0 = node_charge(grid, sim, [ELECTRONS])
    assert sim.step(1) == 0
    q1 = node_charge(grid, sim, [ELECTRONS])
    r = q1 - q0 + grid.dt * divergence(grid, sim.get_field("j_r"), sim.get_field("j_z"))
    rel = np.abs(r[2:-2, 2:-2]).max() / np.abs(q1).max()
    if quirks == "fixed":
        assert rel <= 1e-13
    else:
        assert rel > 1e-3, "the reference's dropped segments must show"
