"""Charge continuity and Gauss's law through the C ABI diagnostics.

The Villasenor-Buneman deposit conserves charge exactly in the node shape of
pcg_node_charge; the double path must close Q(n+1) - Q(n) + dt div J = 0 to
rounding (RTOL_CONT_F64 = 1e-12 of the largest node charge), the float path
to float rounding of its current (RTOL_CONT_F32 = 2e-5).  Gauss's law
eps0 div E - Q keeps its value from step to step on the interior nodes
(the reference's Yee update leaves the outer walls and the axis-wall corner
untouched) to RTOL_GAUSS_F64 = 1e-12.  The node charge itself is checked
against a numpy restatement on the same particles.
"""
import numpy as np
import pytest

from tests.cases import ELECTRONS, IONS, near_axial, particles, small_grid

pytestmark = pytest.mark.gpu

RTOL_CONT_F64 = 1e-12
RTOL_CONT_F32 = 2e-5
RTOL_GAUSS_F64 = 1e-12
EPS0 = 8.85e-12


def _domain(precision, quirks="fixed", current="vb"):
    from picopic_b200 import Domain
    grid = small_grid(pml=False)
    d = Domain(grid, pusher="borisrel", current=current, precision=precision, quirks=quirks, seed=7)
    for sp in (ELECTRONS, IONS):
        d.add(sp, capacity=20000)
    for i, sp in enumerate((ELECTRONS, IONS)):
        d.set_particles(i, *particles(grid, 3000, 21 + i, mass=sp.mass,
                                      boost=30.0 if sp.mass == 1 else 150.0))
    return d, grid


def _numpy_charge(grid, d):
    q = np.zeros(grid.shape)
    for sid, charge in ((0, -1.6e-19), (1, 1.6e-19)):
        p = d.get_particles(sid)
        x, y = p["r"] / grid.dr, p["z"] / grid.dz
        i, k = np.floor(x).astype(int), np.floor(y).astype(int)
        fi = 0.5 + i * (i + 1) / (2 * x) - 0.5 * x
        b = y - k
        qw = charge * p["w"]
        for di, fr in ((0, fi), (1, 1 - fi)):
            for dk, fz in ((0, 1 - b), (1, b)):
                np.add.at(q, (i + di + 2, k + dk + 2), qw * fr * fz)
    return q


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_node_charge_matches_numpy(precision):
    d, grid = _domain(precision)
    d.step(2)
    q = d.node_charge()
    ref = _numpy_charge(grid, d)
    tol = 1e-13 if precision == "f64" else 1e-6
    assert np.abs(q - ref).max() <= tol * np.abs(ref).max()


@pytest.mark.parametrize("quirks", ["fixed", "reference"])
def test_continuity_f64(quirks):
    d, _ = _domain("f64", quirks)
    for _ in range(3):
        r = d.continuity_step()
        assert np.abs(r).max() <= RTOL_CONT_F64


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_continuity_near_axial_face_crossing(precision):
    """Radial steps of 1.2e-15 to 5e-15 m across a z face: the fixed mode's
    segment integrals (and the float path's shares) keep continuity where
    the reference's 1e-15 m segment threshold drops charge."""
    from picopic_b200 import Domain
    grid = small_grid(pml=False)
    d = Domain(grid, pusher="borisrel", current="vb", precision=precision, quirks="fixed", seed=7)
    d.add(ELECTRONS, capacity=4000)
    d.set_particles(0, *near_axial(grid, 2000, 5))
    r = d.continuity_step()
    assert np.abs(r).max() <= (RTOL_CONT_F64 if precision == "f64" else RTOL_CONT_F32)


def test_continuity_f32():
    d, _ = _domain("f32")
    for _ in range(3):
        r = d.continuity_step()
        assert np.abs(r).max() <= RTOL_CONT_F32


def test_gauss_law_is_kept_f64():
    d, grid = _domain("f64")
    g = []
    q_prev = d.node_charge()
    for _ in range(4):
        d.step(1)
        # E after a step was advanced with the current of the step before,
        # so it pairs with the charge before this step's move
        g.append(EPS0 * d.divergence("e") - q_prev)
        q_prev = d.node_charge()
    scale = np.abs(q_prev).max()
    inner = np.s_[3:-3, 3:-3]
    for a, b in zip(g, g[1:]):
        assert np.abs(b - a)[inner].max() <= RTOL_GAUSS_F64 * scale
