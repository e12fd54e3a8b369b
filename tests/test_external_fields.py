"""External fields (ExternalFields, src/maxwellSolver/externalFields.cpp)
in the CPU oracle, against the reference built with ENABLE_EXTERNAL_FIELDS.

The pushers add the gathered external E and H to the solver's
(pusherBoris.cpp:62-65, pusherVay.cpp:48-50, pusherHC.cpp:51-54); the fields
are set after every H update (SMB.cpp:1253-1262).  The reference's electric
name test (externalFields.cpp:51-62) never selects a profile that sets a
field; of its magnetic profiles only const_z sets one (:298-348).
"""
import numpy as np
import pytest

from oracle.harness import FIELDS, STAGES, OracleSim, RefSim, reference_available
from tests.cases import ELECTRONS, IONS, beam_spec, load, small_grid

COMBOS = [("borisrel", "vb"), ("vay", "zigzag")]
H_EXT = 2e5   # A/m: mu0 H = 0.25 T, an electron turns ~4e-3 rad per step of 1e-13 s
E_EXT = 3e6   # V/m


def _same(o, r, nsp, where):
    fo, fr = o.fields(), r.fields()
    for k in FIELDS:
        np.testing.assert_array_equal(fo[k], fr[k], err_msg=f"{where}: field {k}")
    for sid in range(nsp):
        po, pr = o.get_particles(sid), r.get_particles(sid)
        for k in po:
            np.testing.assert_array_equal(po[k], pr[k], err_msg=f"{where}: species {sid} {k}")


@pytest.mark.parametrize("pusher,current", COMBOS)
@pytest.mark.parametrize("electric", ["none", "const_z"])
def test_stagewise_bit_exact_with_external_fields(pusher, current, electric):
    if not reference_available(pusher, current, extf=True):
        pytest.skip("compiled reference with external fields not built (oracle/Makefile.ref)")
    grid = small_grid()
    species = [ELECTRONS, IONS, beam_spec(grid)]
    o, r = OracleSim(grid, pusher, current), RefSim(grid, pusher, current, extf=True)
    for sim in (o, r):
        assert sim.set_external_fields(electric, [E_EXT], "const_z", [H_EXT]) == 0
        load(sim, grid, species, 2000, seed=11)
    o.set_rng("mt19937", 42)
    r.seed(42)
    for step in range(3):
        for st in STAGES:
            assert o.stage(st) == r.stage(st) == 0, st
        _same(o, r, len(species), f"after step {step}")


def test_external_magnetic_field_turns_particles():
    """H_z = const bends the electrons: after a few steps their velocities
    differ from a run without it, and v_r^2 + v_phi^2 changes little."""
    grid = small_grid(pml=False)
    out = []
    for h in (0.0, H_EXT):
        o = OracleSim(grid)
        if h:
            assert o.set_external_fields("none", [], "const_z", [h]) == 0
        load(o, grid, [ELECTRONS], 500, seed=3)
        o.step(4)
        out.append(o.get_particles(0))
    a, b = out
    assert np.abs(a["vr"] - b["vr"]).max() > 1e-3 * np.abs(a["vr"]).max()


def test_reference_semantics_of_the_profile_names():
    grid = small_grid(pml=False)
    o = OracleSim(grid)
    assert o.set_external_fields("none", [], "no_such_profile", [1.0]) == -1   # the reference's FATAL
    assert o.set_external_fields("no_such_profile", [1.0], "none", []) == 0    # its electric test never fails
    f = OracleSim(grid, quirks="fixed")
    assert f.set_external_fields("no_such_profile", [1.0], "none", []) == -1
    assert f.set_external_fields("linerad_z", [1.0], "none", []) == -13
    assert f.set_external_fields("const_z", [], "none", []) == -1              # needs its amplitude


def test_fixed_mode_applies_the_electric_field():
    """PCG_QUIRKS_FIXED applies const_z of the electric field: electrons at
    rest accelerate against E_z, and a magnetic const_r is applied too."""
    grid = small_grid(pml=False)
    o = OracleSim(grid, quirks="fixed")
    assert o.set_external_fields("const_z", [E_EXT], "none", []) == 0
    o.add(ELECTRONS)
    n = 64
    rng = np.random.default_rng(1)
    r = grid.dr * (2 + rng.random(n) * (grid.nr - 4))
    z = grid.dz * (2 + rng.random(n) * (grid.nz - 4))
    o.set_particles(0, r, z, np.zeros(n), np.zeros(n), np.zeros(n), np.ones(n))
    o.stage("push")
    p = o.get_particles(0)
    assert (p["vz"] < 0).all()  # q E dt / m with q < 0
    dv = 1.6e-19 * E_EXT * grid.dt / 9.1e-31
    np.testing.assert_allclose(p["vz"], -dv, rtol=1e-6)
