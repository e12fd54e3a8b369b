"""External fields on the GPU against the CPU oracle (which the reference
built with ENABLE_EXTERNAL_FIELDS pins bit for bit, tests/test_external_fields.py).

Double path: fused steps within the parity tolerances of test_gpu_parity.py
(the external gather is added as the reference adds it).  Float path: the
step gathers E + E_ext and H + H_ext summed in float, within the float
tolerances of test_gpu_f32.py.
"""
import numpy as np
import pytest

from oracle.harness import FIELDS, OracleSim
from tests.cases import ELECTRONS, IONS, beam_spec, particles, random_fields, small_grid

pytestmark = pytest.mark.gpu

H_EXT = 2e5
E_EXT = 3e6
CASES = [("reference", "const_z", "const_z"), ("fixed", "const_z", "const_z"), ("fixed", "const_r", "const_phi")]


def _pair(grid, pusher, current, quirks, precision, electric, magnetic, n=3000, seed=3):
    from picopic_b200 import Domain
    species = [ELECTRONS, IONS, beam_spec(grid)]
    gpu = Domain(grid, pusher=pusher, current=current, precision=precision, quirks=quirks, seed=7)
    orc = OracleSim(grid, pusher, current, quirks=quirks)
    for sim in (gpu, orc):
        sim.set_external_fields(electric, [E_EXT], magnetic, [H_EXT])
    for sp in species:
        gpu.add(sp, capacity=20000)
        orc.add(sp)
    for i, sp in enumerate(species):
        if sp.beam is None:
            p = particles(grid, n, seed + i, mass=sp.mass, boost=30.0 if sp.mass == 1 else 150.0)
            gpu.set_particles(i, *p)
            orc.set_particles(i, *p)
    # random fields as in test_gpu_f32.py: they also turn the beam off the
    # strict-axial path, whose J_r overwrite quirk the float path leaves out
    for name, a in random_fields(grid, seed).items():
        gpu.set_field(name, a)
        orc.set_field(name, a)
    orc.set_rng("philox", 7)
    return gpu, orc, len(species)


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300) if a.size else 0.0


@pytest.mark.parametrize("quirks,electric,magnetic", CASES)
@pytest.mark.parametrize("pusher,current", [("borisrel", "vb"), ("vay", "zigzag")])
def test_f64_fused_steps(pusher, current, quirks, electric, magnetic):
    grid = small_grid()
    gpu, orc, nsp = _pair(grid, pusher, current, quirks, "f64", electric, magnetic)
    gpu.step(10)
    assert orc.step(10) == 0
    for k in FIELDS:
        assert _rel(gpu.get_field(k), orc.get_field(k)) <= 1e-9, k
    for sid in range(nsp):
        pg, po = gpu.get_particles(sid), orc.get_particles(sid)
        np.testing.assert_array_equal(pg["cell_r"], po["cell_r"])
        np.testing.assert_array_equal(pg["cell_z"], po["cell_z"])
        for k in ("r", "z", "vr", "vphi", "vz"):
            assert _rel(pg[k], po[k]) <= 1e-9, (sid, k)


@pytest.mark.parametrize("quirks,electric,magnetic", CASES)
def test_f32_one_step(quirks, electric, magnetic):
    grid = small_grid()
    gpu, orc, nsp = _pair(grid, "borisrel", "vb", quirks, "f32", electric, magnetic)
    gpu.step(1)
    assert orc.step(1) == 0
    for k in FIELDS:
        assert _rel(gpu.get_field(k), orc.get_field(k)) <= 2e-4, k
    for sid in range(nsp):
        pg, po = gpu.get_particles(sid), orc.get_particles(sid)
        assert pg["r"].size == po["r"].size
        assert _rel(pg["r"], po["r"]) <= 1e-6 and _rel(pg["z"], po["z"]) <= 1e-6
        for k in ("vr", "vphi", "vz"):
            assert _rel(pg[k], po[k]) <= 1e-5, (sid, k)


def test_external_field_changes_the_run_and_can_be_removed():
    from picopic_b200 import Domain
    grid = small_grid(pml=False)
    out = []
    for ext in (False, True, "removed"):
        d = Domain(grid, precision="f32", quirks="reference", seed=7)
        d.add(ELECTRONS, capacity=5000)
        d.set_particles(0, *particles(grid, 3000, 5, boost=30.0))
        if ext:
            d.set_external_fields("none", [], "const_z", [H_EXT])
        if ext == "removed":
            d.set_external_fields("none", [], "none", [])
        d.step(3)
        out.append(d.get_particles(0))
    assert np.abs(out[0]["vr"] - out[1]["vr"]).max() > 1e-3 * np.abs(out[0]["vr"]).max()
    np.testing.assert_array_equal(out[0]["vr"], out[2]["vr"])
