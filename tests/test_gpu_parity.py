"""The CUDA double-precision path against the CPU oracle.

Stage by stage (pcg_stage, one kernel per Domain method) and through the
fused step (pcg_step), for every pusher and current scheme, on seeded
inputs with random fields, fast particles (cell crossings, reflections,
removals), PML and beam injection.  Cell indices and particle counts must
be identical; fields and particle data agree to FP64 rounding (atomic sum
order and the last bit of log/pow differ): |gpu - cpu| <= RTOL * max|cpu|.
"""
import numpy as np
import pytest

from oracle.harness import FIELDS, STAGES, OracleSim
from tests.cases import ELECTRONS, IONS, beam_spec, load, small_grid

pytestmark = pytest.mark.gpu

RTOL_STAGE = 1e-12
RTOL_STEPS = 1e-9
COMBOS = [(p, c) for p in ("borisrel", "boris", "vay", "hc") for c in ("vb", "zigzag")]


def _gpu(grid, pusher, current, seed=7, precision="f64", quirks="reference"):
    from picopic_b200 import Domain
    return Domain(grid, pusher=pusher, current=current, precision=precision, quirks=quirks,
                  seed=seed)


def _close(a, b, rtol, what):
    scale = max(np.abs(b).max(), 1e-300)
    err = np.abs(a - b).max() / scale if a.size else 0.0
    assert err <= rtol, f"{what}: max rel err {err:.3e}"


def _compare(gpu, orc, nsp, rtol, where):
    fg, fo = gpu.fields(), orc.fields()
    for k in FIELDS:
        _close(fg[k], fo[k], rtol, f"{where} field {k}")
    for sid in range(nsp):
        pg, po = gpu.get_particles(sid), orc.get_particles(sid)
        assert pg["r"].size == po["r"].size, f"{where} species {sid} count"
        np.testing.assert_array_equal(pg["cell_r"], po["cell_r"], err_msg=f"{where} cell_r")
        np.testing.assert_array_equal(pg["cell_z"], po["cell_z"], err_msg=f"{where} cell_z")
        for k in ("r", "z", "vr", "vphi", "vz", "w"):
            _close(pg[k], po[k], rtol, f"{where} species {sid} {k}")


@pytest.mark.parametrize("pusher,current", COMBOS)
def test_stagewise(pusher, current):
    grid = small_grid()
    species = [ELECTRONS, IONS, beam_spec(grid)]
    gpu, orc = _gpu(grid, pusher, current), OracleSim(grid, pusher, current)
    for sp in species:
        gpu.add(sp, capacity=20000)
        orc.add(sp)
    load_pairs(gpu, orc, grid, species, n=2000, seed=11)
    orc.set_rng("philox", 7)
    for step in range(2):
        for st in STAGES:
            gpu.stage(st)
            assert orc.stage(st) == 0
            if step == 0 and st in ("field_e", "field_h", "push", "reflect", "bind", "current"):
                _compare(gpu, orc, len(species), RTOL_STAGE, f"step {step} after {st}")
    _compare(gpu, orc, len(species), RTOL_STAGE * 100, "after 2 staged steps")
    assert gpu.count(2) == orc.count(2) > 0


@pytest.mark.parametrize("pusher,current", COMBOS)
def test_fused_steps(pusher, current):
    grid = small_grid()
    species = [ELECTRONS, IONS, beam_spec(grid)]
    gpu, orc = _gpu(grid, pusher, current), OracleSim(grid, pusher, current)
    for sp in species:
        gpu.add(sp, capacity=20000)
        orc.add(sp)
    load_pairs(gpu, orc, grid, species, n=3000, seed=3)
    orc.set_rng("philox", 7)
    gpu.step(1)
    assert orc.step(1) == 0
    _compare(gpu, orc, len(species), RTOL_STAGE * 10, "after 1 step")
    gpu.step(9)
    assert orc.step(9) == 0
    _compare(gpu, orc, len(species), RTOL_STEPS, "after 10 steps")
    assert gpu.removed == orc.removed


def test_strict_axial_overwrite_is_reproduced():
    """Beam particles with v_r = v_phi = 0 in zero fields move strictly
    along z; the reference then overwrites J_r at two nodes
    (currentVB.cpp:545-546), wiping earlier particles' J_r there."""
    grid = small_grid(pml=False)
    species = [ELECTRONS, beam_spec(grid)]
    gpu, orc = _gpu(grid, "borisrel", "vb"), OracleSim(grid, "borisrel", "vb")
    for sp in species:
        gpu.add(sp, capacity=20000)
        orc.add(sp)
    from tests.cases import particles
    p = particles(grid, 3000, 5)
    gpu.set_particles(0, *p)
    orc.set_particles(0, *p)
    orc.set_rng("philox", 7)
    gpu.step(1)
    orc.step(1)
    _compare(gpu, orc, 2, RTOL_STAGE * 10, "after 1 step from zero fields")
    jr_all = orc.get_field("j_r")
    assert np.count_nonzero(jr_all) > 0


@pytest.mark.parametrize("staged", [False, True])
def test_wall_reflections(staged):
    """Particles aimed at all four walls (specieP.cpp:493-607), including
    corners, so that every branch of the reflection loop runs."""
    grid = small_grid(pml=False)
    rng = np.random.default_rng(17)
    n = 4000
    dr, dz = grid.dr, grid.dz
    side = rng.integers(0, 4, n)
    r = dr / 2 + rng.random(n) * (grid.radius - dr)
    z = dz / 2 + rng.random(n) * (grid.longitude - dz)
    d = rng.random(n) * 0.1
    r = np.where(side == 0, dr * (0.5 + d), np.where(side == 1, grid.radius - dr * (0.5 + d), r))
    z = np.where(side == 2, dz * (0.5 + d), np.where(side == 3, grid.longitude - dz * (0.5 + d), z))
    corner = rng.random(n) < 0.2
    z = np.where(corner & (side < 2), dz * (0.5 + d), z)
    v = rng.normal(size=(3, n))
    v *= (rng.random(n) * 2.5e8 / np.linalg.norm(v, axis=0))  # |v| < 0.84 c
    sgn = np.where(side % 2 == 0, -1.0, 1.0)
    v[0] = np.where(side < 2, sgn * np.abs(v[0]), v[0])
    v[2] = np.where(side >= 2, sgn * np.abs(v[2]), v[2])
    v[2] = np.where(corner & (side < 2), -np.abs(v[2]), v[2])
    w = np.full(n, 1e5)
    gpu, orc = _gpu(grid, "borisrel", "vb"), OracleSim(grid, "borisrel", "vb")
    for s in (gpu, orc):
        s.add(ELECTRONS, capacity=n) if s is gpu else s.add(ELECTRONS)
        s.set_particles(0, r, z, v[0], v[1], v[2], w)
    if staged:
        for st in STAGES:
            gpu.stage(st)
            orc.stage(st)
    else:
        gpu.step(1)
        orc.step(1)
    pg, po = gpu.get_particles(0), orc.get_particles(0)
    flipped = np.sum(np.sign(po["vz"]) != np.sign(v[2])) + np.sum(np.sign(po["vr"]) != np.sign(v[0]))
    assert flipped > n // 4, "the case must exercise the walls"
    _compare(gpu, orc, 1, RTOL_STAGE * 10, "after wall reflections")


def test_removed_particles_and_errors():
    grid = small_grid(nr=12, nz=24)
    gpu, orc = _gpu(grid, "borisrel", "vb"), OracleSim(grid, "borisrel", "vb")
    for s in (gpu, orc):
        s.add(ELECTRONS)
    # a particle one cell outside the z=L wall is removed by the collector
    r = np.array([5e-4, 5e-4, 6e-4])
    z = np.array([5e-4, grid.longitude + 0.5 * grid.dz, 7e-4])
    zero = np.zeros(3)
    for s in (gpu, orc):
        s.set_particles(0, r, z, zero, zero, zero, np.ones(3))
    gpu.step(1)
    orc.step(1)
    assert gpu.count(0) == orc.count(0)


def test_nan_position_is_an_error():
    from picopic_b200 import PcgError
    grid = small_grid(pml=False)
    gpu = _gpu(grid, "borisrel", "vb")
    gpu.add(ELECTRONS)
    gpu.set_particles(0, [np.nan, 5e-4], [5e-4, 5e-4], [0, 0], [0, 0], [0, 0], [1, 1])
    with pytest.raises(PcgError) as e:
        gpu.step(1)
        gpu.synchronize()
    assert e.value.code == -10


def test_step_status_reports_each_step_a_step_late():
    """pcg_step_status returns the status queued by the previous call: a
    NaN position raised in step 1 shows at the status read after step 2,
    and a clean run reads clean throughout."""
    from picopic_b200 import PcgError
    grid = small_grid(pml=False)
    clean = _gpu(grid, "borisrel", "vb")
    clean.add(ELECTRONS)
    clean.set_particles(0, [5e-4, 6e-4], [5e-4, 5e-4], [0, 0], [0, 0], [0, 0], [1, 1])
    for _ in range(3):
        clean.step(1)
        clean.step_status()
    clean.synchronize()
    gpu = _gpu(grid, "borisrel", "vb")
    gpu.add(ELECTRONS)
    gpu.set_particles(0, [np.nan, 5e-4], [5e-4, 5e-4], [0, 0], [0, 0], [0, 0], [1, 1])
    gpu.step(1)
    gpu.step_status()  # nothing queued before: clean
    gpu.step(1)
    with pytest.raises(PcgError) as e:
        gpu.step_status()  # the block copied after step 1
    assert e.value.code == -10


def load_pairs(gpu, orc, grid, species, n, seed):
    from tests.cases import particles, random_fields
    for i, sp in enumerate(species):
        if sp.beam is None:
            p = particles(grid, n, seed + i, mass=sp.mass, boost=30.0 if sp.mass == 1 else 150.0)
            gpu.set_particles(i, *p)
            orc.set_particles(i, *p)
    for name, a in random_fields(grid, seed).items():
        gpu.set_field(name, a)
        orc.set_field(name, a)
