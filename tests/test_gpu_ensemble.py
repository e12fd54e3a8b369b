"""The ensemble (pcg_ensemble_*): independent runs stepped together from
several host threads give what each run gives stepped alone (same seeds;
fields and particles within RTOL = 1e-10 of each array's maximum on the
double path, where only the order of the deposit's atomic sums differs),
and the autotuner picks a candidate tiling for the runs and leaves them
stepping (float path, particle counts and particle-steps exact)."""
import numpy as np
import pytest

from tests.cases import ELECTRONS, IONS, particles, small_grid

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def _run(grid, precision, seed):
    from picopic_b200 import Domain
    d = Domain(grid, pusher="borisrel", current="vb", precision=precision, quirks="fixed", seed=seed)
    for sp in (ELECTRONS, IONS):
        d.add(sp, capacity=20000)
    for i, sp in enumerate((ELECTRONS, IONS)):
        d.set_particles(i, *particles(grid, 4000, seed + i, mass=sp.mass,
                                      boost=30.0 if sp.mass == 1 else 150.0))
    return d


def _grids():
    return [small_grid(nr=16, nz=32, pml=False), small_grid(nr=24, nz=64, pml=False),
            small_grid(nr=8, nz=48, pml=False)]


def test_ensemble_matches_runs_alone():
    from picopic_b200.ensemble import Ensemble
    alone = [_run(g, "f64", 10 + k) for k, g in enumerate(_grids())]
    for d in alone:
        d.step(6)
    runs = [_run(g, "f64", 10 + k) for k, g in enumerate(_grids())]
    ens = Ensemble(runs, threads=3)
    ms = ens.step(6)
    assert ms > 0
    for a, b in zip(alone, runs):
        for k in ("e_r", "e_z", "h_phi", "j_r", "j_z"):
            fa, fb = a.get_field(k), b.get_field(k)
            assert np.abs(fa - fb).max() <= RTOL * max(np.abs(fa).max(), 1e-300), k
        for sid in (0, 1):
            pa, pb = a.get_particles(sid), b.get_particles(sid)
            assert len(pa["r"]) == len(pb["r"])
            for k in ("r", "z", "vr", "vz"):
                assert np.abs(pa[k] - pb[k]).max() <= RTOL * np.abs(pa[k]).max(), (sid, k)


def test_autotune_then_step():
    from picopic_b200.ensemble import CANDIDATES, Ensemble
    runs = [_run(g, "f32", 20 + k) for k, g in enumerate(_grids())]
    ens = Ensemble(runs, threads=2)
    assert ens.autotune(trial_steps=2) in CANDIDATES
    before = [(d.diag().particle_steps, d.diag().particles) for d in runs]
    ens.step(4)
    for d, (ps, n) in zip(runs, before):
        dg = d.diag()
        assert dg.particles == n  # closed walls: nothing leaves
        assert dg.particle_steps == ps + 4 * n
