"""The ensemble (pcg_ensemble_*): independent runs stepped together from
several host threads give what each run gives stepped alone (same seeds;
fields and particles within RTOL = 1e-10 of each array's maximum on the
double path, where only the order of the deposit's atomic sums differs),
and the autotuner picks a candidate tiling for the runs and leaves them
stepping (float path, particle counts and particle-steps exact).  The same
holds in graph mode, where a batch of steps of all runs is captured into
one CUDA graph and issued as one launch: double path within RTOL of the
runs alone, float path with its beam injecting (captured counts and
re-sorts) within float rounding of the direct ensemble and with exact
particle counts."""
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


@pytest.mark.parametrize("graph", [False, True])
def test_ensemble_matches_runs_alone(graph):
    from picopic_b200.ensemble import Ensemble
    alone = [_run(g, "f64", 10 + k) for k, g in enumerate(_grids())]
    for d in alone:
        d.step(6)
    runs = [_run(g, "f64", 10 + k) for k, g in enumerate(_grids())]
    ens = Ensemble(runs, threads=3)
    if graph:
        ens.set_graph(True)
        assert ens.step(1) > 0  # the first batch steps directly
        assert ens.step(2) > 0  # captured
        nodes, _ = ens.graph_info()
        assert nodes >= 2 * len(runs) * 3  # every run's E, H and particle kernels of both steps
        ms = ens.step(3)        # the same shape: the graph updated in place
    else:
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


def _beam_run(grid, seed):
    """A float run with a beam injecting every step (device Philox), so that
    each captured step has its own particle counts and the beam's first tile
    sort falls inside a capture."""
    from picopic_b200 import Domain
    from tests.cases import beam_spec
    d = Domain(grid, pusher="borisrel", current="vb", precision="f32", quirks="fixed", seed=seed)
    for sp in (ELECTRONS, IONS):
        d.add(sp, capacity=20000)
    d.add(beam_spec(grid), capacity=20000)
    for i, sp in enumerate((ELECTRONS, IONS)):
        d.set_particles(i, *particles(grid, 4000, seed + i, mass=sp.mass,
                                      boost=30.0 if sp.mass == 1 else 150.0))
    return d


def test_graph_ensemble_float_with_beams_matches_direct():
    from picopic_b200.ensemble import Ensemble
    grids = [small_grid(nr=16, nz=64, pml=False), small_grid(nr=24, nz=64, pml=False)]
    direct = [_beam_run(g, 40 + k) for k, g in enumerate(grids)]
    ens_d = Ensemble(direct, threads=1)
    ens_d.step(1)
    ens_d.step(7)
    graphed = [_beam_run(g, 40 + k) for k, g in enumerate(grids)]
    ens_g = Ensemble(graphed, threads=1)
    ens_g.set_graph(True)
    ens_g.step(1)
    ens_g.step(3)
    ens_g.step(4)
    for a, b in zip(direct, graphed):
        da, db = a.diag(), b.diag()
        assert da.particles == db.particles and da.particle_steps == db.particle_steps
        assert len(a.get_particles(2)["r"]) == len(b.get_particles(2)["r"]) > 0
        for k in ("e_r", "e_z", "h_phi", "j_z"):
            fa, fb = a.get_field(k), b.get_field(k)
            assert np.abs(fa - fb).max() <= 1e-4 * max(np.abs(fa).max(), 1e-300), k
