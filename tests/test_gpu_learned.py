"""The learned collision step against its CPU restatement and the binary
operator (the committed model picopic_b200/models/collision_p12.npz).

* Features: pcg_cell_features equals the float64 restatement of
  oracle/learned_oracle.py from the same cell moments to RTOL_FEAT = 1e-5
  (they are stored as float).
* The moment-matching transform: after one learned step every cell on the
  learned path keeps each species' momentum and its kinetic energy to
  RTOL_CONS = 1e-12 (FP64 layout), and its new axis temperatures are the
  restated T' = T + T_m S y of the network outputs (within 1e-4 of T: the
  host and device feed the BF16 network features rounded differently).
* Relaxation: the electron anisotropy relaxation time at a bi-Maxwellian
  start (the rate of the first step; the binary estimate averaged over 800
  passes, standard error 0.3-0.6 %) matches the binary operator's within 1 %
  at 3e20 m^-3, Te 2/1 eV (measured 0.6 %) and within 2.5 % at the hotter
  denser and the colder states (measured +1.6 % and -1.9 %): the 1 % target
  holds there as a strict expected failure.  Over a whole relaxation (the
  e-folding time fitted down to 1/e) the binary operator slows as its cold
  core isotropises before its tails, which a transform of second moments
  does not follow: the learned time is 18-20 % shorter (the strict expected
  failure of 1 %, and a test of the measured band).
* What the network gains: the learned step is at least 5x faster than the
  binary pass at the same relaxation time.
* Cells outside the training box (widened by 25 %) take the binary operator.
* The wide model (8-200 macroparticles per cell, n down to 1e16 m^-3) takes
  cells of 12 macroparticles per species on the learned path and matches
  the binary relaxation time there to 1 % plus three standard errors.
"""
import functools

import numpy as np
import pytest

from oracle.learned_oracle import features, transform_scales

pytestmark = pytest.mark.gpu

RTOL_FEAT = 1e-5
RTOL_CONS = 1e-12
ME = 9.1e-31


def _grid(nr=32, nz=64, dt=1e-13):
    from picopic_b200 import Geometry
    dr = 1e-5
    return Geometry(nr, nz, nr * dr, nz * dr, dt)


def _random_domain(grid, seed=3, precision="f64", scheme=None):
    """Random learned-box cell states; scheme (pusher, current, quirks) in
    place of the default relativistic Boris, VB, fixed quirks."""
    from picopic_b200 import learned as L
    from picopic_b200 import Domain
    rng = np.random.default_rng(seed)
    te, ti, dens, drift, ppc = L.cell_states(grid, rng, L.Sampling())
    pe = L.cell_particles(grid, rng, te, dens[0], drift, ppc[0], 1.0)
    pi = L.cell_particles(grid, rng, ti, dens[1], np.zeros_like(drift), ppc[1], L.MASS_ION)
    cap = max(pe[0].size, pi[0].size) + 16
    if scheme is None:
        d = L._domain(grid, 0, seed, capacity=cap, precision=precision)
    else:
        d = Domain(grid, pusher=scheme[0], current=scheme[1], precision=precision, quirks=scheme[2], seed=seed)
        d.add(L.ELECTRONS, capacity=cap)
        d.add(L.IONS, capacity=cap)
    d.set_particles(0, *pe)
    d.set_particles(1, *pi)
    if precision == "f32":  # group the slots by tile, as steps keep them
        d.tile_sort(0)
        d.tile_sort(1)
    return d


def test_features_match_restatement():
    g = _grid()
    d = _random_domain(g)
    x, S = d.cell_features()
    xo, So, _ = features(d.cell_moments(), g, g.dt, (ME, 1836 * ME), (-1.6e-19, 1.6e-19))
    ok = np.isfinite(xo).all(1)
    assert ok.mean() > 0.99 and np.array_equal(np.isfinite(x).all(1), ok)
    assert np.abs(x[ok] - xo[ok]).max() <= RTOL_FEAT * np.abs(xo[ok]).max()
    assert np.abs(S - So).max() <= 1e-12 * So.max()


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_learned_step_conserves_and_matches_transform(precision):
    from picopic_b200 import learned as L
    from picopic_b200.mlp import Mlp
    g = _grid()
    d = _random_domain(g, seed=4, precision=precision)
    params, norm = L.load_model()
    d.set_collision_model(params, norm)
    m0 = d.cell_moments()
    x, S, state = features(m0, g, g.dt, (ME, 1836 * ME), (-1.6e-19, 1.6e-19))
    net = Mlp(seed=0)
    net.params = params
    xs = np.nan_to_num((x - norm[:13]) / norm[13:26]).astype(np.float32)
    y = net.forward(xs) * norm[32:38] + norm[26:32]
    learned, fallback = d.collide_learned()
    assert learned > 0.9 * g.nr * g.nz
    m1 = d.cell_moments()
    T1, _ = L.temperatures(m1)
    # cells on the learned path: their new temperatures are the restated ones
    T0 = state[0]
    expect = T0 * transform_scales(y.astype(np.float64), S, state) ** 2
    with np.errstate(invalid="ignore"):
        rel = np.abs(T1 - expect).max((1, 2)) / np.abs(T0).max((1, 2))
    on = np.isfinite(rel) & (rel <= 1e-4)  # BF16 network: outputs agree to ~1e-3 of y, y S ~ 1e-4
    assert on.sum() >= learned
    # per cell: each species' momentum and the total kinetic energy unchanged
    # (to FP64 rounding; the float layout stores the new velocities in FP32)
    rtol = RTOL_CONS if precision == "f64" else 1e-6
    for l in (0, 1):
        dp = np.abs(m1[on, 8 * l + 2:8 * l + 5] - m0[on, 8 * l + 2:8 * l + 5]).max(1)
        scale = np.sqrt(m0[on, 8 * l + 1] * m0[on, 8 * l + 5:8 * l + 8].sum(1))
        assert (dp <= rtol * scale).all()
    e0 = ME * m0[on, 5:8].sum(1) + 1836 * ME * m0[on, 13:16].sum(1)
    e1 = ME * m1[on, 5:8].sum(1) + 1836 * ME * m1[on, 13:16].sum(1)
    assert (np.abs(e1 - e0) <= rtol * e0).all()


# (density, electron T_par/T_perp eV, ion T eV)
STATE_MET = (3e20, (2.0, 1.0), 0.5)
STATES_OFF = ((1e21, (3.0, 1.5), 1.0), (3e20, (1.0, 0.5), 0.25))


@functools.lru_cache(maxsize=None)
def _initial_ratio(state):
    from picopic_b200 import learned as L
    g = _grid(64, 128)
    n, te, ti = state
    tb, eb, _ = L.initial_relaxation_time(g, "binary", passes=800, density=n, te=te, ti=ti)
    tl, _, _ = L.initial_relaxation_time(g, "learned", passes=1, density=n, te=te, ti=ti)
    assert eb / tb < 0.006  # the binary estimate's standard error
    return tl / tb


def test_initial_relaxation_time_within_1pct():
    assert abs(_initial_ratio(STATE_MET) - 1) <= 0.01


@pytest.mark.parametrize("state", STATES_OFF)
def test_initial_relaxation_time_within_2p5pct(state):
    assert abs(_initial_ratio(state) - 1) <= 0.025


@pytest.mark.xfail(strict=True, reason="measured +1.6 % and -1.9 % at these states")
@pytest.mark.parametrize("state", STATES_OFF)
def test_initial_relaxation_time_within_1pct_off_states(state):
    assert abs(_initial_ratio(state) - 1) <= 0.01


@functools.lru_cache(maxsize=None)
def _curve_ratio():
    """Learned / binary e-folding time of the anisotropy fitted over a decay
    to 1/e at 3e20 m^-3, Te 2/1 eV (about 1000 collision steps)."""
    from picopic_b200 import learned as L
    g = _grid(64, 128)
    n, te, ti = STATE_MET
    passes = 1050
    s1, v1, _ = L.anisotropy_run(g, "binary", passes, density=n, te=te, ti=ti)
    s2, v2, _ = L.anisotropy_run(g, "learned", passes, density=n, te=te, ti=ti)
    return L.relaxation_time(s2, v2, np.exp(-1)) / L.relaxation_time(s1, v1, np.exp(-1))


def test_full_relaxation_time_band():
    assert 0.75 <= _curve_ratio() <= 0.9  # measured 0.82


@pytest.mark.xfail(strict=True, reason="a second-moment transform misses the core-before-tail slow-down (0.82)")
def test_full_relaxation_time_within_1pct():
    assert abs(_curve_ratio() - 1) <= 0.01


def test_learned_step_is_faster_than_binary():
    from picopic_b200 import learned as L
    g = _grid(128, 256)
    _, _, sb = L.initial_relaxation_time(g, "binary", passes=6, density=3e20)
    _, _, sl = L.initial_relaxation_time(g, "learned", passes=6, density=3e20)
    assert sb / sl >= 5.0


def test_out_of_box_cells_take_the_binary_operator():
    """Electrons streaming at four times sqrt(T_e/m_e) through the ions are
    far outside the training states (drift up to 0.1 thermal speeds)."""
    from picopic_b200 import learned as L
    g = _grid(16, 32)
    rng = np.random.default_rng(1)
    cells = g.nr * g.nz
    te = np.full((cells, 3), 1.0)
    drift = np.zeros((cells, 3))
    drift[:, 2] = 4 * np.sqrt(1.6e-19 / ME)
    d = L._domain(g, 0, 1, capacity=cells * 100 + 16)
    pp = np.full(cells, 100)
    d.set_particles(0, *L.cell_particles(g, rng, te, np.full(cells, 1e20), drift, pp, 1.0))
    d.set_particles(1, *L.cell_particles(g, rng, te / 2, np.full(cells, 1e20), np.zeros((cells, 3)), pp,
                                         L.MASS_ION))
    d.set_collision_model(*L.load_model())
    learned, fallback = d.collide_learned()
    assert learned == 0 and fallback == cells


def _host_moments(d, g, slots=(0, 1)):
    """Domain.cell_moments restated from the exported particles."""
    m = np.zeros((g.nr * g.nz, 16))
    for l, slot in enumerate(slots):
        p = d.get_particles(slot)
        c = p["cell_r"] * g.nz + p["cell_z"]
        ok = (p["cell_r"] >= 0) & (p["cell_r"] < g.nr) & (p["cell_z"] >= 0) & (p["cell_z"] < g.nz)
        w = p["w"]
        cols = [np.ones_like(w), w, w * p["vr"], w * p["vphi"], w * p["vz"],
                w * p["vr"] * p["vr"], w * p["vphi"] * p["vphi"], w * p["vz"] * p["vz"]]
        for q, v in enumerate(cols):
            np.add.at(m[:, 8 * l + q], c[ok], v[ok])
    return m


def test_float_layout_moments_by_tile():
    """Cell moments of tile-sorted float species (a block per tile, the
    tile's cells summed in shared memory), with particles that left their
    tile since the sort and slots appended after it, equal the sums over
    the exported particles."""
    from picopic_b200 import learned as L
    g = _grid(40, 96, dt=2e-14)  # 5 x 3 tiles, the last row of tiles partly outside the grid
    rng = np.random.default_rng(7)
    cells = g.nr * g.nz
    te = np.full((cells, 3), 2.0)
    drift = np.zeros((cells, 3))
    drift[:, 2] = 1e8  # 0.2 cells per step along z: particles cross tile borders
    pp = rng.integers(10, 30, cells)
    d = L._domain(g, 0, 5, capacity=cells * 80, precision="f32")
    d.set_particles(0, *L.cell_particles(g, rng, te, np.full(cells, 1e20), drift, pp, 1.0))
    d.set_particles(1, *L.cell_particles(g, rng, te / 4, np.full(cells, 1e20), np.zeros((cells, 3)), pp,
                                         L.MASS_ION))
    d.step(2)
    d.tile_sort(0)
    d.tile_sort(1)
    d.step(1)
    extra = L.cell_particles(g, rng, te, np.full(cells, 1e20), drift, np.full(cells, 2), 1.0)
    d.set_particles(0, *extra, append=True)
    m = d.cell_moments()
    h = _host_moments(d, g)
    scale = np.abs(h).max(0) + 1e-300
    assert (np.abs(m - h) <= 1e-12 * scale).all()


@pytest.mark.parametrize("scheme", [None, ("vay", "zigzag", "reference")])
def test_fused_learned_step_matches_collide_then_step(scheme):
    """A float step with learned collisions sums the cell moments in its push
    and applies the transforms in its move.  In the first step of a fresh
    domain the fields are zero and the push only rounds, so the step equals
    a learned collision pass (moments, network, transform in their own
    kernels) followed by a collisionless step, to float rounding.  With the
    Vay pusher and the ZigZag current (reference quirks) the move half and
    the collisionless step both run the pair kernel's fast paths."""
    from picopic_b200 import learned as L
    g = _grid()
    out = []
    for fused in (True, False):
        d = _random_domain(g, seed=6, precision="f32", scheme=scheme)
        d.set_collision_model(*L.load_model())
        if fused:
            d.set_collisions("learned")
        else:
            learned, _ = d.collide_learned()
            assert learned > 0.9 * g.nr * g.nz
        d.step(1)
        out.append([d.get_particles(s) for s in (0, 1)])
    for a, b in zip(*out):
        for k in ("r", "z", "vr", "vphi", "vz", "w"):
            scale = np.abs(b[k]).max()
            assert np.abs(a[k] - b[k]).max() <= 1e-5 * scale, k


def test_fallback_collides_every_fallback_cell():
    """Reference quirks: the binary pass stops a row at its first empty
    cell (collisionsP12.cpp:351-354).  The fallback pass of a learned step
    runs over the fallback cells only, and a cell left to the learned path
    is not an empty cell of that pass: every fallback cell collides, also
    behind learned cells in its row."""
    from picopic_b200 import Domain
    from picopic_b200 import learned as L
    g = _grid(16, 32)
    rng = np.random.default_rng(2)
    cells = g.nr * g.nz
    te = np.full((cells, 3), 1.0)
    drift = np.zeros((cells, 3))
    odd = np.arange(cells) % 2 == 1
    drift[odd, 2] = 4 * np.sqrt(1.6e-19 / ME)  # outside the training box
    d = Domain(g, precision="f64", quirks="reference", seed=1)
    d.add(L.ELECTRONS, capacity=cells * 100 + 16)
    d.add(L.IONS, capacity=cells * 100 + 16)
    pp = np.full(cells, 100)
    d.set_particles(0, *L.cell_particles(g, rng, te, np.full(cells, 1e20), drift, pp, 1.0))
    d.set_particles(1, *L.cell_particles(g, rng, te / 2, np.full(cells, 1e20), np.zeros((cells, 3)), pp,
                                         L.MASS_ION))
    d.set_collision_model(*L.load_model())
    m0 = d.cell_moments()
    learned, fallback = d.collide_learned()
    m1 = d.cell_moments()
    assert fallback == odd.sum() and learned == cells - odd.sum()
    changed = np.any(m1[:, 5:8] != m0[:, 5:8], axis=1)
    assert changed[odd].all()


@pytest.mark.parametrize("mode", ["binary", "learned"])
def test_pcg_step_with_collisions(mode):
    """pcg_step with collisions: the electron anisotropy of a bi-Maxwellian
    plasma falls over the steps, several times more than the collisionless
    run's drift."""
    from picopic_b200 import Domain
    from picopic_b200 import learned as L
    g = _grid(32, 64, dt=1e-14)  # 0.42 of the Courant limit

    def run(collisions):
        d = Domain(g, precision="f32", quirks="fixed", seed=3)
        d.add(L.ELECTRONS, capacity=g.nr * g.nz * 100)
        d.add(L.IONS, capacity=g.nr * g.nz * 100)
        d.seed_plasma_cells(0, 100, 1e22, 2.0, 1.0, seed=1)
        d.seed_plasma_cells(1, 100, 1e22, 0.5, seed=2)
        if collisions != "none":
            d.set_collision_model(*L.load_model())
            d.set_collisions(collisions)
        m = d.cell_moments().sum(0)
        a0 = m[7] / (0.5 * (m[5] + m[6])) - 1
        d.step(30)
        m = d.cell_moments().sum(0)
        return a0, m[7] / (0.5 * (m[5] + m[6])) - 1

    a0, a1 = run(mode)
    b0, b1 = run("none")
    assert a1 < a0 - 0.03
    assert a0 - a1 > 3 * abs(b1 - b0)  # well beyond the collisionless drift of the PIC noise


def test_wide_model_covers_few_particles_per_cell():
    from picopic_b200 import learned as L
    g = _grid(64, 128)
    model = L.load_model(L.WIDE_MODEL_PATH)
    tb, eb, _ = L.initial_relaxation_time(g, "binary", passes=120, density=3e20, ppc=12)
    tl, _, _ = L.initial_relaxation_time(g, "learned", passes=1, density=3e20, ppc=12, model=model)
    assert abs(tl / tb - 1) <= 0.01 + 3 * eb / tb
    # a weakly collisional plasma of 12 per cell (collision numbers ~1e-6 per step)
    cells = g.nr * g.nz
    rng = np.random.default_rng(3)
    d = L._domain(g, 0, 3, capacity=cells * 12 + 16)
    pp = np.full(cells, 12)
    te = np.full((cells, 3), 1.0)
    d.set_particles(0, *L.cell_particles(g, rng, te, np.full(cells, 1e18), np.zeros((cells, 3)), pp, 1.0))
    d.set_particles(1, *L.cell_particles(g, rng, te / 10, np.full(cells, 1e18), np.zeros((cells, 3)), pp,
                                         L.MASS_ION))
    d.set_collision_model(*model)
    learned, fallback = d.collide_learned()
    assert learned >= 0.9 * cells
