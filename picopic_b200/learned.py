"""The learned collision operator: training data from the binary operator,
training of the collision MLP on the GPU, and relaxation measurements.

The binary operator (``Domain.collide``, Perez 2012) is run for one step on
cells of randomly drawn plasma states; the cell moments before and after
give the training pairs:

  x  the 13 features of ``Domain.cell_features`` (anisotropies, temperature
     ratio, collision numbers s_ee, s_ei, s_ii of the step, drift, density
     ratio, macroparticle noise);
  y  the change of the six axis temperatures over the step in units of
     T_s S (S = s_ee + s_ei + s_ii), the quantity the learned step
     (``Domain.collide_learned``) applies.

``fit`` trains the network with the library's own tensor-core kernels
(``picopic_b200.mlp.Mlp``).  The binary operator stays the judge: the
relaxation time of an anisotropic plasma under both operators is what
``relaxation_time`` measures.

Command lines (one GPU) of the two committed models:
    python -m picopic_b200.learned train --out picopic_b200/models/collision_p12.npz
    python -m picopic_b200.learned train --wide --batches 96 --steps 1000000 \
        --out picopic_b200/models/collision_p12_wide.npz
"""
from __future__ import annotations

import argparse
import dataclasses
import os
import time

import numpy as np

from .mlp import PARAMS, Mlp

ME, E_CHARGE = 9.1e-31, 1.6e-19
MASS_ION = 1836.0
FEATURES, TARGETS = 13, 6
MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "models", "collision_p12.npz")
# trained on Sampling.wide() with inverse-noise weighting: for few macroparticles
# per cell or weakly collisional plasmas, where the default model's box ends
WIDE_MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "models", "collision_p12_wide.npz")


@dataclasses.dataclass
class Sampling:
    """Ranges of the random cell states of the training data."""
    te: tuple = (0.5, 4.0)            # electron temperature, eV (log-uniform)
    ti: tuple = (0.1, 2.0)            # ion temperature, eV (log-uniform)
    density: tuple = (1e19, 1e21)     # m^-3 (log-uniform), equal for both species
    e_aniso: float = 0.6              # electron axis temperatures T (1 + U(-a, a)), renormalised
    i_aniso: float = 0.3
    drift: float = 0.1                # electron drift per axis, in thermal speeds
    ppc: tuple = (60, 140)            # macroparticles per cell per species (log-uniform)
    ion_density: float = 0.2          # ion density n_e exp(U(-a, a))

    @classmethod
    def wide(cls):
        """The states of the wide model: down to 2 macroparticles per cell
        and 1e16 m^-3 (collision numbers down to ~1e-7 per step), with the
        drift, anisotropy and density-ratio spread that few particles per
        cell show."""
        return cls(ti=(0.05, 2.0), density=(1e16, 1e21), e_aniso=0.8, i_aniso=0.6, drift=0.6,
                   ppc=(2, 200), ion_density=1.0)


class _Spec:
    def __init__(self, name, charge, mass, id):
        self.name, self.charge, self.mass, self.id, self.beam = name, charge, mass, id, None


ELECTRONS = _Spec("electrons", -1, 1, 1)
IONS = _Spec("ions", 1, MASS_ION, 2)


def cell_states(grid, rng, s: Sampling):
    """Per-cell random plasma parameters: T_e (cells, 3), T_i (cells, 3),
    electron and ion densities, electron drift (cells, 3) in m/s, electron
    and ion particles per cell."""
    cells = grid.nr * grid.nz

    def logu(lo, hi, n):
        return np.exp(rng.uniform(np.log(lo), np.log(hi), n))

    def axes(a):
        f = 1.0 + rng.uniform(-a, a, (cells, 3))
        return f / f.mean(1, keepdims=True)

    te = logu(*s.te, cells)[:, None] * axes(s.e_aniso)
    ti = logu(*s.ti, cells)[:, None] * axes(s.i_aniso)
    dens = logu(*s.density, cells)
    vth = np.sqrt(E_CHARGE * te.mean(1) / ME)
    drift = rng.uniform(-s.drift, s.drift, (cells, 3)) * vth[:, None]
    ppc = np.rint(np.exp(rng.uniform(np.log(s.ppc[0]), np.log(s.ppc[1]), (2, cells)))).astype(np.int64)
    dens_i = dens * np.exp(rng.uniform(-s.ion_density, s.ion_density, cells))
    return te, ti, (dens, dens_i), drift, ppc


def cell_particles(grid, rng, temps, dens, drift, ppc, mass):
    """Macroparticles of one species: ppc[c] per cell c, uniform in the cell
    volume, Maxwellian with the cell's axis temperatures, equal weights
    n V_cell / ppc."""
    cells = grid.nr * grid.nz
    c = np.repeat(np.arange(cells), ppc)
    i, k = c // grid.nz, c % grid.nz
    u0, u1 = rng.random(c.size), rng.random(c.size)
    r = grid.dr * np.sqrt(i * i + u0 * (2 * i + 1))       # uniform in r^2 within the cell
    z = grid.dz * (k + u1)
    sig = np.sqrt(E_CHARGE * temps[c] / (mass * ME))
    v = rng.normal(size=(c.size, 3)) * sig + drift[c]
    vol = np.pi * grid.dz * grid.dr ** 2 * (2 * i + 1)
    w = dens[c] * vol / ppc[c]
    return r, z, v[:, 0], v[:, 1], v[:, 2], w


def temperatures(m):
    """Axis temperatures (cells, 2, 3) in eV and weights (cells, 2) of the
    electron and ion lists from Domain.cell_moments."""
    out, W = np.zeros((m.shape[0], 2, 3)), np.zeros((m.shape[0], 2))
    for l, mass in ((0, ME), (1, MASS_ION * ME)):
        ml = m[:, 8 * l:8 * l + 8]
        with np.errstate(invalid="ignore", divide="ignore"):
            u = ml[:, 2:5] / ml[:, 1:2]
            out[:, l] = mass * (ml[:, 5:8] / ml[:, 1:2] - u * u) / E_CHARGE
        W[:, l] = ml[:, 1]
    return out, W


def _domain(grid, device, seed, capacity, precision="f64"):
    from .domain import Domain
    d = Domain(grid, precision=precision, quirks="fixed", seed=seed, device=device)
    d.add(ELECTRONS, capacity=capacity)
    d.add(IONS, capacity=capacity)
    return d


def generate(grid, batches, seed=1, sampling: Sampling = Sampling(), device=0, log=print, expectation=True,
             pairings=8):
    """Training pairs (x, y) from one binary-operator step on `batches`
    grids of random cell states.  With expectation (the default) the
    targets are the operator's mean change (Domain.collide_expectation:
    each collision's mean over its scattering draw, given the velocities it
    meets), averaged over `pairings` passes from the same start, else one
    random draw: the mean removes the Monte Carlo noise that dwarfs the
    per-step change."""
    xs, ys = [], []
    for b in range(batches):
        t0 = time.time()
        rng = np.random.default_rng(seed + 7919 * b)
        te, ti, dens, drift, ppc = cell_states(grid, rng, sampling)
        pe = cell_particles(grid, rng, te, dens[0], drift, ppc[0], 1.0)
        pi = cell_particles(grid, rng, ti, dens[1], np.zeros_like(drift), ppc[1], MASS_ION)
        d = _domain(grid, device, seed + b, capacity=max(pe[0].size, pi[0].size) + 16)
        d.set_particles(0, *pe)
        d.set_particles(1, *pi)
        x, S = d.cell_features()
        m0 = d.cell_moments()
        T0, _ = temperatures(m0)
        if expectation:  # the operator's mean change, over `pairings` passes from the same start
            dm = np.zeros((m0.shape[0], 12))
            for q in range(pairings):
                if q:
                    d.set_particles(0, *pe)
                    d.set_particles(1, *pi)
                dm += d.collide_expectation()
            dm /= pairings
            m1 = m0.copy()
            for l in (0, 1):
                m1[:, 8 * l + 2:8 * l + 8] += dm[:, 6 * l:6 * l + 6]
        else:  # one random draw
            d.collide()
            m1 = d.cell_moments()
        T1, _ = temperatures(m1)
        Tm = T0.mean(2)
        with np.errstate(invalid="ignore", divide="ignore"):
            y = ((T1 - T0) / (Tm[:, :, None] * S[:, None, None])).reshape(-1, TARGETS)
        ok = np.isfinite(x).all(1) & np.isfinite(y).all(1) & (S > 0)
        xs.append(x[ok])
        ys.append(y[ok].astype(np.float32))
        del d
        log(f"batch {b}: {ok.sum()} pairs, {time.time() - t0:.1f} s")
    return np.concatenate(xs), np.concatenate(ys)


def normalisation(x, y):
    """The 64-float block of pcg_set_collision_model: feature mean, std,
    target mean, std, and the training box (0.05 and 99.95 percentiles)."""
    xm, xsd = x.mean(0), np.maximum(x.std(0), 1e-6)
    ym, ysd = y.mean(0), np.maximum(y.std(0), 1e-12)
    lo, hi = np.percentile(x, 0.05, axis=0), np.percentile(x, 99.95, axis=0)
    return np.concatenate([xm, xsd, ym, ysd, lo, hi]).astype(np.float32)


def inverse_noise_resample(x, y, seed=0):
    """Pairs resampled with probability proportional to the macroparticle
    count N of their cell (feature 12 is 1/sqrt(N)): the variance of a
    target given its features falls as 1/N, so this is the inverse-variance
    weighting of the squared loss, which keeps the many noisy low-count
    cells from swamping the fit where the targets are sharp."""
    wgt = 1.0 / np.square(x[:, 12].astype(np.float64))
    idx = np.random.default_rng(seed).choice(len(x), size=len(x), p=wgt / wgt.sum())
    return x[idx], y[idx]


def fit(x, y, steps=20000, batch=8192, lr=2e-3, seed=3, device=0, log=print):
    """Train the collision MLP on (x, y) with the library's kernels; returns
    (params, norm, final loss)."""
    norm = normalisation(x, y)
    xn = (x - norm[:13]) / norm[13:26]
    yn = (y - norm[26:32]) / norm[32:38]
    m = Mlp(device=device, seed=seed)
    m.set_data(xn, yn)
    loss = None
    for stage, frac in enumerate((0.5, 0.3, 0.2)):
        loss = m.train(int(steps * frac), batch=batch, lr=lr * (0.3 ** stage))
        log(f"stage {stage}: minibatch loss {loss:.4f}")
    params = m.params
    m.close()
    return params, norm, loss


def save_model(path, params, norm, meta: dict):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, params=np.asarray(params, np.float32), norm=np.asarray(norm, np.float32),
             meta=np.array(repr(meta)))


def load_model(path=MODEL_PATH):
    d = np.load(path)
    if d["params"].size != PARAMS or d["norm"].size != 64:
        raise ValueError(f"{path}: {d['params'].size} parameters and {d['norm'].size} normalisation "
                         f"values, the network has {PARAMS} and 64")
    return d["params"], d["norm"]


def anisotropy_run(grid, operator, passes, seed=5, device=0, ppc=100, te=(2.0, 1.0), ti=0.5,
                   density=1e20, model=None, precision="f64", every=1):
    """Electron T_par / T_perp - 1 after each `every` collision steps of a
    uniform plasma (electrons at T_par = te[0], T_perp = te[1], ions at ti)
    under the binary or the learned operator.  Returns (steps, anisotropy,
    seconds spent in the operator)."""
    rng = np.random.default_rng(seed)
    cells = grid.nr * grid.nz
    te_axes = np.tile([te[1], te[1], te[0]], (cells, 1)).astype(float)
    ti_axes = np.full((cells, 3), float(ti))
    dens = np.full(cells, float(density))
    ppcs = np.full(cells, ppc)
    d = _domain(grid, device, seed, capacity=cells * ppc + 16, precision=precision)
    d.set_particles(0, *cell_particles(grid, rng, te_axes, dens, np.zeros((cells, 3)), ppcs, 1.0))
    d.set_particles(1, *cell_particles(grid, rng, ti_axes, dens, np.zeros((cells, 3)), ppcs, MASS_ION))
    if operator == "learned":
        d.set_collision_model(*(model if model is not None else load_model()))

    def aniso():
        m = d.cell_moments().sum(0)
        W, u = m[1], m[2:5] / m[1]
        T = ME * (m[5:8] / W - u * u) / E_CHARGE
        return T[2] / (0.5 * (T[0] + T[1])) - 1.0

    steps, values, spent = [0], [aniso()], 0.0
    for s in range(1, passes + 1):
        d.synchronize()
        t0 = time.perf_counter()
        if operator == "learned":
            d.collide_learned()
        else:
            d.collide()
        spent += time.perf_counter() - t0
        if s % every == 0:
            steps.append(s)
            values.append(aniso())
    return np.array(steps), np.array(values), spent


def initial_relaxation_time(grid, operator, passes=1, seed=5, device=0, ppc=100, te=(2.0, 1.0), ti=0.5,
                            density=1e20, model=None, precision="f64"):
    """Temperature-relaxation time of the electron anisotropy
    A = T_par / T_perp - 1 at a bi-Maxwellian start: tau = A / (-dA/dstep),
    dA the change of one collision step, averaged over `passes` independent
    passes from the same start (the binary operator's Monte Carlo spread),
    after one untimed pass.  Returns (tau in steps, its standard error,
    seconds per pass)."""
    rng = np.random.default_rng(seed)
    cells = grid.nr * grid.nz
    te_axes = np.tile([te[1], te[1], te[0]], (cells, 1)).astype(float)
    ti_axes = np.full((cells, 3), float(ti))
    dens = np.full(cells, float(density))
    ppcs = np.full(cells, ppc)
    pe = cell_particles(grid, rng, te_axes, dens, np.zeros((cells, 3)), ppcs, 1.0)
    pi = cell_particles(grid, rng, ti_axes, dens, np.zeros((cells, 3)), ppcs, MASS_ION)
    d = _domain(grid, device, seed, capacity=cells * ppc + 16, precision=precision)
    if operator == "learned":
        d.set_collision_model(*(model if model is not None else load_model()))

    def aniso():
        m = d.cell_moments().sum(0)
        u = m[2:5] / m[1]
        T = ME * (m[5:8] / m[1] - u * u) / E_CHARGE
        return T[2] / (0.5 * (T[0] + T[1])) - 1.0

    if operator == "learned":  # one untimed pass: first-call set-up (scratch, kernel attributes)
        d.set_particles(0, *pe)
        d.set_particles(1, *pi)
        d.collide_learned()
    else:
        d.set_particles(0, *pe)
        d.set_particles(1, *pi)
        d.collide()
    d.set_particles(0, *pe)
    d.set_particles(1, *pi)
    a0 = aniso()
    rates, spent = [], 0.0
    for q in range(passes):
        if q:
            d.set_particles(0, *pe)
            d.set_particles(1, *pi)
        d.synchronize()  # the import's kernels stay out of the timed pass
        t0 = time.perf_counter()
        if operator == "learned":
            d.collide_learned()
        else:
            d.collide()
        spent += time.perf_counter() - t0
        rates.append(a0 - aniso())
    r = np.array(rates)
    tau = a0 / r.mean()
    err = tau * (r.std() / np.sqrt(len(r)) / r.mean()) if len(r) > 1 else 0.0
    return tau, err, spent / passes


def relaxation_time(steps, values, lo=0.95):
    """Temperature-relaxation time: the e-folding time (steps) of the
    anisotropy from a least-squares fit of its logarithm over the part of
    the curve above lo times its start.  The default keeps the first 5 % of
    the decay, where the velocity distribution is still bi-Maxwellian: later
    the binary operator relaxes the slow core before the fast tails, which a
    transform of second moments does not follow (over a decay to 70 % the
    binary curve's fitted time is ~10 % longer)."""
    keep = values > lo * values[0]
    p = np.polyfit(steps[keep], np.log(values[keep]), 1)
    return -1.0 / p[0]


RELAX_STATES = (  # density m^-3, electron (T_par, T_perp) eV, ion T eV, macroparticles per cell
    (5e19, (2.0, 1.0), 0.5, 100), (1e20, (2.0, 1.0), 0.5, 100), (3e20, (2.0, 1.0), 0.5, 100),
    (1e21, (3.0, 1.5), 1.0, 100), (3e20, (1.0, 0.5), 0.25, 100), (3e20, (2.0, 1.0), 0.5, 12))


def relax_table(paths, passes=200, device=0, log=print):
    """Initial electron-anisotropy relaxation time of each model against the
    binary operator (mean of `passes` passes, with its standard error) on a
    64 x 128 slab of cells of 1e-5 m, dt 1e-13 s, for RELAX_STATES."""
    from .domain import Geometry
    g = Geometry(64, 128, 64e-5, 128e-5, 1e-13)
    models = [load_model(p) for p in paths]
    rows = []
    for n, te, ti, ppc in RELAX_STATES:
        tb, eb, _ = initial_relaxation_time(g, "binary", passes=passes, density=n, te=te, ti=ti, ppc=ppc,
                                            device=device)
        ratios = [initial_relaxation_time(g, "learned", passes=1, density=n, te=te, ti=ti, ppc=ppc,
                                          model=m, device=device)[0] / tb for m in models]
        rows.append((n, te, ti, ppc, tb, eb, ratios))
        log(f"n {n:.0e} Te {te} Ti {ti} ppc {ppc}: binary {tb:.1f} +- {eb:.1f} steps; " +
            ", ".join(f"{os.path.basename(p)} {x:.4f}" for p, x in zip(paths, ratios)))
    return rows


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", default=MODEL_PATH)
    t.add_argument("--nr", type=int, default=128)
    t.add_argument("--nz", type=int, default=512)
    t.add_argument("--batches", type=int, default=24)
    t.add_argument("--dt", type=float, default=1e-13)
    t.add_argument("--steps", type=int, default=200000)
    t.add_argument("--seed", type=int, default=1)
    t.add_argument("--wide", action="store_true",
                   help="the wide model: Sampling.wide() states, inverse-noise weighting")
    r = sub.add_parser("relax", help="relaxation-time ratio learned / binary on six plasma states")
    r.add_argument("--model", action="append", default=None, help="model file (repeatable)")
    r.add_argument("--passes", type=int, default=200)
    a = ap.parse_args(argv)
    from .domain import Geometry
    if a.cmd == "relax":
        relax_table(a.model or [MODEL_PATH, WIDE_MODEL_PATH], a.passes)
        return
    dr = 1e-5
    grid = Geometry(a.nr, a.nz, a.nr * dr, a.nz * dr, a.dt)
    t0 = time.time()
    sampling = Sampling.wide() if a.wide else Sampling()
    x, y = generate(grid, a.batches, seed=a.seed, sampling=sampling)
    t1 = time.time()
    xf, yf = inverse_noise_resample(x, y, seed=a.seed + 5) if a.wide else (x, y)
    params, norm, loss = fit(xf, yf, steps=a.steps, seed=a.seed + 2)
    meta = {"pairs": int(x.shape[0]), "grid": [a.nr, a.nz], "dr": dr, "dt": a.dt,
            "sampling": dataclasses.asdict(sampling), "weighting": "inverse noise" if a.wide else "uniform",
            "final_minibatch_loss": loss, "generate_s": round(t1 - t0, 1), "train_s": round(time.time() - t1, 1)}
    save_model(a.out, params, norm, meta)
    print("saved", a.out, meta)


if __name__ == "__main__":
    main()
