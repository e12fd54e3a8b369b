"""Seeded synthetic inputs shared by the parity tests.

Particles are placed inside the reflecting walls (r in [dr/2, R-dr/2],
z in [dz/2, L-dz/2]) with Maxwellian velocities scaled up by ``boost`` so
that a few steps exercise cell crossings, reflections and the 4/7/10-node
branches of the current deposition.  Fields are random so every gather
and Yee branch sees non-zero data.
"""
import numpy as np

from oracle.harness import FIELDS, GridSpec, SpeciesSpec

ELECTRONS = SpeciesSpec("electrons", -1, 1, id=1)
IONS = SpeciesSpec("ions", 1, 1836, id=2)


def small_grid(nr=24, nz=48, pml=True, dt=1.0e-13):
    dr = 1e-4
    return GridSpec(nr, nz, nr * dr, nz * dr, dt,
                    pml_size=(0, 0, nr // 5, nz // 6) if pml else (0, 0, 0, 0),
                    pml_sigma=(1e-5, 0.07) if pml else (0.0, 0.0))


def beam_spec(grid, macro_amount=20000):
    return SpeciesSpec("beam_electrons", -1, 1, id=1000,
                       beam=dict(macro_amount=macro_amount, start_time=0.0,
                                 radius=grid.radius * 0.3, density=1e16, amount=2,
                                 length=grid.longitude * 0.2, distance=grid.longitude * 0.3,
                                 velocity=2.8e8))


def particles(grid, n, seed, mass=1.0, boost=30.0):
    rng = np.random.default_rng(seed)
    r = grid.dr / 2 + rng.random(n) * (grid.radius - grid.dr)
    z = grid.dz / 2 + rng.random(n) * (grid.longitude - grid.dz)
    sigma = np.sqrt(1.6e-19 * 1.0 / (9.1e-31 * mass)) * boost
    v = rng.normal(size=(3, n)) * sigma
    w = rng.random(n) * 1e6 + 1e5
    return (r, z, v[0], v[1], v[2], w)


def near_axial(grid, n, seed, dt=None):
    """Particles that cross a z cell face in one step while moving radially
    by only 1.2e-15 to 5e-15 m, so that the part of the step behind the face
    moves less than the reference's 1e-15 m segment threshold radially."""
    rng = np.random.default_rng(seed)
    dt = grid.dt if dt is None else dt
    vz = 2.0e8
    step = vz * dt / grid.dz
    r = (1.5 + rng.random(n) * (grid.nr / 2)) * grid.dr
    k = rng.integers(2, grid.nz - 4, size=n)
    z = (k + 1.0 - step * (0.05 + 0.9 * rng.random(n))) * grid.dz
    dr = (1.2e-15 + rng.random(n) * 3.8e-15) * rng.choice([-1.0, 1.0], size=n)
    w = rng.random(n) * 1e6 + 1e5
    return (r, z, dr / dt, np.zeros(n), np.full(n, vz), w)


def quiet_plasma(grid, density, per_cell=4, v0=0.0):
    """Cold, exactly neutral plasma for the Langmuir test: a regular lattice of
    per_cell x per_cell points per cell over the region between the
    reflecting walls (r in [dr/2, R - dr/2], z in [dz/2, L - dz/2]), each
    point's weight its ring volume times `density`.  Electrons and ions share
    the lattice; the electrons get v_z = v0 sin(2 pi z / L).  Returns the
    electron and ion arrays (r, z, vr, vphi, vz, w)."""
    nr_p, nz_p = per_cell * (grid.nr - 1), per_cell * (grid.nz - 1)
    hr, hz = (grid.radius - grid.dr) / nr_p, (grid.longitude - grid.dz) / nz_p
    r1 = grid.dr / 2 + (np.arange(nr_p) + 0.5) * hr
    z1 = grid.dz / 2 + (np.arange(nz_p) + 0.5) * hz
    r, z = (a.ravel() for a in np.meshgrid(r1, z1, indexing="ij"))
    w = density * 2 * np.pi * r * hr * hz
    zero = np.zeros_like(r)
    vz = v0 * np.sin(2 * np.pi * z / grid.longitude)
    return (r, z, zero, zero, vz, w), (r.copy(), z.copy(), zero, zero, zero, w.copy())


def dominant_frequency(x, dt, lo, hi):
    """Angular frequency in [lo, hi] at which |sum (x - mean) e^{-i w t}| peaks
    (a fine scan refined by a parabola through the peak)."""
    x = np.asarray(x, dtype=float) - np.mean(x)
    t = np.arange(len(x)) * dt
    w = np.linspace(lo, hi, 4001)
    p = np.abs(np.exp(-1j * np.outer(w, t)) @ x)
    m = int(np.clip(np.argmax(p), 1, len(w) - 2))
    a, b, c = p[m - 1], p[m], p[m + 1]
    return w[m] + 0.5 * (a - c) / (a - 2 * b + c) * (w[1] - w[0])


def plasma_frequency(density, mass=1.0):
    """sqrt(n e^2 / (eps0 m)) with the reference's constants (constant.hpp)."""
    return np.sqrt(density * 1.6e-19 ** 2 / (8.85e-12 * 9.1e-31 * mass))


def map_particles(grid, n, seed, mass=1.0):
    """Particles for the diagnostic maps: a quarter inside r <= dr/2, a
    quarter in dr/2 < r <= dr (the three radial branches of the
    reference's weighting), thermal speeds with a tenth above 5e7 m/s."""
    rng = np.random.default_rng(seed)
    r = grid.dr / 2 + rng.random(n) * (grid.radius - grid.dr)
    q = n // 4
    r[:q] = rng.random(q) * grid.dr / 2
    r[q:2 * q] = grid.dr / 2 + rng.random(q) * grid.dr / 2
    z = grid.dz / 2 + rng.random(n) * (grid.longitude - grid.dz)
    v = rng.normal(size=(3, n)) * np.sqrt(1.6e-19 * 2.0 / (9.1e-31 * mass))
    fast = rng.random(n) < 0.1
    v[2, fast] = np.sign(rng.random(fast.sum()) - 0.5) * (6e7 + rng.random(fast.sum()) * 1e8)
    w = rng.random(n) * 1e6 + 1e5
    return (r, z, v[0], v[1], v[2], w)


def random_fields(grid, seed, scale=1e3):
    rng = np.random.default_rng(seed + 7919)
    return {f: rng.normal(size=grid.shape) * scale for f in FIELDS}


def load(sim, grid, species, n, seed, fields=True):
    for sp in species:
        sim.add(sp)
    for i, sp in enumerate(species):
        if sp.beam is None:
            sim.set_particles(i, *particles(grid, n, seed + i, mass=sp.mass,
                                            boost=30.0 if sp.mass == 1 else 150.0))
    if fields:
        for name, a in random_fields(grid, seed).items():
            sim.set_field(name, a)


def thermal_plasma(grid, n, seed, mass=1.0, temperature_ev=1.0, density=1e20, t_par_ratio=1.0):
    """Uniform plasma of n macroparticles of equal weight (density in m^-3),
    Maxwellian at temperature_ev, the z temperature scaled by t_par_ratio:
    the collisional cases."""
    rng = np.random.default_rng(seed)
    r = grid.dr / 2 + rng.random(n) * (grid.radius - grid.dr)
    z = grid.dz / 2 + rng.random(n) * (grid.longitude - grid.dz)
    s = np.sqrt(temperature_ev * 1.6e-19 / (mass * 9.1e-31))
    v = rng.normal(size=(3, n)) * s
    v[2] *= np.sqrt(t_par_ratio)
    w = np.full(n, density * np.pi * grid.radius ** 2 * grid.longitude / n)
    return (r, z, v[0], v[1], v[2], w)
