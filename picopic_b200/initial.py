"""The reference's own plasma initial condition, on the host.

`Domain::distribute` (domain.cpp:86-94) fills every plasma species with its
default switches (configure.ac:102-106: "flat" placement, "thermal"
velocities); this module builds the same particles for `Domain.set_particles`.

* Placement (`SpecieP::rectangular_random_placement`, specieP.cpp:127-189,
  SWITCH_PLASMA_SPATIAL_FLAT): macroparticle i sits at the radical inverses
  of i in base 13 (r) and of N-1-i in base 11 (z) (`random_reverse`,
  rand.cpp:57-76), over the domain shrunk by one cell at the outer walls and
  shifted by half a cell.  Deterministic: equal to the reference bit for bit.
* Weights (`SpecieP::set_weight`, specieP.cpp:280-331): each macroparticle's
  share of the real particles is proportional to its ring volume.  Sums run
  in particle order, as the reference's loops do, so the weights are equal
  bit for bit too.
* Velocities (`SpecieP::thermal_velocity_distribution`, specieP.cpp:346-384):
  an energy E per macroparticle, a speed sqrt(2 E e / m) / sqrt(2) (or the
  relativistic form above REL_LIMIT), and each component that speed times an
  independent uniform number in [-1, 1].  The energies follow the
  reference's sampler (`maxwellJuettner`, maxwellJuettner.cpp:330-400):
  below T = 0.1 the Maxwell-Boltzmann kinetic energy at T eV; from 0.1 up,
  gamma - 1 of a Maxwell-Juettner distribution whose temperature T is read
  in units of m c^2, the result then used as eV (so an electron plasma of
  "1 eV" has a mean energy of 2.37 eV and a kinetic temperature of 0.79
  eV).  The draws come from numpy's seeded generator: the distribution is
  the reference's, the individual numbers are not.
"""
from __future__ import annotations

import math

import numpy as np

# constant.hpp:35-57
PI = 3.1415926535897932
EL_MASS = 9.1e-31
EL_CHARGE = 1.6e-19
LIGHT_VEL = 3e8
MNZL = 1e-15
REL_LIMIT = 5e7


def radical_inverse(index, base: int) -> np.ndarray:
    """random_reverse (rand.cpp:57-76): the digits of floor(index) in `base`
    mirrored about the radix point, summed from the lowest digit up."""
    iv = np.floor(np.asarray(index, dtype=np.float64)).astype(np.int64)
    r = np.zeros(iv.shape)
    order = 1
    while (iv >= 1).any():
        ost = iv % base
        r = np.where(iv >= 1, r + ost * (float(base) ** (-order)), r)
        iv = (iv - ost) // base
        order += 1
    return r


def flat_positions(n: int, nr: int, nz: int, dr: float, dz: float):
    """(r, z) of n macroparticles of a one-domain grid with all four walls
    (cfg.cpp:398-429), as specieP.cpp:127-189 places them."""
    r_size = nr * dr - dr   # (ext - int) dr, less one cell at the r = R wall
    z_size = nz * dz - dz
    i = np.arange(n, dtype=np.float64)
    rand_r = radical_inverse(i, 13)
    rand_z = radical_inverse(n - 1 - i, 11)
    rand_r[rand_r == 0] = MNZL
    rand_z[rand_z == 0] = MNZL
    r = r_size * rand_r + dr / 2.
    z = z_size * rand_z + dz / 2.
    return r, z


def flat_weights(r: np.ndarray, nr: int, nz: int, dr: float, dz: float, density: float) -> np.ndarray:
    """SpecieP::set_weight (specieP.cpp:280-331) for a uniform density."""
    n = r.size
    if n == 0:
        return np.zeros(0)
    z_size = nz * dz - dz
    inner = r > dr / 2
    vol = np.where(inner, 2 * PI * r * dr * dz, PI * r * r * dz)
    v_sum = float(np.add.accumulate(vol)[-1])   # in particle order
    v_avg = v_sum / n
    top = float(nr - 1)
    n_total = (density + density) / 2 * PI * dr * dr * (top * top - 0.0 * 0.0) * z_size
    n_per_macro_avg = n_total / n
    norm = np.where(inner, 2 * PI * r * dr * dz / v_avg, PI * r * r * dz / v_avg)
    return n_per_macro_avg * norm


def juettner_gamma_minus_one(n: int, theta: float, rng: np.random.Generator) -> np.ndarray:
    """gamma - 1 drawn from the Maxwell-Juettner density
    f(gamma) ~ gamma sqrt(gamma^2 - 1) exp(-gamma / theta), by inverting its
    cumulative distribution tabulated on a grid dense near 0."""
    x_max = theta * 80.0 + 10.0 * theta * theta
    u = np.linspace(0.0, 1.0, 400001)
    x = x_max * u * u                       # x = gamma - 1
    f = (1.0 + x) * np.sqrt(x * (x + 2.0)) * np.exp(-x / theta)
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (f[1:] + f[:-1]) * np.diff(x))])
    cdf /= cdf[-1]
    return np.interp(rng.random(n), cdf, x)


def thermal_energies(n: int, temperature: float, rng: np.random.Generator) -> np.ndarray:
    """The energies maxwellJuettner(n, T) returns (maxwellJuettner.cpp:330-400),
    in the units the caller then reads as eV."""
    if temperature < 0.1:
        return rng.gamma(1.5, temperature, n)   # Maxwell-Boltzmann kinetic energy
    return juettner_gamma_minus_one(n, temperature, rng)


def thermal_velocities(n: int, temperature: float, mass_e: float, rng: np.random.Generator):
    """specieP.cpp:346-384 with the energies above; mass in electron masses."""
    mass = mass_e * EL_MASS
    two_over_mass = 2 * EL_CHARGE / mass
    mc_inv = EL_CHARGE / (mass * LIGHT_VEL)
    e = thermal_energies(n, temperature, rng)
    v = e * mc_inv
    rel = v > REL_LIMIT
    v = np.where(rel, v / np.sqrt(1.0 + v * v / (LIGHT_VEL * LIGHT_VEL)), np.sqrt(e * two_over_mass))
    v = v * 0.7071067811865475
    d = rng.uniform(-1.0, 1.0, size=(3, n))
    return d[0] * v, d[1] * v, d[2] * v


def reference_plasma(n: int, nr: int, nz: int, dr: float, dz: float, density: float,
                     temperature: float, mass_e: float, seed: int = 0):
    """One plasma species as Domain::distribute makes it: (r, z, vr, vphi,
    vz, w) for `Domain.set_particles`."""
    r, z = flat_positions(n, nr, nz, dr, dz)
    w = flat_weights(r, nr, nz, dr, dz, density)
    vr, vphi, vz = thermal_velocities(n, temperature, mass_e, np.random.default_rng(seed))
    return r, z, vr, vphi, vz, w


def _self_check():
    # the mean of gamma - 1 under Maxwell-Juettner is 3 theta + K1/K2 - 1; at
    # theta = 1 that is 2.3704
    g = juettner_gamma_minus_one(200000, 1.0, np.random.default_rng(1))
    assert abs(g.mean() - 2.3704) < 0.02, g.mean()
    assert math.isclose(radical_inverse(np.array([1.0]), 13)[0], 1 / 13)


if __name__ == "__main__":
    _self_check()
    print("ok")
