"""The reference's plasma initial condition restated on the host
(picopic_b200.initial) against the compiled reference's own
Domain::distribute (oracle/_ref): placement and weights bit for bit, the
velocity distribution statistically (the draws differ)."""
import json
import os

import numpy as np
import pytest

from oracle.harness import GridSpec, RefSim, SpeciesSpec, reference_available
from picopic_b200 import config, initial

HERE = os.path.dirname(os.path.abspath(__file__))
FUNCTIONAL = os.path.join(HERE, "golden", "functional", "PiCoPiC.json")


def test_radical_inverse():
    """random_reverse (rand.cpp:57-76): 1 -> 1/13, 13 -> 1/169, 14 -> 1/13 + 1/169."""
    r = initial.radical_inverse(np.array([0.0, 1.0, 13.0, 14.0, 2.7]), 13)
    assert r[0] == 0.0
    assert r[1] == 1 / 13 and r[2] == 13.0 ** -2 and r[3] == 1 / 13 + 13.0 ** -2
    assert r[4] == 2 / 13  # floor first
    i = np.arange(11 ** 3)
    np.testing.assert_allclose(np.sort(initial.radical_inverse(i, 11)), i / 11 ** 3, rtol=1e-13, atol=1e-16)


def test_juettner_energies():
    """The mean of gamma - 1 under Maxwell-Juettner is 3 theta + K1(1/theta)/K2(1/theta) - 1:
    2.37044 at theta = 1, 0.166989 at theta = 0.1."""
    rng = np.random.default_rng(4)
    assert abs(initial.juettner_gamma_minus_one(400000, 1.0, rng).mean() / 2.37044 - 1) < 5e-3
    assert abs(initial.juettner_gamma_minus_one(400000, 0.1, rng).mean() / 0.166989 - 1) < 5e-3
    e = initial.thermal_energies(400000, 0.05, rng)  # below 0.1: Maxwell-Boltzmann at T eV
    assert abs(e.mean() / 0.075 - 1) < 5e-3


def _reference_species(cfg, seed):
    g = cfg.geometry
    grid = GridSpec(g.nr, g.nz, g.radius, g.longitude, g.dt, pml_size=g.pml_size, pml_sigma=g.pml_sigma)
    r = RefSim(grid)
    r.seed(seed)
    for k, s in enumerate(cfg.species):
        r.add_plasma(SpeciesSpec(s["name"], s["charge"], s["mass"], id=k), s["macro_amount"],
                     s["density"], s["temperature"])
    r.distribute()
    return r


def test_restated_placement_and_weights_equal_the_reference():
    if not reference_available():
        pytest.skip("compiled reference not built (oracle/Makefile.ref)")
    cfg = config.load(FUNCTIONAL)
    g = cfg.geometry
    r = _reference_species(cfg, seed=3)
    for k, s in enumerate(cfg.species):
        p = r.get_particles(k)
        rr, zz, vr, vphi, vz, w = initial.reference_plasma(s["macro_amount"], g.nr, g.nz, g.dr, g.dz,
                                                           s["density"], s["temperature"], s["mass"], seed=k)
        assert rr.size == p["r"].size == s["macro_amount"]
        np.testing.assert_array_equal(rr, p["r"])
        np.testing.assert_array_equal(zz, p["z"])
        np.testing.assert_array_equal(w, p["w"])
        # the velocity distribution: kinetic energy mean and quantiles, and
        # the spread of each component, within the sampling error of 1e5 draws
        m = initial.EL_MASS * s["mass"]
        e_ref = m * (p["vr"] ** 2 + p["vphi"] ** 2 + p["vz"] ** 2) / initial.EL_CHARGE
        e_new = m * (vr ** 2 + vphi ** 2 + vz ** 2) / initial.EL_CHARGE
        assert abs(e_new.mean() / e_ref.mean() - 1) < 0.015, s["name"]
        q = [0.1, 0.5, 0.9]
        np.testing.assert_allclose(np.quantile(e_new, q), np.quantile(e_ref, q), rtol=0.02)
        for a, b in ((vr, p["vr"]), (vphi, p["vphi"]), (vz, p["vz"])):
            assert abs(a.std() / b.std() - 1) < 0.015
            assert abs(a.mean()) < 0.01 * a.std()


def test_functional_known_answers_fixture():
    """tests/golden/functional/step80.json holds the nine probes' known answers."""
    with open(os.path.join(HERE, "golden", "functional", "step80.json")) as f:
        doc = json.load(f)
    comps = doc["components"]
    assert sorted(comps) == sorted(f"{a}/{b}" for a in "EHJ" for b in ("r", "phi", "z"))
    for v in comps.values():
        assert abs(v["std"] ** 2 / v["var"] - 1) < 1e-6
