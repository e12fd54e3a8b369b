"""The reference's functional test (test/functional/test.py) on the GPU.

The configuration tests/golden/functional/PiCoPiC.json runs through the
drop-in path a user takes (picopic_b200.config: build_domain with the
reference's own plasma initial condition, then run with the reference's
probe schedule), and frame 4 of each of the nine probes is held to the
reference's known answers (tests/golden/functional/step80.json): every run
within 0.2 of each standard deviation, the mean over three seeds within the
reference's own rtol 0.15 (tests/test_functional_golden.py says why).  The
double-precision run also equals the oracle, started from the same particles
with the same Philox beam draws, to 1e-9 of each field's largest value after
the 81 steps.
"""
import numpy as np
import pytest

from oracle.harness import FIELDS, OracleSim
from picopic_b200 import config, initial
from tests.test_functional_golden import (FUNCTIONAL, RTOL_ONE_RUN, STEPS, check, functional_grid,
                                          known_answers, specs)

pytestmark = pytest.mark.gpu

SEEDS = (7, 8, 9)
PROBE = "rec/0-32_0-128"


def run(precision, seed):
    cfg = config.load(FUNCTIONAL)
    d, slots = config.build_domain(cfg, precision=precision, quirks="reference", seed=seed, plasma="reference")
    frames = config.run(cfg, d, slots, steps=STEPS, log=lambda *a: None)
    std = {}
    for comp in known_answers():
        f = frames[f"{comp}/{PROBE}"]
        assert f.shape == (5, 32, 128), f.shape   # iterations 0, 20, 40, 60, 80
        assert np.isfinite(f).all()
        std[comp] = float(f[4].std())
    return cfg, d, slots, std


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_functional_known_answers(precision):
    runs = []
    for seed in SEEDS:
        _, d, slots, std = run(precision, seed)
        assert d.count(slots["beam_electrons"]) > 400  # the bunch entered
        d.close()
        check(std, RTOL_ONE_RUN, f"{precision} seed {seed}")
        runs.append(std)
    mean = {c: float(np.mean([r[c] for r in runs])) for c in runs[0]}
    check(mean, 0.15, f"{precision} mean of {len(SEEDS)} seeds")


def test_functional_run_equals_the_oracle():
    seed = SEEDS[0]
    cfg, d, slots, _ = run("f64", seed)
    g = cfg.geometry
    plasma, beams = specs(cfg)
    orc = OracleSim(functional_grid(cfg), quirks="reference")
    for sp in plasma + beams:
        orc.add(sp)
    for k, s in enumerate(cfg.species):
        # the particles build_domain(plasma="reference", seed=seed) imported
        orc.set_particles(k, *initial.reference_plasma(s["macro_amount"], g.nr, g.nz, g.dr, g.dz, s["density"],
                                                       s["temperature"], s["mass"], seed=seed * 1000 + k))
    orc.set_rng("philox", seed)
    assert orc.step(STEPS) == 0
    for k, name in enumerate(list(slots)):
        assert d.count(slots[name]) == orc.count(k), name
    for name in FIELDS:
        a, b = d.get_field(name), orc.get_field(name)
        scale = max(np.abs(b).max(), 1e-300)
        assert np.abs(a - b).max() <= 1e-9 * scale, f"{name}: {np.abs(a - b).max() / scale:.3e}"
    d.close()
