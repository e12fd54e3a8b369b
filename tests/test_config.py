"""PiCoPiC.json read into a run (picopic_b200.config): the geometry, PML
cells, macroparticle amounts (Cfg::weight_macro_amount, cfg.cpp:489-571)
and probe paths (Cfg::init_probes, cfg.cpp:204-290) of
tests/golden/configs/small.json, its refusals, and on a GPU a run that
writes every probe on its schedule."""
import copy
import json
import os

import numpy as np
import pytest

from picopic_b200 import config

CFG = os.path.join(os.path.dirname(__file__), "golden", "configs", "small.json")


def test_load_small_configuration():
    c = config.load(CFG)
    g = c.geometry
    assert (g.nr, g.nz) == (32, 128) and abs(g.dr - 1e-4) < 1e-18 and abs(g.dz - 1e-4) < 1e-18
    assert g.pml_size == (0, 0, 4, 8)  # floor(wall fraction x cells): left, outer, right
    assert c.steps == 30
    # norm = 2e5 / (32 * 128 * 2 + (0.001/1e-4) * (0.002 * 2/1e-4) * 2) = 2e5 / 8992
    assert [s["macro_amount"] for s in c.species] == [91103, 91103]
    assert c.beams[0]["name"] == "beam_electrons" and c.beams[0]["macro_amount"] == 17793
    assert [p.path for p in c.probes] == ["E/r/rec/0-32_0-128", "density/electrons/rec/0-16_0-64",
                                         "temperature/ions/row/4", "H/phi/dot/4_64", "J/z/col/64"]


def test_refusals():
    with open(CFG) as f:
        raw = json.load(f)
    bad = copy.deepcopy(raw)
    bad["data"]["probes"][0]["end"]["r"] = 40  # beyond the grid
    with pytest.raises(ValueError):
        config.load(bad)
    bad = copy.deepcopy(raw)
    bad["data"]["probes"][0]["shape"] = "ring"
    with pytest.raises(ValueError):
        config.load(bad)
    bad = copy.deepcopy(raw)
    bad["particles"].append(dict(bad["particles"][0]))
    with pytest.raises(ValueError):
        config.load(bad)


def test_unknown_plasma_initialiser_is_refused():
    with pytest.raises(ValueError):
        config.build_domain(config.load(CFG), plasma="uniform")


class _CountingDomain:
    """Stands in for a Domain: every grid holds the number of steps taken."""
    def __init__(self, shape):
        self.shape, self.steps = shape, 0

    def step(self, n):
        self.steps += n

    def get_field(self, which):
        return np.full(self.shape, float(self.steps))

    def species_map(self, slot, which):
        return np.full((3,) + self.shape if which == "momentum" else self.shape, float(self.steps))

    def synchronize(self):
        pass


def test_probe_schedule_is_the_references():
    """Frame j of a probe of schedule s is the state after s j + 1 steps: the
    reference's writers run after the step of iteration k, while the clock
    still reads k dt (PiCoPiC.cpp:326-347, outController.cpp:341-351)."""
    c = config.load(CFG)
    g = c.geometry
    d = _CountingDomain((g.nr + 4, g.nz + 4))
    slots = {"electrons": 0, "ions": 1}
    out = config.run(c, d, slots, steps=31, log=lambda *a: None)
    assert d.steps == 31
    frames = {p.path: p.schedule for p in c.probes}
    for path, a in out.items():
        s = frames[path]
        want = [s * j + 1 for j in range((31 - 1) // s + 1)]
        got = [float(np.asarray(f).flat[0]) for f in a]
        assert got == want, (path, got, want)


@pytest.mark.gpu
def test_run_writes_probes(tmp_path):
    c = config.load(CFG)
    d, slots = config.build_domain(c, precision="f32", seed=3)
    assert d.count(slots["electrons"]) == 91103
    out = config.run(c, d, slots, steps=30, out_dir=str(tmp_path), log=lambda *a: None)
    shapes = {"E/r/rec/0-32_0-128": (3, 32, 128), "density/electrons/rec/0-16_0-64": (3, 16, 64),
              "temperature/ions/row/4": (2, 128), "H/phi/dot/4_64": (6,), "J/z/col/64": (3, 32)}
    for path, shape in shapes.items():
        a = np.load(os.path.join(tmp_path, path + ".npy"))
        assert a.shape == shape and np.isfinite(a).all(), path
        assert np.array_equal(a, out[path])
    assert np.abs(out["E/r/rec/0-32_0-128"][-1]).max() > 0
    assert d.count(slots["beam_electrons"]) > 0  # the bunch entered
