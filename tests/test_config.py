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
