"""The CPU oracle against golden fixtures made by the compiled reference.

tests/golden/make_golden.py ran the reference's own sources (oracle/_ref)
on seeded inputs and stored the inputs plus the outputs after 1 and 10
steps.  The oracle must reproduce them bit for bit; this pins the oracle on
machines that do not have the reference sources.
"""
import glob
import os

import numpy as np
import pytest

from oracle.harness import FIELDS, GridSpec, OracleSim
from tests.cases import ELECTRONS, IONS, beam_spec

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _grid(g):
    return GridSpec(int(g[0]), int(g[1]), g[2], g[3], g[4], g[5],
                    pml_size=tuple(int(x) for x in g[6:10]), pml_sigma=(g[10], g[11]))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_reference_fixture(path):
    d = np.load(path)
    grid = _grid(d["grid"])
    pusher, current = [str(x) for x in d["switches"]]
    species = [ELECTRONS, IONS] + ([beam_spec(grid, macro_amount=4000)] if bool(d["beam"]) else [])
    sim = OracleSim(grid, pusher, current)
    for sp in species:
        sim.add(sp)
    nsp = int(d["nsp"])
    for sid in range(nsp):
        if species[sid].beam is None:
            sim.set_particles(sid, *[d[f"in/p{sid}/{k}"] for k in ("r", "z", "vr", "vphi", "vz", "w")])
    for k in FIELDS:
        sim.set_field(k, d[f"in/{k}"])
    sim.set_rng("mt19937", int(d["seed"]))
    for tag, steps in (("step1", 1), ("step10", 9)):
        assert sim.step(steps) == 0
        for k in FIELDS:
            np.testing.assert_array_equal(sim.get_field(k), d[f"{tag}/{k}"], err_msg=f"{tag} {k}")
        for sid in range(nsp):
            p = sim.get_particles(sid)
            for k, v in p.items():
                np.testing.assert_array_equal(v, d[f"{tag}/p{sid}/{k}"], err_msg=f"{tag} p{sid} {k}")


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 5


def test_oracle_collisions_match_reference_fixture():
    """tests/golden/collisions/p12_pass.npz: one Perez-2012 pass of the
    reference (no shuffle, mt19937 seeded) reproduced bit for bit."""
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "collisions", "p12_pass.npz"))
    grid = _grid(d["grid"])
    o = OracleSim(grid, quirks="reference")
    o.add(ELECTRONS)
    o.add(IONS)
    for sid in (0, 1):
        o.set_particles(sid, *[d[f"in/p{sid}/{k}"] for k in ("r", "z", "vr", "vphi", "vz", "w")])
    o.set_rng("mt19937", int(d["seed"]))
    assert o.collide() > 0
    for sid in (0, 1):
        p = o.get_particles(sid)
        for k in ("vr", "vphi", "vz"):
            np.testing.assert_array_equal(p[k], d[f"out/p{sid}/{k}"], err_msg=f"species {sid} {k}")


def test_oracle_ta77s_matches_reference_fixture():
    """tests/golden/collisions/ta77s_pass.npz: one Takizuka-Abe pass of the
    reference with its velocity correction (no shuffle, mt19937 seeded)
    reproduced bit for bit."""
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "collisions", "ta77s_pass.npz"))
    grid = _grid(d["grid"])
    o = OracleSim(grid, quirks="reference")
    o.add(ELECTRONS)
    o.add(IONS)
    for sid in (0, 1):
        o.set_particles(sid, *[d[f"in/p{sid}/{k}"] for k in ("r", "z", "vr", "vphi", "vz", "w")])
    o.set_rng("mt19937", int(d["seed"]))
    assert o.collide(scheme="ta77s") > 0
    for sid in (0, 1):
        p = o.get_particles(sid)
        for k in ("vr", "vphi", "vz"):
            np.testing.assert_array_equal(p[k], d[f"out/p{sid}/{k}"], err_msg=f"species {sid} {k}")


def test_oracle_sk98_matches_reference_fixture():
    """tests/golden/collisions/sk98_pass.npz: one CollisionsSK98 pass of the
    reference (no shuffle, mt19937 seeded) reproduced bit for bit."""
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "collisions", "sk98_pass.npz"))
    grid = _grid(d["grid"])
    o = OracleSim(grid, quirks="reference")
    o.add(ELECTRONS)
    o.add(IONS)
    for sid in (0, 1):
        o.set_particles(sid, *[d[f"in/p{sid}/{k}"] for k in ("r", "z", "vr", "vphi", "vz", "w")])
    o.set_rng("mt19937", int(d["seed"]))
    assert o.collide(scheme="sk98") > 0
    for sid in (0, 1):
        p = o.get_particles(sid)
        for k in ("vr", "vphi", "vz"):
            np.testing.assert_array_equal(p[k], d[f"out/p{sid}/{k}"], err_msg=f"species {sid} {k}")
