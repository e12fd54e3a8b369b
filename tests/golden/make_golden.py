"""Generate golden fixtures from the reference's own compiled sources.

Run from the repository root after ``make -f oracle/Makefile.ref``:

    python tests/golden/make_golden.py

Each case stores its seeded inputs (particles, fields, grid, switches) and
the reference's outputs after 1 and 10 full steps, so that the CPU oracle
can be checked on machines where the reference sources are absent.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.harness import FIELDS, RefSim  # noqa: E402
from tests.cases import ELECTRONS, IONS, beam_spec, load, small_grid, thermal_plasma  # noqa: E402

CASES = [
    ("borisrel_vb_beam", "borisrel", "vb", True, True),
    ("boris_vb", "boris", "vb", False, True),
    ("vay_zigzag", "vay", "zigzag", False, False),
    ("hc_vb", "hc", "vb", False, True),
    ("borisrel_zigzag", "borisrel", "zigzag", True, False),
]
N = 200
SEED = 2024


def snapshot(sim, nsp, tag, out):
    for k in FIELDS:
        out[f"{tag}/{k}"] = sim.get_field(k)
    for sid in range(nsp):
        p = sim.get_particles(sid)
        for k, v in p.items():
            out[f"{tag}/p{sid}/{k}"] = v


def main():
    for name, pusher, current, beam, pml in CASES:
        grid = small_grid(nr=12, nz=24, pml=pml)
        species = [ELECTRONS, IONS] + ([beam_spec(grid, macro_amount=4000)] if beam else [])
        sim = RefSim(grid, pusher, current)
        load(sim, grid, species, N, seed=SEED)
        sim.seed(SEED)
        out = {"grid": np.array([grid.nr, grid.nz, grid.radius, grid.longitude, grid.dt,
                                 grid.t_start, *grid.pml_size, *grid.pml_sigma]),
               "switches": np.array([pusher, current], dtype="U16"),
               "nsp": np.array(len(species)), "seed": np.array(SEED), "n": np.array(N),
               "beam": np.array(beam)}
        snapshot(sim, len(species), "in", out)
        assert sim.step(1) == 0
        snapshot(sim, len(species), "step1", out)
        assert sim.step(9) == 0
        snapshot(sim, len(species), "step10", out)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print("wrote", name)


def collisions_fixture(scheme="p12"):
    """One collision pass of the reference (no shuffle, mt19937): scheme
    "p12" (CollisionsP12), "ta77s" (CollisionsTA77S with its velocity
    correction) or "sk98" (CollisionsSK98)."""
    grid = small_grid(nr=8, nz=16, pml=False)
    n = grid.nr * grid.nz * 10
    sim = RefSim(grid)
    sim.add(ELECTRONS)
    sim.add(IONS)
    sim.set_particles(0, *thermal_plasma(grid, n, 1, 1.0, 1.0, 1e20, t_par_ratio=2.0))
    sim.set_particles(1, *thermal_plasma(grid, n + 7, 2, 1836.0, 0.5, 1e20))
    sim.seed(SEED)
    out = {"grid": np.array([grid.nr, grid.nz, grid.radius, grid.longitude, grid.dt,
                             grid.t_start, 0, 0, 0, 0, 0.0, 0.0]),
           "seed": np.array(SEED), "n": np.array(n)}
    for sid in (0, 1):
        for k, v in sim.get_particles(sid).items():
            out[f"in/p{sid}/{k}"] = v
    out["ncol"] = np.array(sim.collide(scheme=scheme))
    for sid in (0, 1):
        for k, v in sim.get_particles(sid).items():
            out[f"out/p{sid}/{k}"] = v
    np.savez_compressed(os.path.join(HERE, "collisions", f"{scheme}_pass.npz"), **out)
    print(f"wrote collisions/{scheme}_pass")


if __name__ == "__main__":
    main()
    collisions_fixture("p12")
    collisions_fixture("ta77s")
    collisions_fixture("sk98")
