"""The acceptance figures of the float production path, at a size that runs in seconds.

A reduced wakefield workload: the benchmark's plasma (1e17 m^-3, Te 1 eV, Ti 0.1 eV) and its
5 MeV Gaussian bunch on 256 x 512 cells of 1e-4 m at 10 macroparticles per cell per
species, relativistic Boris and Villasenor-Buneman in the fixed-quirks mode, the float path
and the FP64 path started from the same seeded particles.

* Field energy: after 1000 steps the float path's electric field energy is within 1e-4 of
  the FP64 path's (RTOL_ENERGY; measured 6.9e-5 here and 7.6e-5 on the full 256 x 4096
  grid), the magnetic within 1e-4 (measured 1.4e-5).
* Charge continuity of step 1001, max |Q(n+1) - Q(n) + dt div J| over the nodes behind the
  injection plane relative to max |Q|: the FP64 path within 1e-10 (measured 5e-13).  The
  float path closes it to RTOL_CONT_F32 = 2e-8 (measured 6-8e-9): its node charges come from
  float offsets and its current is accumulated in float, so it conserves to float rounding
  (each node carries ~1e-7 of the charge its particles move in rounding), not to 1e-10.
  test_float_continuity_meets_1e10 states the 1e-10 target as an expected failure (strict:
  it must keep failing until the path meets it).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS = 1000
RTOL_ENERGY = 1e-4
RTOL_CONT_F64 = 1e-10
RTOL_CONT_F32 = 2e-8
TARGET_CONT = 1e-10


@pytest.fixture(scope="module")
def runs():
    """Both precisions after STEPS steps and one more step's continuity residual."""
    import torch

    import bench
    w = bench.scaled(bench.WORKLOAD, nz=512, ppc=10)
    out = {}
    for prec in ("f32", "f64"):
        d, _, _, _ = bench.make_domain(w, prec, seed=1234, quirks="fixed")
        d.step(STEPS)
        dg = d.diag()
        r = d.continuity_step()
        out[prec] = {"e": dg.field_energy_e, "h": dg.field_energy_h,
                     "cont": float(np.abs(r[:, 2:]).max())}
        d.close()
        del d
        torch.cuda.empty_cache()
    return out


def test_float_field_energy_matches_fp64(runs):
    a, b = runs["f32"], runs["f64"]
    assert b["e"] > 0 and b["h"] > 0
    assert abs(a["e"] - b["e"]) <= RTOL_ENERGY * abs(b["e"])
    assert abs(a["h"] - b["h"]) <= RTOL_ENERGY * abs(b["h"])


def test_fp64_continuity_meets_1e10(runs):
    assert runs["f64"]["cont"] <= RTOL_CONT_F64


def test_float_continuity_to_float_rounding(runs):
    assert runs["f32"]["cont"] <= RTOL_CONT_F32


@pytest.mark.xfail(strict=True, reason="the float path conserves charge to float rounding (6-8e-9), not 1e-10")
def test_float_continuity_meets_1e10(runs):
    assert runs["f32"]["cont"] <= TARGET_CONT
