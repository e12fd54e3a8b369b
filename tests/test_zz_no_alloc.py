"""The allocation-free current deposit against the handle-based one and the oracle.

pcg_current_vb_f64_noalloc is for callers that may not call cudaMalloc — a
host code that owns and pre-partitions the device memory, or one that cannot
take cudaMalloc's device synchronisation inside its step loop.  It keeps its
scratch in a fixed device array instead of allocating.  Here it must
reproduce the current that PCG_STAGE_CURRENT of a handle deposits for the
same particles (tolerance: |a - b| <= 1e-12 max|b|, the double-precision
stage tolerance), on two calls in a row with different particles, including
particles in strict axial motion whose J_r overwrite uses the scratch, in
both quirk modes; the second call must leave the device's free memory as it
was.  One case also goes straight to the oracle's current stage.

This file is collected last so that a stop-at-first-failure run has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

from tests.cases import ELECTRONS, particles, small_grid

pytestmark = pytest.mark.gpu

RTOL = 1e-12
QUIRKS = {"reference": 0, "fixed": 1}
MOVE = ("dump_old", "move", "pos_rz", "reflect", "vel_rz", "bind")


def _inputs(grid, seed, n):
    r, z, vr, vphi, vz, w = particles(grid, n, seed)
    still = np.random.default_rng(seed + 1).random(n) < 0.05
    vr = np.where(still, 0.0, vr)      # strict axial motion for 5 % of them
    vphi = np.where(still, 0.0, vphi)
    return (r, z, vr, vphi, vz, w), int(still.sum())


def _handle_path(grid, seed, quirks, n=3000):
    """Particles moved by the stage kernels, then PCG_STAGE_CURRENT."""
    from picopic_b200 import Domain
    d = Domain(grid, "borisrel", "vb", precision="f64", quirks=quirks)
    d.add(ELECTRONS, capacity=n)
    p, still = _inputs(grid, seed, n)
    d.set_particles(0, *p)
    for st in MOVE + ("reset_current", "current"):
        d.stage(st)
    new = d.get_particles(0)
    J = {k: d.get_field(k) for k in ("j_r", "j_phi", "j_z")}
    d.close()
    return (p[0], p[1]), new, J, still


def _noalloc(grid, old, new, quirks):
    """One call on torch-owned device arrays; returns J, the move-error count
    and the device's free bytes just before and just after the call."""
    import torch
    from picopic_b200 import _ffi
    lib = _ffi.load()
    dev = torch.device("cuda", 0)
    t = {k: torch.tensor(np.ascontiguousarray(v), dtype=torch.float64, device=dev)
         for k, v in (("r", new["r"]), ("z", new["z"]), ("r_old", old[0]), ("z_old", old[1]),
                      ("vphi", new["vphi"]), ("w", new["w"]))}
    J = {k: torch.zeros(grid.shape, dtype=torch.float64, device=dev) for k in ("j_r", "j_phi", "j_z")}
    errors = ctypes.c_ulonglong(123)
    stream = torch.cuda.current_stream(dev).cuda_stream
    torch.cuda.synchronize(dev)
    free0 = torch.cuda.mem_get_info(dev)[0]
    rc = lib.pcg_current_vb_f64_noalloc(
        grid.nr, grid.nz, grid.radius, grid.longitude, grid.dt, new["r"].size, -1.0,
        *[ctypes.c_void_p(t[k].data_ptr()) for k in ("r", "z", "r_old", "z_old", "vphi", "w")],
        *[ctypes.c_void_p(J[k].data_ptr()) for k in ("j_r", "j_phi", "j_z")],
        QUIRKS[quirks], ctypes.c_void_p(stream), ctypes.byref(errors))
    torch.cuda.synchronize(dev)
    free1 = torch.cuda.mem_get_info(dev)[0]
    assert rc == 0, rc
    return {k: v.cpu().numpy() for k, v in J.items()}, errors.value, (free0, free1)


def _compare(J, J_ref, what):
    for k in J_ref:
        scale = max(np.abs(J_ref[k]).max(), 1e-300)
        err = np.abs(J[k] - J_ref[k]).max() / scale
        assert err <= RTOL, f"{what}: {k} rel err {err:.3e}"


@pytest.mark.parametrize("quirks", ["reference", "fixed"])
def test_noalloc_matches_stage_current_twice(quirks):
    grid = small_grid(pml=False)
    for call, seed in enumerate((101, 202)):
        old, new, J_ref, still = _handle_path(grid, seed, quirks)
        assert still > 50
        J, errors, (free0, free1) = _noalloc(grid, old, new, quirks)
        assert errors == 0
        _compare(J, J_ref, f"{quirks} call {call + 1}")
        if call == 1:  # the first call may load the module; the second allocates nothing
            assert free1 == free0, f"device free memory changed by {free0 - free1} bytes"


def test_noalloc_matches_oracle():
    from oracle.harness import OracleSim
    grid = small_grid(pml=False)
    orc = OracleSim(grid, "borisrel", "vb")
    orc.add(ELECTRONS)
    p, still = _inputs(grid, 303, 3000)
    assert still > 50
    orc.set_particles(0, *p)
    for st in MOVE:
        orc.stage(st)
    new = orc.get_particles(0)
    orc.stage("reset_current")
    orc.stage("current")
    J_ref = {k: orc.get_field(k) for k in ("j_r", "j_phi", "j_z")}
    # the oracle's own old positions: its reflection stage may move them
    J, errors, _ = _noalloc(grid, (new["r_old"], new["z_old"]), new, "reference")
    assert errors == 0
    _compare(J, J_ref, "oracle")


def test_noalloc_rejects_grids_beyond_its_scratch():
    from picopic_b200 import _ffi
    lib = _ffi.load()
    # (nr+4)*(nz+4) = 1004*1004 > PCG_NOALLOC_MAX_NODES = 262144: refused before any device work
    null = ctypes.c_void_p(0)
    rc = lib.pcg_current_vb_f64_noalloc(1000, 1000, 0.1, 0.1, 1e-13, 0, -1.0, *[null] * 6,
                                        ctypes.c_void_p(1), ctypes.c_void_p(1), ctypes.c_void_p(1),
                                        0, null, None)
    assert rc == -5
