"""`bench.py --impl reference`: the line the reference arm prints.

Runs the arm at reduced size on the CPU (it is the reference's own code,
compiled by oracle/Makefile.ref; the GPU is not involved) and checks the
keys of its JSON line; a rank other than 0 prints nothing and exits 0.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--small", "--steps", "25"],
                          cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_line():
    from oracle.harness import reference_available, smb_available
    if not (smb_available() or reference_available("borisrel", "vb", perf=True)):
        pytest.skip("compiled reference not built (oracle/Makefile.ref)")
    r = _run({"RANK": "0"})
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] == 25 and line["warmup"] == 5  # the K and W it was given
    assert line["unit"] == "particle-steps/s" and line["config"]["workload"]
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["cores"] >= 1 and cb["kind"] == "reference" and cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    if smb_available():
        assert "SMB" in cb["sample"]


def test_reference_arm_other_ranks_are_silent():
    r = _run({"RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
