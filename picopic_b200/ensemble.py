"""Many independent runs advanced together (pcg_ensemble_* in include/pcg.h).

    runs = [Domain(...), ...]            # each with its own grid, species, beam
    ens = Ensemble(runs, threads=8)
    ens.autotune(trial_steps=5)          # a tiling per run, timed run by run
    ms = ens.step(100)                   # device ms of the whole batch
    ens.set_graph(True)
    ms = ens.step(20)                    # 20 steps of all runs as one graph launch
"""
from __future__ import annotations

import ctypes

from . import _ffi
from ._ffi import PcgError

# (target blocks per run, shared: times the run's share of the particles, min particles per block)
CANDIDATES = [(1184, False, 1024), (148, False, 2048), (1184, True, 1024), (4736, True, 512),
              (592, False, 512), (2368, False, 512)]


class Ensemble:
    def __init__(self, runs, threads: int = 8):
        self.lib = _ffi.load()
        self.runs = list(runs)  # keeps the Domains (and their handles) alive
        arr = (ctypes.c_void_p * len(self.runs))(*[d.h.value if hasattr(d.h, "value") else d.h
                                                    for d in self.runs])
        e = ctypes.c_void_p()
        rc = self.lib.pcg_ensemble_create(arr, len(self.runs), threads, ctypes.byref(e))
        if rc != 0:
            raise PcgError(rc, "pcg_ensemble_create", "")
        self.e = e

    def step(self, n: int = 1) -> float:
        """Advance every run by n steps; returns the batch's device time (ms)."""
        ms = ctypes.c_float(0.0)
        rc = self.lib.pcg_ensemble_step(self.e, int(n), ctypes.byref(ms))
        if rc != 0:
            raise PcgError(rc, "pcg_ensemble_step", "")
        return float(ms.value)

    def autotune(self, trial_steps: int = 5):
        """The fastest of CANDIDATES, timed on the whole ensemble and applied
        to every run; the runs advance by 6 * (trial_steps + 1) steps.
        Returns the chosen candidate."""
        choice = ctypes.c_int(0)
        rc = self.lib.pcg_ensemble_autotune(self.e, int(trial_steps), ctypes.byref(choice))
        if rc != 0:
            raise PcgError(rc, "pcg_ensemble_autotune", "")
        return CANDIDATES[choice.value]

    def set_graph(self, on: bool = True):
        """Graph mode: each later step(n) captures the n steps of every run
        into one CUDA graph and issues it as one launch (the first batch of
        an ensemble steps directly)."""
        rc = self.lib.pcg_ensemble_set_graph(self.e, 1 if on else 0)
        if rc != 0:
            raise PcgError(rc, "pcg_ensemble_set_graph", "")

    def graph_info(self):
        """(nodes of the last graph, host ms of its capture and instantiation or update)."""
        nodes, ms = ctypes.c_ulonglong(0), ctypes.c_float(0.0)
        rc = self.lib.pcg_ensemble_graph_info(self.e, ctypes.byref(nodes), ctypes.byref(ms))
        if rc != 0:
            raise PcgError(rc, "pcg_ensemble_graph_info", "")
        return int(nodes.value), float(ms.value)

    def close(self):
        if getattr(self, "e", None):
            self.lib.pcg_ensemble_destroy(self.e)
            self.e = None

    def __del__(self):
        self.close()
