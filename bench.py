#!/usr/bin/env python
"""Throughput of the PIC step: particle-steps/s on one B200.

Workload (default): the beam-plasma wakefield configuration — a 256 x 4096
cell r-z grid (dr = dz = 1e-4 m), electron and proton plasma at 1e17 m^-3
with 50 macroparticles per cell per species (Te = 1 eV, Ti = 0.1 eV),
a 5 MeV electron bunch (1e16 m^-3, radius 2 mm, Gaussian sigma_z = 1 mm,
100 macroparticles per cell of the bunch) injected at z = 0, relativistic
Boris pusher, Villasenor-Buneman current, Yee fields, dt = 0.5 Courant.
The plasma is seeded on the device (Philox); nothing is read from disk.

Timed: exactly K steps after W warm-up steps, CUDA events on the library's
stream, a barrier and device synchronisation on both sides, the maximum over
ranks.  The particle arrays (2.9 GB) exceed L2 (126 MB), so no flush is
needed between steps.  One JSON line is printed by rank 0.

`--impl reference` times the reference's own hot-path sources (compiled by
oracle/Makefile.ref with its release flags) on the host cores instead.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "particle-steps/s on 1 B200 (FP32 vs FP64 oracle); learned vs binary collision speedup"
UNIT = "particle-steps/s"
BYTES_PER_PARTICLE_F32 = 52   # read cell, 2 offsets, 3 velocities, weight (28 B); write all but weight (24 B)
BYTES_PER_PARTICLE_F64 = 88   # read r, z, 3 velocities, weight (48 B); write r, z, 3 velocities (40 B)

C = 3.0e8
DR = 1e-4
WORKLOAD = dict(
    name="beam-plasma wakefield 256x4096, 50 ppc/species e+p, 5 MeV Gaussian bunch",
    nr=256, nz=4096, dr=DR, dz=DR, density=1e17, ppc=50, te=1.0, ti=0.1,
    beam_energy_mev=5.0, beam_density=1e16, beam_radius=2e-3, beam_sigma_z=1e-3,
    beam_ppc=100, pusher="borisrel", current="vb")


def dt_courant(dr):
    return 0.5 * dr / (C * np.sqrt(2.0))


def beam_velocity(mev):
    gamma = 1.0 + mev * 1e6 * 1.6e-19 / (9.1e-31 * C * C)
    return C * np.sqrt(1.0 - 1.0 / gamma ** 2)


def scaled(w, nz=None, ppc=None):
    w = dict(w)
    if nz:
        w["nz"] = nz
    if ppc:
        w["ppc"] = ppc
    return w


# ---------------------------------------------------------------------------
# GPU arm

def make_domain(w, precision, seed=1234, host_beam=False, device=0, beam_capacity=0, quirks="reference"):
    from picopic_b200 import Domain, Geometry
    g = Geometry(w["nr"], w["nz"], w["nr"] * w["dr"], w["nz"] * w["dz"], dt_courant(w["dr"]))
    d = Domain(g, pusher=w["pusher"], current=w["current"], precision=precision, seed=seed,
               device=device, quirks=quirks)
    n = w["nr"] * w["nz"] * w["ppc"]
    vb = beam_velocity(w["beam_energy_mev"])
    cells_b = (w["beam_radius"] / w["dr"]) * (6 * w["beam_sigma_z"] / w["dz"])
    nb = max(int(w["beam_ppc"] * cells_b * 1.05) + 4096, beam_capacity)
    e = d.add(_spec("electrons", -1, 1, 1), capacity=n)
    i = d.add(_spec("ions", 1, 1836, 2), capacity=n)
    if host_beam:
        b = d.add(_spec("beam_electrons", -1, 1, 1000), capacity=nb)
    else:
        b = d.add(_spec("beam_electrons", -1, 1, 1000, beam=dict(
            macro_amount=max(1, int(w["beam_ppc"] * cells_b)), start_time=0.0,
            radius=w["beam_radius"], density=w["beam_density"], amount=1,
            length=6 * w["beam_sigma_z"], distance=0.0, velocity=vb)), capacity=nb)
        d.set_beam_profile(b, "gaussian", w["beam_sigma_z"], w["beam_ppc"])
    d.seed_plasma(e, n, w["density"], w["te"], seed)
    d.seed_plasma(i, n, w["density"], w["ti"], seed + 1)
    return d, (e, i, b), g, vb


class _spec:
    def __init__(self, name, charge, mass, id, beam=None):
        self.name, self.charge, self.mass, self.id, self.beam = name, charge, mass, id, beam


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic():
    p = os.path.join(REPO, "profiles", "ncu_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


def timed_steps(d, K, stream_ptr):
    import torch
    stream = torch.cuda.ExternalStream(stream_ptr)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    d.step(K)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def run_gpu(args):
    import torch
    from picopic_b200.replicas import Replicas
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    rep = Replicas("nccl")
    rank, world = rep.rank, rep.world
    barrier, allmax, allsum = rep.barrier, rep.allmax, rep.allsum

    w = WORKLOAD if not args.small else scaled(WORKLOAD, nz=512, ppc=10)
    w = scaled(w, nz=args.nz, ppc=args.ppc)
    d, slots, g, vb = make_domain(w, "f32", seed=rep.seed(1234), device=local)
    if args.target_blocks:
        d.set_tiling(target_blocks=args.target_blocks)
    d.step(args.warmup)
    d.synchronize()
    diag0 = d.diag()
    p0 = diag0.particle_steps
    d.kernel_times()
    d.enable_timers(True)
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    ms = timed_steps(d, args.steps, d.stream)
    clocks = sampler.stop()
    barrier()
    ms_max = allmax(ms)
    kt = d.kernel_times()
    d.enable_timers(False)
    diag = d.diag()
    psteps = allsum(float(diag.particle_steps - p0))
    value = psteps / (ms_max * 1e-3)
    live = diag.particles
    # roofline of the dominant kernel: algorithmic bytes of one step's particle
    # launches over their measured duration
    part_ms, part_n = kt["particles"]
    per_launch_ms = part_ms / max(part_n, 1)
    particles_per_step = (diag.particle_steps - p0) / args.steps
    alg_bytes = BYTES_PER_PARTICLE_F32 * particles_per_step
    achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = None
    tr = ncu_traffic().get("f32_particle_step")
    if tr:
        traffic = tr["bytes_per_particle"] * particles_per_step
    f64 = None
    e2e = None
    cpu = None
    if not args.no_f64:
        del d
        torch.cuda.empty_cache()
        d64, _, _, _ = make_domain(w, "f64", seed=rep.seed(1234), device=local)
        d64.step(max(2, args.warmup // 2))
        d64.synchronize()
        q0 = d64.diag().particle_steps
        k64 = max(3, args.steps // 5)
        barrier()
        ms64 = allmax(timed_steps(d64, k64, d64.stream))
        q1 = d64.diag().particle_steps
        f64 = {"value": allsum(float(q1 - q0)) / (ms64 * 1e-3), "unit": UNIT,
               "ms_per_step": ms64 / k64, "steps": k64,
               "bytes_per_particle_step": BYTES_PER_PARTICLE_F64}
        del d64
        torch.cuda.empty_cache()
    if not args.no_e2e:
        e2e = run_e2e(w, args, rank, local, barrier, allmax, allsum)
    cfg0 = None
    if not args.no_config0:
        cfg0 = run_config0(args, local, barrier, allmax, allsum, rank, world)
    acc = None
    if not args.no_accuracy and world == 1:
        acc = run_accuracy(w, args, local)
    coll = None
    if not args.no_collisions:
        coll = run_collisions(args, local, barrier, allmax)
    large = None
    if not args.no_large:
        large = run_large(args, local, barrier, allmax, allsum)
    ensemble = None
    if not args.no_ensemble and world == 1:
        ensemble = run_ensemble(args, local)
    slab_leg = None
    if not args.no_slabs and world == 1:
        slab_leg = run_slabs(args, local)
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(w)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w["name"], "grid": [w["nr"], w["nz"]], "particles": int(live),
                       "pusher": w["pusher"], "current": w["current"], "precision": "f32",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (particle arrays 2.9 GB)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "kernel": "f32 fused particle step",
                         "algorithmic_bytes_per_particle": BYTES_PER_PARTICLE_F32,
                         "kernel_ms_per_step": per_launch_ms},
            "kernel_ms_per_step": {k: v[0] / max(v[1], 1) for k, v in kt.items() if v[1]},
            "clocks": clocks,
            "f64": f64,
            "config0": cfg0,
            "e2e": e2e,
            "collisions": coll,
            "large": large,
            "ensemble": ensemble,
            "slabs": slab_leg,
            "accuracy": acc,
            "cpu_baseline": cpu,
            "gpu_launches": int(diag.kernel_launches - diag0.kernel_launches),
        }
        print(json.dumps(line))
    rep.close()


def run_slabs(args, local, counts=(2, 4), steps=20, warmup=3):
    """The wakefield workload at nz = 1024 split along z into slabs of one
    GPU (picopic_b200.slabs, device-to-device exchange after every step)
    against the same workload undivided; wall clock, as the exchange waits
    for each slab's step on the host (a band's particle count)."""
    import time
    import torch
    from picopic_b200 import Domain, Geometry, slabs
    w = scaled(WORKLOAD, nz=1024)
    dt = dt_courant(w["dr"])
    g = Geometry(w["nr"], w["nz"], w["nr"] * w["dr"], w["nz"] * w["dz"], dt)
    vb = beam_velocity(w["beam_energy_mev"])
    cells_b = (w["beam_radius"] / w["dr"]) * (6 * w["beam_sigma_z"] / w["dz"])
    nb = int(w["beam_ppc"] * cells_b * 1.05) + 4096
    beam = dict(macro_amount=max(1, int(w["beam_ppc"] * cells_b)), start_time=0.0, radius=w["beam_radius"],
                density=w["beam_density"], amount=1, length=6 * w["beam_sigma_z"], distance=0.0, velocity=vb)
    species = [_spec("electrons", -1, 1, 1), _spec("ions", 1, 1836, 2), _spec("beam_electrons", -1, 1, 1000)]

    def wall(fn, k):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn(k)
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) * 1e3 / k

    whole, _, _, _ = make_domain(w, "f32", device=local)
    whole.step(warmup)
    ms_whole = wall(whole.step, steps)
    n_whole = whole.diag().particles
    del whole
    torch.cuda.empty_cache()
    out = {"workload": w["name"].replace("4096", "1024"), "precision": "f32", "steps": steps,
           "timing": "wall clock", "undivided_ms_per_step": ms_whole, "particles": int(n_whole)}
    for count in counts:
        def make(geometry, slab):
            d = Domain(geometry, pusher=w["pusher"], current=w["current"], precision="f32", seed=1234,
                       device=local)
            n = geometry.nr * geometry.nz * w["ppc"]
            d.add(species[0], capacity=int(n * 1.1))
            d.add(species[1], capacity=int(n * 1.1))
            d.add(_spec("beam_electrons", -1, 1, 1000, beam=beam if slab.first else None), capacity=nb)
            return d
        ghost = 2 * 6 * w["nr"] * w["ppc"] * 2
        grp = slabs.SlabGroup(g, count, make, species, ghost_capacity=ghost, on_device=True)
        for se in grp.parts:
            d, geo = se.engine, slabs.slab_geometry(g, se.slab)
            n = geo.nr * geo.nz * w["ppc"]
            d.seed_plasma(0, n, w["density"], w["te"], 1234 + 2 * se.slab.index)
            d.seed_plasma(1, n, w["density"], w["ti"], 1235 + 2 * se.slab.index)
            if se.slab.first:
                d.set_beam_profile(2, "gaussian", w["beam_sigma_z"], w["beam_ppc"])
            for t in range(2):  # the seeded ghost cells belong to the neighbours
                d.keep_range(t, se.lo, se.hi)
        grp.exchange()
        grp.step(warmup)
        ms = wall(grp.step, steps)
        live = sum(se.engine.count(t) for se in grp.parts for t in range(3))
        out[f"slabs{count}"] = {"ms_per_step": ms, "over_undivided": ms / ms_whole,
                                "particles_with_ghosts": int(live)}
        del grp
        torch.cuda.empty_cache()
    return out


def run_accuracy(w, args, local):
    """The float path against the FP64 path on the wakefield workload from
    the same seeded start (the same Philox plasma and bunch): relative field
    energy difference after `n` steps, and the charge continuity residual
    of one step, max |Q(n+1) - Q(n) + dt div J| over the nodes behind the
    injection plane (k >= 2) relative to max |Q|, in both precisions.  Both
    runs use PCG_QUIRKS_FIXED: the reference's strict-axial J_r overwrite
    (currentVB.cpp:545-546), which the injected beam's purely axial motion
    triggers, breaks charge conservation by design."""
    import torch
    n = 200 if args.small else 1000
    out = {"steps": n}
    energies = {}
    for prec in ("f32", "f64"):
        d, _, _, _ = make_domain(w, prec, seed=1234, device=local, quirks="fixed")
        d.step(n)
        dg = d.diag()
        energies[prec] = (dg.field_energy_e, dg.field_energy_h, dg.kinetic_energy)
        r = d.continuity_step()
        q = np.abs(r[:, 2:]).max()
        out[f"continuity_{prec}"] = float(q)
        del d
        torch.cuda.empty_cache()
    e32, e64 = energies["f32"], energies["f64"]
    out["field_energy_e_rel_diff"] = abs(e32[0] - e64[0]) / abs(e64[0])
    out["field_energy_h_rel_diff"] = abs(e32[1] - e64[1]) / abs(e64[1])
    out["kinetic_energy_rel_diff"] = abs(e32[2] - e64[2]) / abs(e64[2])
    out["field_energy_f64_J"] = e64[0] + e64[1]
    return out


# The large configuration: 1024 x 16384 cells of 5e-5 m, n = 1e18 m^-3, 12
# macroparticles per cell per species (4.0e8 plasma particles), a 20 MeV
# Gaussian bunch (R = 1 mm, sigma_z = 0.5 mm; its density is not given for
# this configuration, 1e17 m^-3 here), Vay pusher, ZigZag current.
LARGE = dict(
    name="large beam-plasma 1024x16384, 12 ppc/species e+p, 20 MeV Gaussian bunch, Vay + ZigZag",
    nr=1024, nz=16384, dr=5e-5, dz=5e-5, density=1e18, ppc=12, te=1.0, ti=0.1,
    beam_energy_mev=20.0, beam_density=1e17, beam_radius=1e-3, beam_sigma_z=5e-4,
    beam_ppc=100, pusher="vay", current="zigzag")


def _large_leg(w, args, local, barrier, allmax, allsum):
    """One large-grid leg: particle-steps/s of the collisionless step, then
    the step with the learned collision operator (the wide model; binary
    fallback for cells outside its training box) between push and move."""
    from picopic_b200 import learned as L
    d, _, _, _ = make_domain(w, "f32", seed=4321, device=local)
    d.step(3)
    d.synchronize()
    p0 = d.diag().particle_steps
    k = 10 if args.small else 20
    barrier()
    ms = allmax(timed_steps(d, k, d.stream))
    dg = d.diag()
    out = {"workload": w["name"], "grid": [w["nr"], w["nz"]], "particles": int(dg.particles),
           "pusher": w["pusher"], "current": w["current"], "precision": "f32",
           "value": allsum(float(dg.particle_steps - p0)) / (ms * 1e-3), "unit": UNIT,
           "ms_per_step": ms / k, "steps": k}
    d.set_collision_model(*L.load_model(L.WIDE_MODEL_PATH))  # few per cell, n 1e18: the wide model's states
    learned, fallback = d.collide_learned()
    d.set_collisions("learned")
    d.step(1)
    d.synchronize()
    kc = 10
    barrier()
    ms_c = allmax(timed_steps(d, kc, d.stream))
    cells = w["nr"] * w["nz"]
    out["with_learned_collisions"] = {"ms_per_step": ms_c / kc, "steps": kc,
                                      "learned_cell_fraction": learned / cells,
                                      "fallback_cell_fraction": fallback / cells}
    d.close()
    return out


def run_large(args, local, barrier, allmax, allsum):
    """The large configuration in the float path at 12 macroparticles per
    cell per species (4e8 particles), and at 6 (2e8)."""
    import torch
    w = LARGE if not args.small else scaled(LARGE, nz=2048)
    out = _large_leg(w, args, local, barrier, allmax, allsum)
    w6 = dict(w, ppc=6, name=w["name"].replace("12 ppc", "6 ppc"))
    out["ppc6"] = _large_leg(w6, args, local, barrier, allmax, allsum)
    torch.cuda.empty_cache()
    return out


# The batched configuration: 64 independent runs, nr ~ U{64..256}, nz ~
# U{256..2048}, n = 1e17 m^-3, 20-50 macroparticles per cell per species,
# each with the wakefield's 5 MeV Gaussian bunch at a density log-uniform in
# 1e15..1e17 m^-3 (cells of 1e-4 m, dt 0.5 Courant, float path).
ENSEMBLE = dict(name="ensemble of 64 runs: nr U{64..256}, nz U{256..2048}, n 1e17, 20-50 ppc/species e+p, "
                     "5 MeV Gaussian bunch n_b log-uniform 1e15..1e17", runs=64, seed=99)


def run_ensemble(args, local):
    """The batched configuration through pcg_ensemble: particle-steps/s of K
    steps of all runs issued from one host thread with the default tiling,
    from 8 threads with the default tiling, from 8 threads after the
    autotuner's tiling, chosen on the whole ensemble, and, with that tiling,
    as one CUDA graph launch per batch (the device time of each batch)."""
    import torch
    from picopic_b200.ensemble import Ensemble
    rng = np.random.default_rng(ENSEMBLE["seed"])
    nruns = 8 if args.small else ENSEMBLE["runs"]
    runs, sizes = [], []
    for k in range(nruns):
        nr, nz, ppc = int(rng.integers(64, 257)), int(rng.integers(256, 2049)), int(rng.integers(20, 51))
        nb = float(np.exp(rng.uniform(np.log(1e15), np.log(1e17))))
        w = dict(WORKLOAD, nr=nr, nz=nz, ppc=ppc, beam_density=nb)
        d, _, _, _ = make_domain(w, "f32", seed=5000 + k, device=local)
        runs.append(d)
        sizes.append((nr, nz, ppc))
    k_steps = 5 if args.small else 20

    def timed(ens):
        p0 = sum(d.diag().particle_steps for d in runs)
        ms = ens.step(k_steps)
        p1 = sum(d.diag().particle_steps for d in runs)
        return (p1 - p0) / (ms * 1e-3), ms / k_steps

    one = Ensemble(runs, threads=1)
    one.step(3)
    v1, ms1 = timed(one)
    one.close()
    many = Ensemble(runs, threads=8)
    many.step(2)
    v8, ms8 = timed(many)
    choices = many.autotune(trial_steps=3)
    many.step(2)
    vt, mst = timed(many)
    many.set_graph(True)
    many.step(k_steps)  # the first captured batch: instantiates the graph
    vg, msg = timed(many)
    nodes, capture_ms = many.graph_info()
    many.close()
    particles = sum(d.diag().particles for d in runs)
    out = {"workload": ENSEMBLE["name"], "runs": nruns, "particles": int(particles),
           "cells": int(sum(a * b for a, b, _ in sizes)), "steps": k_steps, "unit": UNIT,
           "one_thread_default_tiling": {"value": v1, "ms_per_step": ms1},
           "threads8_default_tiling": {"value": v8, "ms_per_step": ms8},
           "threads8_autotuned": {"value": vt, "ms_per_step": mst},
           "graph_autotuned": {"value": vg, "ms_per_step": msg, "graph_nodes": nodes,
                               "steps_per_graph": k_steps, "host_capture_ms_per_step": capture_ms / k_steps,
                               "note": "each batch of steps of all runs captured into one CUDA graph, "
                                       "one graph launch (device time of the launch)"},
           "autotune_choice": {"target_blocks": choices[0], "times_particle_share": choices[1],
                               "min_particles_per_block": choices[2]}}
    del runs
    torch.cuda.empty_cache()
    return out


# Collisional anisotropy relaxation: 512 x 2048 cells of dr = dz = 1e-5 m
# (the cell size is not given for this workload; 1e-5 m is ~14 Debye
# lengths at 1 eV and 1e20 m^-3), 100 macroparticles per cell per species,
# electrons T_par = 2 eV, T_perp = 1 eV, ions 0.5 eV, dt = 0.5 Courant.
COLLISIONS = dict(name="collisional anisotropy relaxation 512x2048, 100 ppc/species e+p, n 1e20",
                  nr=512, nz=2048, dr=1e-5, density=1e20, ppc=100, te_par=2.0, te_perp=1.0, ti=0.5)


def run_collisions(args, local, barrier, allmax):
    """One collision step on the collisional workload, binary (Perez 2012,
    FP64 per pair) against learned (BF16 tensor-core MLP + FP64 transform):
    device time per step, and the electron anisotropy relaxation time of
    both operators at the same start on a 64 x 128-cell slab (the binary
    one averaged over independent passes)."""
    import torch
    from picopic_b200 import Domain, Geometry
    from picopic_b200 import learned as L
    c = COLLISIONS
    if args.small:
        c = dict(c, nr=128, nz=256)
    if args.coll_nz:
        c = dict(c, nz=args.coll_nz)
    g = Geometry(c["nr"], c["nz"], c["nr"] * c["dr"], c["nz"] * c["dr"], dt_courant(c["dr"]))
    n = c["nr"] * c["nz"] * c["ppc"]
    d = Domain(g, precision="f32", quirks="fixed", seed=11, device=local)
    d.add(L.ELECTRONS, capacity=n)
    d.add(L.IONS, capacity=n)
    d.seed_plasma_cells(0, c["ppc"], c["density"], c["te_par"], c["te_perp"], seed=1)
    d.seed_plasma_cells(1, c["ppc"], c["density"], c["ti"], seed=2)
    d.set_collision_model(*L.load_model())
    # the slots grouped by tile, as every step keeps them (the collision
    # passes of a running simulation see that layout)
    d.tile_sort(0)
    d.tile_sort(1)
    d.collide()
    d.collide_learned()
    d.synchronize()
    stream = torch.cuda.ExternalStream(d.stream)

    def timed(fn, k):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = [fn() for _ in range(k)]
        e1.record(stream)
        e1.synchronize()
        return allmax(e0.elapsed_time(e1)) / k, out

    bin_ms, _ = timed(d.collide, 3)
    lrn_ms, counts = timed(d.collide_learned, 10)
    del d
    torch.cuda.empty_cache()
    cells = c["nr"] * c["nz"]
    out = {"workload": c["name"] if not args.coll_nz else f"{c['name']} at {c['nr']}x{c['nz']}",
           "particles": 2 * n, "precision": "f32 particles, FP64 collision arithmetic",
           "binary_ms_per_step": bin_ms, "learned_ms_per_step": lrn_ms, "speedup": bin_ms / lrn_ms,
           "learned_cell_fraction": counts[-1][0] / cells, "fallback_cell_fraction": counts[-1][1] / cells}
    if args.no_relax:
        return out
    gs = Geometry(64, 128, 64 * c["dr"], 128 * c["dr"], 1e-13)
    tb, eb, _ = L.initial_relaxation_time(gs, "binary", passes=60, density=3e20, device=local)
    tl, _, _ = L.initial_relaxation_time(gs, "learned", passes=1, density=3e20, device=local)
    out["relaxation_time_steps"] = {"slab": "64x128 cells, 100 ppc, n 3e20, dt 1e-13, Te 2/1 eV, Ti 0.5 eV",
                                    "binary": tb, "binary_stderr": eb, "learned": tl, "ratio": tl / tb}
    return out


def run_e2e(w, args, rank, local, barrier, allmax, allsum):
    """Same metric through the C ABI with host buffers: every step appends
    that step's bunch slice from pinned host memory and reads the device
    status block back (pcg_step_status: a step late, so that a step stays
    queued; pcg_synchronize after the last)."""
    import torch
    K = args.steps
    vb = beam_velocity(w["beam_energy_mev"])
    dl = vb * dt_courant(w["dr"])
    mps = w["beam_ppc"] * (w["beam_radius"] / w["dr"]) * (dl / w["dz"])
    d, slots, g, vb = make_domain(w, "f32", seed=4321 + 7919 * rank, host_beam=True, device=local,
                                  beam_capacity=int(mps * (args.warmup + K)) + 4096)
    rng = np.random.default_rng(99 + rank)
    slab = np.pi * (w["beam_radius"] ** 2 - (0.5 * w["dr"]) ** 2) * dl
    w0 = w["beam_density"] * slab / mps
    steps_total = args.warmup + K
    slices = []
    for m in range(steps_total):
        cnt = int(np.floor((m + 1) * mps) - np.floor(m * mps))
        u0, u1 = rng.random(cnt), rng.random(cnt)
        r = np.sqrt((0.5 * w["dr"]) ** 2 + u0 * (w["beam_radius"] ** 2 - (0.5 * w["dr"]) ** 2))
        z = dl * u1 + 0.5 * w["dz"]
        s = (m + 1) * dl - dl * u1 - 3 * w["beam_sigma_z"]
        wt = w0 * np.exp(-s * s / (2 * w["beam_sigma_z"] ** 2))
        buf = torch.empty((6, cnt), dtype=torch.float64, pin_memory=True).numpy()
        buf[0], buf[1], buf[2], buf[3], buf[4], buf[5] = r, z, 0.0, 0.0, vb, wt
        slices.append(buf)
    beam = slots[2]

    def one(m):
        b = slices[m]
        if b.shape[1]:
            d.set_particles(beam, *b, append=True)  # waits for its own copies only
        d.step(1)
        d.step_status()  # the status block of every step, read one step late

    for m in range(args.warmup):
        one(m)
    d.synchronize()
    p0 = d.diag().particle_steps
    h2d = sum(slices[m].nbytes for m in range(args.warmup, steps_total))
    barrier()
    t0 = time.perf_counter()
    for m in range(args.warmup, steps_total):
        one(m)
    d.synchronize()  # the last step's status
    t1 = time.perf_counter()
    barrier()
    el = allmax(t1 - t0)
    p1 = d.diag().particle_steps
    del d
    torch.cuda.empty_cache()
    return {"value": allsum(float(p1 - p0)) / el, "unit": UNIT, "h2d_bytes_per_step": h2d / K,
            "d2h_bytes_per_step": 32, "ms_per_step": el * 1e3 / K,
            "path": "pcg_append_species (pinned host, bunch slice) + pcg_step(1) + pcg_step_status (each step's status block, read a step late), pcg_synchronize at the end"}


# The plain FP64 configuration: 128 x 512 cells of 1e-4 m, electrons and
# protons at 1e17 m^-3, 20 macroparticles per cell per species (r = R sqrt(U),
# z uniform), Maxwellian at Te = 1 eV, Ti = 0.1 eV, relativistic Boris, VB,
# Yee, dt 0.5 Courant, no bunch, no collisions.
CONFIG0 = dict(name="plain FP64 plasma 128x512, 20 ppc/species e+p, Te 1 eV, Ti 0.1 eV",
               nr=128, nz=512, dr=DR, dz=DR, density=1e17, ppc=20, te=1.0, ti=0.1,
               pusher="borisrel", current="vb")


def run_config0(args, local, barrier, allmax, allsum, rank, world):
    """The plain configuration in FP64 on the GPU (particle-steps/s over K
    steps) and, on rank 0 of a one-GPU run, the reference's own hot path on
    one host core over the whole configuration with host-generated particles
    of the same distribution (2 steps after one warm-up), so that the FP64
    speed-up is stated without a precision change."""
    import torch
    from picopic_b200 import Domain, Geometry
    w = CONFIG0
    g = Geometry(w["nr"], w["nz"], w["nr"] * w["dr"], w["nz"] * w["dz"], dt_courant(w["dr"]))
    d = Domain(g, pusher=w["pusher"], current=w["current"], precision="f64", seed=1234, device=local)
    n = w["nr"] * w["nz"] * w["ppc"]
    e = d.add(_spec("electrons", -1, 1, 1), capacity=n)
    i = d.add(_spec("ions", 1, 1836, 2), capacity=n)
    d.seed_plasma(e, n, w["density"], w["te"], 1234)
    d.seed_plasma(i, n, w["density"], w["ti"], 1235)
    d.step(args.warmup)
    d.synchronize()
    p0 = d.diag().particle_steps
    k = max(10, args.steps)
    barrier()
    ms = allmax(timed_steps(d, k, d.stream))
    p1 = d.diag().particle_steps
    out = {"workload": w["name"], "grid": [w["nr"], w["nz"]], "particles": int(d.diag().particles),
           "precision": "f64", "pusher": w["pusher"], "current": w["current"],
           "value": allsum(float(p1 - p0)) / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / k, "steps": k,
           "bytes_per_particle_step": BYTES_PER_PARTICLE_F64}
    del d
    torch.cuda.empty_cache()
    if rank == 0 and world == 1 and not args.no_cpu:
        sim, kind, npart = _ref_domain(w, w["nz"], 11)
        sim.step(1)
        t0 = time.perf_counter()
        steps = 2
        sim.step(steps)
        el = time.perf_counter() - t0
        out["cpu_reference_1core"] = {"value": npart * steps / el, "unit": UNIT, "cores": 1, "kind": kind,
                                      "sample": f"the whole configuration, {npart} particles, {steps} steps "
                                                "after 1, reference hot path compiled with its release flags"}
        out["gpu_over_cpu_1core"] = out["value"] / out["cpu_reference_1core"]["value"]
    return out


# ---------------------------------------------------------------------------
# CPU arms (the reference's own sources, compiled by oracle/Makefile.ref)

def _plasma_sample(w, nz, seed):
    """Host-generated plasma of the same distribution on a z-slab."""
    rng = np.random.default_rng(seed)
    R, L, dr, dz = w["nr"] * w["dr"], nz * w["dz"], w["dr"], w["dz"]
    n = w["nr"] * nz * w["ppc"]
    out = []
    for mass, T in ((1.0, w["te"]), (1836.0, w["ti"])):
        r0, r1 = 0.5 * dr, R - 0.5 * dr
        r = np.sqrt(r0 ** 2 + rng.random(n) * (r1 ** 2 - r0 ** 2))
        z = 0.5 * dz + rng.random(n) * (L - dz)
        s = np.sqrt(T * 1.6e-19 / (mass * 9.1e-31))
        v = rng.normal(size=(3, n)) * s
        wt = np.full(n, w["density"] * np.pi * (r1 ** 2 - r0 ** 2) * (L - dz) / n)
        out.append((r, z, v[0], v[1], v[2], wt))
    return out


def _ref_domain(w, nz, seed):
    from oracle.harness import GridSpec, RefSim, SpeciesSpec, reference_available, OracleSim
    grid = GridSpec(w["nr"], nz, w["nr"] * w["dr"], nz * w["dz"], dt_courant(w["dr"]))
    if reference_available("borisrel", "vb", perf=True):
        sim, kind = RefSim(grid, "borisrel", "vb", perf=True), "reference"
    else:
        sim, kind = OracleSim(grid, "borisrel", "vb"), "port"
    sim.add(SpeciesSpec("electrons", -1, 1, id=1))
    sim.add(SpeciesSpec("ions", 1, 1836, id=2))
    n = 0
    for sid, p in enumerate(_plasma_sample(w, nz, seed)):
        sim.set_particles(sid, *p)
        n += p[0].size
    return sim, kind, n


def cpu_baseline(w, nz=256, steps=2):
    """One core, one domain: a 256 x 256 z-slab of the workload (6.6e6
    particles), 2 full steps of the reference step order."""
    sim, kind, n = _ref_domain(w, nz, 7)
    sim.step(1)
    t0 = time.perf_counter()
    sim.step(steps)
    el = time.perf_counter() - t0
    return {"value": n * steps / el, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"{w['nr']}x{nz} z-slab of the workload, {n} particles, {steps} steps, "
                      "reference hot path compiled with its release flags"}


def _smb_reference(w, steps, warmup=1):
    """The reference's own scheduler (src/SMB.cpp, unmodified, release flags,
    OpenMP over domains, its overlays): the workload's radial extent cut into
    square 64 x 64-cell domains (its overlays need square domains, and each
    axis 1 or an even number of them), with enough z-domains that every host
    thread has one.  Plasma from the reference's own initialiser at the
    workload's density, temperatures and macroparticles per cell."""
    from oracle.harness import GridSpec, SmbSim, SpeciesSpec
    cells = 64
    threads = len(os.sched_getaffinity(0))
    r_dom = max(1, w["nr"] // cells)
    if r_dom > 1 and r_dom % 2:
        r_dom -= 1
    z_dom = max(2, 2 * -(-threads // (2 * r_dom)))
    nr, nz = r_dom * cells, z_dom * cells
    grid = GridSpec(nr, nz, nr * w["dr"], nz * w["dz"], dt_courant(w["dr"]))
    smb = SmbSim(grid, r_dom, z_dom)
    smb.seed(7)
    for sid, (name, q, m, T) in enumerate((("electrons", -1, 1, w["te"]), ("ions", 1, 1836, w["ti"]))):
        smb.add_species(SpeciesSpec(name, q, m, id=sid), nr * nz * w["ppc"], w["density"], T)
    smb.build()
    smb.distribute()
    n = smb.particles()
    assert smb.step(warmup) == 0
    t0 = time.perf_counter()
    assert smb.step(steps) == 0
    el = time.perf_counter() - t0
    sample = (f"reference SMB scheduler, {r_dom} x {z_dom} domains of {cells} x {cells} cells "
              f"({nr} x {nz}, {n} particles), {smb.threads()} OpenMP threads, {steps} steps")
    return n, el, smb.threads(), sample


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = WORKLOAD if not args.small else scaled(WORKLOAD, nz=512, ppc=10)
    # the same K and W as the GPU arm (a slab step takes ~0.2 s on 16 threads),
    # at least 8 steps after 1, at most 60 after 10 so that the arm ends
    # within a few minutes on small hosts
    steps, warmup = max(8, min(args.steps, 60)), max(1, min(args.warmup, 10))
    from oracle.harness import smb_available
    if smb_available():
        n, el, threads, sample = _smb_reference(w, steps, warmup)
        value = n * steps / el
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
                "steps": steps, "warmup": warmup, "ms_per_step": el * 1e3 / steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": w["name"], "sample": sample},
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                                 "sample": sample},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    threads = os.cpu_count() or 1
    nz = 64 if not args.small else 32
    sims = []
    kind = None
    for t in range(threads):
        s, kind, n = _ref_domain(w, nz, 100 + t)
        sims.append((s, n))
    for s, _ in sims:  # warm-up steps per domain
        s.step(warmup)

    def work(s):
        s.step(steps)

    t0 = time.perf_counter()
    th = [threading.Thread(target=work, args=(s,)) for s, _ in sims]
    for t in th:
        t.start()
    for t in th:
        t.join()
    el = time.perf_counter() - t0
    total = sum(n for _, n in sims) * steps
    value = total / el
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
            "steps": steps, "warmup": warmup, "ms_per_step": el * 1e3 / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": w["name"], "sample": f"{threads} domains of {w['nr']}x{nz} cells, "
                                                        f"one per host thread"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"{threads} independent {w['nr']}x{nz} z-slab domains "
                                       f"({sum(n for _, n in sims)} particles), {steps} steps"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--small", action="store_true", help="a reduced grid for quick checks")
    ap.add_argument("--ppc", type=int, default=None, help="override plasma macroparticles per cell")
    ap.add_argument("--nz", type=int, default=None, help="override the axial cell count")
    ap.add_argument("--no-f64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-collisions", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-config0", action="store_true")
    ap.add_argument("--no-slabs", action="store_true")
    ap.add_argument("--coll-nz", type=int, default=0, help="axial cells of the collisional workload (profiling)")
    ap.add_argument("--no-relax", action="store_true", help="skip the relaxation-time measurement")
    ap.add_argument("--target-blocks", type=int, default=0,
                    help="float step: blocks the tile sort aims for (0 keeps the default)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
