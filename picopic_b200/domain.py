"""Host-side mirror of the reference's per-domain façade, on the GPU.

:class:`Domain` exposes the methods that the reference scheduler (``SMB``)
calls on ``Domain`` (src/domain.cpp:86-204) — ``weight_field_e``,
``weight_field_h``, ``push_particles``, ``dump_particle_positions_to_old``,
``update_particles_coords``, ``particles_back_position_to_rz``, ``reflect``,
``particles_back_velocity_to_rz``, ``bind_cell_numbers``,
``reset_current``, ``weight_current``, ``manage_beam`` — each one a CUDA
kernel behind the C ABI, plus :meth:`step`, the fused step of
src/PiCoPiC.cpp:326-347.  Field and particle access follows the reference
layouts (``Grid<double>`` with a 2-cell halo; ``SpecieP::particles``).

Errors surface as :class:`PcgError`, the counterpart of the reference's
``LOG_S(FATAL)`` aborts.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from ._ffi import Band, Config, Diagnostics, PcgError, load

PUSHERS = {"boris": 0, "borisadaptive": 1, "borisrel": 2, "vay": 3, "hc": 4}
CURRENTS = {"vb": 0, "zigzag": 1}
PRECISIONS = {"f64": 0, "f32": 1}
QUIRKS = {"reference": 0, "fixed": 1}
STAGES = ["inject", "field_e", "field_h", "push", "dump_old", "move", "pos_rz", "reflect",
          "vel_rz", "bind", "collect", "reset_current", "current", "advance_time"]
STAGE = {n: i for i, n in enumerate(STAGES)}
FIELDS = ["e_r", "e_phi", "e_z", "h_r", "h_phi", "h_z", "hat_r", "hat_phi", "hat_z",
          "j_r", "j_phi", "j_z"]
FIELD = {n: i for i, n in enumerate(FIELDS)}

_PD = ctypes.POINTER(ctypes.c_double)
_PI32 = ctypes.POINTER(ctypes.c_int32)


def _dp(a):
    return a.ctypes.data_as(_PD)


@dataclass
class Geometry:
    """One domain at the origin with all four walls (src/cfg.cpp:379-429)."""
    nr: int
    nz: int
    radius: float
    longitude: float
    dt: float
    t_start: float = 0.0
    pml_size: tuple = (0, 0, 0, 0)
    pml_sigma: tuple = (0.0, 0.0)

    @property
    def dr(self):
        return self.radius / self.nr

    @property
    def dz(self):
        return self.longitude / self.nz

    @property
    def shape(self):
        return (self.nr + 4, self.nz + 4)


class Domain:
    """A simulation domain on one GPU, driven like the reference ``Domain``."""

    def __init__(self, geometry, pusher="borisrel", current="vb", precision="f64",
                 quirks="reference", device=0, seed=0):
        self.lib = load()
        self.grid = geometry
        c = Config()
        c.nr, c.nz = int(geometry.nr), int(geometry.nz)
        c.radius, c.longitude = float(geometry.radius), float(geometry.longitude)
        c.dt, c.t_start = float(geometry.dt), float(geometry.t_start)
        for i in range(4):
            c.pml_size[i] = int(geometry.pml_size[i])
        c.pml_sigma[0], c.pml_sigma[1] = float(geometry.pml_sigma[0]), float(geometry.pml_sigma[1])
        c.pusher, c.current = PUSHERS[pusher], CURRENTS[current]
        c.precision, c.quirks = PRECISIONS[precision], QUIRKS[quirks]
        c.device, c.seed = int(device), int(seed)
        h = ctypes.c_void_p()
        rc = self.lib.pcg_create(ctypes.byref(c), ctypes.byref(h))
        if rc != 0:
            raise PcgError(rc, "pcg_create", "invalid configuration or no CUDA device")
        self.h = h
        self.precision = precision
        self.device = int(device)
        self.species = []

    # -- error handling ------------------------------------------------------
    def _check(self, rc, where):
        if rc != 0:
            msg = self.lib.pcg_last_error(self.h)
            raise PcgError(rc, where, msg.decode() if msg else "")
        return rc

    # -- species (SpecieP / BeamP) ----------------------------------------------
    def add(self, spec, capacity=None) -> int:
        """Add a species or beam described like ``SpecieP``/``BeamP``."""
        cap = int(capacity or getattr(spec, "capacity", 0) or 1 << 16)
        slot = ctypes.c_int()
        if getattr(spec, "beam", None) is None:
            self._check(self.lib.pcg_add_species(self.h, int(spec.id), spec.name.encode(),
                                                 float(spec.charge), float(spec.mass), cap,
                                                 ctypes.byref(slot)), "pcg_add_species")
        else:
            b = spec.beam
            self._check(self.lib.pcg_add_beam(self.h, int(spec.id), spec.name.encode(),
                                              float(spec.charge), float(spec.mass), cap,
                                              int(b["macro_amount"]), b["start_time"],
                                              b["radius"], b["density"], b["amount"], b["length"],
                                              b["distance"], b["velocity"], ctypes.byref(slot)),
                        "pcg_add_beam")
        self.species.append(spec)
        return slot.value

    def set_particles(self, slot, r, z, vr, vphi, vz, w, append=False):
        arrs = [np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (r, z, vr, vphi, vz, w)]
        if len({a.size for a in arrs}) != 1:
            raise ValueError(f"particle arrays differ in length: {[a.size for a in arrs]}")
        fn = self.lib.pcg_append_species if append else self.lib.pcg_import_species
        self._check(fn(self.h, slot, arrs[0].size, *[_dp(a) for a in arrs]), "pcg_import_species")

    def seed_plasma(self, slot, n, density, temperature_ev, seed=0):
        """Fill a species on the device with a uniform Maxwellian plasma."""
        self._check(self.lib.pcg_seed_plasma(self.h, slot, int(n), float(density),
                                             float(temperature_ev), int(seed)), "pcg_seed_plasma")

    def seed_plasma_cells(self, slot, per_cell, density, t_par_ev, t_perp_ev=None, seed=0):
        """Fill a species on the device with per_cell particles in every cell,
        bi-Maxwellian (t_par along z, t_perp along r and phi)."""
        t_perp_ev = t_par_ev if t_perp_ev is None else t_perp_ev
        self._check(self.lib.pcg_seed_plasma_cells(self.h, slot, int(per_cell), float(density), float(t_par_ev),
                                                   float(t_perp_ev), int(seed)), "pcg_seed_plasma_cells")

    def set_beam_profile(self, slot, profile="gaussian", sigma_z=0.0, macro_per_cell=0.0):
        code = {"rectangle": 0, "gaussian": 1}[profile]
        self._check(self.lib.pcg_set_beam_profile(self.h, slot, code, float(sigma_z),
                                                  float(macro_per_cell)), "pcg_set_beam_profile")

    def enable_timers(self, on=True):
        self._check(self.lib.pcg_enable_timers(self.h, 1 if on else 0), "pcg_enable_timers")

    TIMERS = ["field_e", "field_h", "inject", "particles", "deposit"]

    def kernel_times(self) -> dict:
        """Milliseconds and launches per kernel class since the last call."""
        n = len(self.TIMERS)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_int * n)()
        self._check(self.lib.pcg_kernel_times(self.h, ms, cnt, n), "pcg_kernel_times")
        return {k: (ms[i], cnt[i]) for i, k in enumerate(self.TIMERS)}

    def count(self, slot) -> int:
        n = ctypes.c_size_t()
        self._check(self.lib.pcg_count(self.h, slot, ctypes.byref(n)), "pcg_count")
        return n.value

    def get_particles(self, slot) -> dict:
        n = self.count(slot)
        m = max(n, 1)
        out = {k: np.zeros(m) for k in ("r", "z", "vr", "vphi", "vz", "w")}
        cr = np.zeros(m, dtype=np.int32)
        cz = np.zeros(m, dtype=np.int32)
        got = ctypes.c_size_t()
        self._check(self.lib.pcg_export_species(self.h, slot, m, *[_dp(out[k]) for k in
                                                ("r", "z", "vr", "vphi", "vz", "w")],
                                                cr.ctypes.data_as(_PI32), cz.ctypes.data_as(_PI32),
                                                ctypes.byref(got)), "pcg_export_species")
        out = {k: v[:n] for k, v in out.items()}
        out["cell_r"] = cr[:n].astype(np.int64)
        out["cell_z"] = cz[:n].astype(np.int64)
        return out

    # -- fields (Grid<double> with halo) -------------------------------------------
    def set_field(self, which, arr):
        idx = FIELD[which] if isinstance(which, str) else int(which)
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != tuple(self.grid.shape):
            raise ValueError(f"field {which!r}: shape {a.shape}, the grid is {tuple(self.grid.shape)}")
        self._check(self.lib.pcg_set_field(self.h, idx, _dp(a)), "pcg_set_field")

    def get_field(self, which) -> np.ndarray:
        idx = FIELD[which] if isinstance(which, str) else int(which)
        a = np.zeros(self.grid.shape)
        self._check(self.lib.pcg_export_field(self.h, idx, _dp(a)), "pcg_export_field")
        return a

    def fields(self) -> dict:
        return {n: self.get_field(n) for n in FIELDS}

    def get_field_columns(self, which, c0, c1) -> np.ndarray:
        """Array columns [c0, c1) of a field: (nr+4) x (c1-c0)."""
        idx = FIELD[which] if isinstance(which, str) else int(which)
        a = np.zeros((self.grid.shape[0], max(c1 - c0, 0)))
        self._check(self.lib.pcg_get_field_columns(self.h, idx, int(c0), int(c1), _dp(a)),
                    "pcg_get_field_columns")
        return a

    def set_field_columns(self, which, c0, arr):
        """Array columns [c0, c0 + arr.shape[1]) of a field from arr."""
        idx = FIELD[which] if isinstance(which, str) else int(which)
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.ndim != 2 or a.shape[0] != self.grid.shape[0]:
            raise ValueError(f"field {which!r}: columns of shape {a.shape}, rows must be {self.grid.shape[0]}")
        self._check(self.lib.pcg_set_field_columns(self.h, idx, int(c0), int(c0) + a.shape[1], _dp(a)),
                    "pcg_set_field_columns")

    # -- particles in a band of z (hand-over between domains split along z) --------
    def export_range(self, slot, lo, hi) -> dict:
        """The live particles with lo <= z < hi, in slot order."""
        keys = ("r", "z", "vr", "vphi", "vz", "w")
        n = ctypes.c_size_t()
        null = [None] * 6
        rc = self.lib.pcg_export_species_range(self.h, slot, float(lo), float(hi), 0, *null, ctypes.byref(n))
        if rc == 0:
            return {k: np.zeros(0) for k in keys}
        if rc != -5:  # PCG_ERR_CAPACITY: the count is set
            self._check(rc, "pcg_export_species_range")
        m = n.value
        out = {k: np.zeros(m) for k in keys}
        self._check(self.lib.pcg_export_species_range(self.h, slot, float(lo), float(hi), m,
                                                      *[_dp(out[k]) for k in keys], ctypes.byref(n)),
                    "pcg_export_species_range")
        return {k: v[:n.value] for k, v in out.items()}

    def transfer_range(self, slot, lo, hi, shift, dst, dst_slot, append=True) -> int:
        """Device to device: this domain's live particles with lo <= z < hi,
        z - shift, appended to (or replacing) dst's species dst_slot; returns
        their count."""
        n = ctypes.c_size_t()
        rc = self.lib.pcg_transfer_species_range(self.h, slot, float(lo), float(hi), float(shift), dst.h,
                                                 int(dst_slot), 1 if append else 0, ctypes.byref(n))
        if rc != 0:
            self._raise_pair(rc, "pcg_transfer_species_range", dst)
        return n.value

    def transfer_bands(self, bands) -> list:
        """Several bands at once, one wait for all counts: bands of
        (slot, lo, hi, shift, dst, dst_slot, append), selected from this
        domain's particles as they are now, then imported in order; returns
        each band's count."""
        n = len(bands)
        arr = (Band * max(n, 1))()
        for q, (slot, lo, hi, shift, dst, dst_slot, append) in enumerate(bands):
            arr[q] = Band(int(slot), float(lo), float(hi), float(shift), dst.h.value, int(dst_slot),
                          1 if append else 0)
        counts = (ctypes.c_size_t * max(n, 1))()
        rc = self.lib.pcg_transfer_species_bands(self.h, n, arr, counts)
        if rc != 0:
            dst = bands[0][4] if bands else self
            self._raise_pair(rc, "pcg_transfer_species_bands", dst)
        return [counts[q] for q in range(n)]

    def _raise_pair(self, rc, where, dst):
        """An error of a call on two handles: the last message of each."""
        msgs = [(self.lib.pcg_last_error(d.h) or b"").decode() for d in (self, dst)]
        raise PcgError(rc, where, f"source: {msgs[0]!r}; destination: {msgs[1]!r}")

    def copy_field_columns(self, c0, c1, dst, g0, which=None):
        """Device to device: array columns [c0, c1) of a field (all twelve
        when which is None) into dst's columns from g0."""
        idx = -1 if which is None else (FIELD[which] if isinstance(which, str) else int(which))
        rc = self.lib.pcg_copy_field_columns(self.h, idx, int(c0), int(c1), dst.h, int(g0))
        if rc != 0:
            self._raise_pair(rc, "pcg_copy_field_columns", dst)

    # -- device buffers: torch CUDA tensors on this domain's GPU ------------------------
    @property
    def torch_device(self):
        return f"cuda:{self.device}"

    def _ready(self):
        """Work queued on torch's current stream of this GPU (the tensors'
        producers) is complete."""
        import torch
        torch.cuda.current_stream(self.device).synchronize()

    def export_range_device(self, slot, lo, hi):
        """The live particles with lo <= z < hi as a (6, n) float64 CUDA tensor
        (rows r, z, v_r, v_phi, v_z, w), copied device to device."""
        import torch
        n = ctypes.c_size_t()
        rc = self.lib.pcg_export_species_range(self.h, slot, float(lo), float(hi), 0, *[None] * 6, ctypes.byref(n))
        if rc == 0:
            return torch.zeros((6, 0), dtype=torch.float64, device=self.torch_device)
        if rc != -5:  # PCG_ERR_CAPACITY: the count is set
            self._check(rc, "pcg_export_species_range")
        m = n.value
        t = torch.empty((6, m), dtype=torch.float64, device=self.torch_device)
        self._ready()
        ptrs = [ctypes.cast(t[k].data_ptr(), _PD) for k in range(6)]
        self._check(self.lib.pcg_export_species_range(self.h, slot, float(lo), float(hi), m, *ptrs, ctypes.byref(n)),
                    "pcg_export_species_range")
        return t

    def set_particles_device(self, slot, t, append=False):
        """Particles from a (6, n) float64 CUDA tensor on this GPU."""
        import torch
        t = t.to(dtype=torch.float64).contiguous()
        if t.dim() != 2 or t.shape[0] != 6:
            raise ValueError(f"particles as a (6, n) tensor, not {tuple(t.shape)}")
        self._ready()
        ptrs = [ctypes.cast(t[k].data_ptr(), _PD) for k in range(6)]
        fn = self.lib.pcg_append_species if append else self.lib.pcg_import_species
        self._check(fn(self.h, slot, int(t.shape[1]), *ptrs), "pcg_import_species")

    def get_field_columns_device(self, which, c0, c1):
        """Array columns [c0, c1) of a field as a (nr+4, c1-c0) float64 CUDA tensor."""
        import torch
        idx = FIELD[which] if isinstance(which, str) else int(which)
        t = torch.empty((self.grid.shape[0], c1 - c0), dtype=torch.float64, device=self.torch_device)
        self._ready()
        self._check(self.lib.pcg_get_field_columns(self.h, idx, int(c0), int(c1), ctypes.cast(t.data_ptr(), _PD)),
                    "pcg_get_field_columns")
        return t

    def set_field_columns_device(self, which, c0, t):
        """Array columns [c0, c0 + t.shape[1]) of a field from a float64 CUDA tensor."""
        import torch
        idx = FIELD[which] if isinstance(which, str) else int(which)
        t = t.to(dtype=torch.float64).contiguous()
        self._ready()
        self._check(self.lib.pcg_set_field_columns(self.h, idx, int(c0), int(c0) + int(t.shape[1]),
                                                   ctypes.cast(t.data_ptr(), _PD)), "pcg_set_field_columns")

    def keep_range(self, slot, lo, hi):
        """Remove the live particles outside lo <= z < hi."""
        self._check(self.lib.pcg_keep_species_range(self.h, slot, float(lo), float(hi)),
                    "pcg_keep_species_range")

    def collide(self) -> int:
        """One binary-collision pass (Perez 2012, CollisionsP12::operator());
        returns the number of pair collisions attempted."""
        n = ctypes.c_ulonglong(0)
        self._check(self.lib.pcg_collide(self.h, ctypes.byref(n)), "pcg_collide")
        return int(n.value)

    # -- learned collisions (no reference counterpart) ---------------------------------
    def set_collision_model(self, params, norm):
        """Load the collision MLP's parameters (PCG_MLP_PARAMS floats) and its
        normalisation / training box (PCG_LEARNED_NORM floats)."""
        p = np.ascontiguousarray(params, dtype=np.float32)
        n = np.ascontiguousarray(norm, dtype=np.float32)
        pf = ctypes.POINTER(ctypes.c_float)
        self._check(self.lib.pcg_set_collision_model(self.h, p.ctypes.data_as(pf), n.ctypes.data_as(pf)),
                    "pcg_set_collision_model")

    def tile_sort(self, slot):
        """Sort species `slot` into its tiles now (float layout); returns the
        per-cell counts the sorted tiles hold (nr, nz) and how many
        particles sit outside their tile."""
        counts = np.zeros((self.grid.nr, self.grid.nz), dtype=np.uint32)
        mis = ctypes.c_ulonglong(0)
        self._check(self.lib.pcg_tile_sort(self.h, int(slot), counts.ctypes.data_as(ctypes.POINTER(ctypes.c_uint)),
                                           ctypes.byref(mis)), "pcg_tile_sort")
        return counts, int(mis.value)

    def set_tiling(self, sort_interval=0, target_blocks=0, min_split=0):
        """Tiling of the float step (pcg_set_tiling; 0 keeps a value)."""
        self._check(self.lib.pcg_set_tiling(self.h, int(sort_interval), int(target_blocks), int(min_split)),
                    "pcg_set_tiling")

    MAPS = {"density": 0, "temperature": 1, "energy": 2, "momentum": 3}

    def species_map(self, slot, which) -> np.ndarray:
        """SpecieP::calc_<which> of species `slot` ("density", "temperature",
        "energy" or "momentum"): a grid shaped like the fields, (3, ...) for
        the momentum's r, phi, z."""
        k = self.MAPS[which]
        out = np.zeros((3 if k == 3 else 1,) + self.grid.shape)
        self._check(self.lib.pcg_species_map(self.h, int(slot), k, _dp(out)), "pcg_species_map")
        return out if k == 3 else out[0]

    def set_collision_scheme(self, scheme):
        """Binary operator of collide() and "binary" steps: "p12" (CollisionsP12,
        the default), "ta77s" (CollisionsTA77S with its velocity correction) or
        "sk98" (CollisionsSK98)."""
        code = {"p12": 0, "ta77s": 1, "sk98": 2}[scheme]
        self._check(self.lib.pcg_set_collision_scheme(self.h, code), "pcg_set_collision_scheme")

    def set_external_fields(self, electric="none", e_params=(), magnetic="none", m_params=()):
        """External E and H fields (ExternalFields, externalFields.cpp), by the
        formfactor names of PiCoPiC.json's external_fields section; params[0]
        is the amplitude.  See pcg_set_external_fields for what applies in
        each quirk mode."""
        ep = np.ascontiguousarray(e_params, dtype=np.float64).reshape(-1)
        mp = np.ascontiguousarray(m_params, dtype=np.float64).reshape(-1)
        self._check(self.lib.pcg_set_external_fields(self.h, electric.encode(), _dp(ep) if ep.size else None,
                                                     ep.size, magnetic.encode(), _dp(mp) if mp.size else None,
                                                     mp.size), "pcg_set_external_fields")

    def set_collision_crowding(self, threshold):
        """Cells of more than `threshold` particles run their collisions on a
        warp each (pcg_set_collision_crowding; the result does not change)."""
        self._check(self.lib.pcg_set_collision_crowding(self.h, int(threshold)), "pcg_set_collision_crowding")

    def set_collisions(self, mode):
        """Collisions inside step(): "none", "binary" or "learned" (one pass opens every step)."""
        code = {"none": 0, "binary": 1, "learned": 2}[mode]
        self._check(self.lib.pcg_set_collisions(self.h, code), "pcg_set_collisions")

    def collide_learned(self):
        """One learned collision step; returns (learned cells, binary fallback cells)."""
        a, b = ctypes.c_ulonglong(0), ctypes.c_ulonglong(0)
        self._check(self.lib.pcg_collide_learned(self.h, ctypes.byref(a), ctypes.byref(b)), "pcg_collide_learned")
        return int(a.value), int(b.value)

    def collide_expectation(self) -> np.ndarray:
        """One binary pass; returns (nr*nz, 12): per cell and list the sum over its
        collisions of each collision's mean change of sum w v (3), sum w v^2 (3)."""
        m = np.zeros((self.grid.nr * self.grid.nz, 12))
        self._check(self.lib.pcg_collide_expectation(self.h, _dp(m)), "pcg_collide_expectation")
        return m

    def cell_moments(self) -> np.ndarray:
        """(nr*nz, 16): per cell, electron list then ion list: N, sum w, sum w v (3), sum w v^2 (3)."""
        m = np.zeros((self.grid.nr * self.grid.nz, 16))
        self._check(self.lib.pcg_cell_moments(self.h, _dp(m)), "pcg_cell_moments")
        return m

    def cell_features(self):
        """Raw features (nr*nz, 13; NaN where a cell takes no collisions) and the scale S."""
        cells = self.grid.nr * self.grid.nz
        x = np.zeros((cells, 13), dtype=np.float32)
        s = np.zeros(cells)
        self._check(self.lib.pcg_cell_features(self.h, x.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), _dp(s)),
                    "pcg_cell_features")
        return x, s

    # -- acceptance diagnostics of the deposit (no reference counterpart) ------------
    def node_charge(self) -> np.ndarray:
        """Node charges (C) in the shape the Villasenor-Buneman deposit conserves."""
        a = np.zeros(self.grid.shape)
        self._check(self.lib.pcg_node_charge(self.h, _dp(a)), "pcg_node_charge")
        return a

    def divergence(self, which: str) -> np.ndarray:
        """Flux divergence of J ("j") or E ("e") over the Yee face areas (A m^2 or V m)."""
        a = np.zeros(self.grid.shape)
        self._check(self.lib.pcg_divergence(self.h, FIELD["j_r" if which == "j" else "e_r"], _dp(a)),
                    "pcg_divergence")
        return a

    def continuity_step(self) -> np.ndarray:
        """Take one step and return the charge continuity residual of every
        node, Q(n+1) - Q(n) + dt div J, relative to the largest |Q(n+1)|
        (real nodes only; beam injection and runaway removal add or drop
        charge without a current and show up here)."""
        q0 = self.node_charge()
        self.step(1)
        q1 = self.node_charge()
        r = q1 - q0 + self.grid.dt * self.divergence("j")
        return r[2:-2, 2:-2] / max(np.abs(q1).max(), 1e-300)

    # -- the Domain façade (src/domain.cpp:86-204) -----------------------------------
    def stage(self, name) -> int:
        idx = STAGE[name] if isinstance(name, str) else int(name)
        return self._check(self.lib.pcg_stage(self.h, idx), "pcg_stage")

    def manage_beam(self): return self.stage("inject")
    def weight_field_e(self): return self.stage("field_e")
    def weight_field_h(self): return self.stage("field_h")
    def push_particles(self): return self.stage("push")
    def dump_particle_positions_to_old(self): return self.stage("dump_old")
    def update_particles_coords(self): return self.stage("move")
    def particles_back_position_to_rz(self): return self.stage("pos_rz")
    def reflect(self): return self.stage("reflect")
    def particles_back_velocity_to_rz(self): return self.stage("vel_rz")
    def bind_cell_numbers(self): return self.stage("bind")
    def particles_runaway_collector(self): return self.stage("collect")
    def reset_current(self): return self.stage("reset_current")
    def weight_current(self): return self.stage("current")

    def step(self, n: int = 1) -> int:
        """``n`` full steps (inject, E, H, advance particles, current) on the device."""
        self._check(self.lib.pcg_step(self.h, int(n)), "pcg_step")
        return 0

    def step_status(self):
        """Check the status of the steps before the previous call without
        waiting for the later ones (pcg_step_status); raises on an error."""
        self._check(self.lib.pcg_step_status(self.h), "pcg_step_status")

    def synchronize(self):
        self._check(self.lib.pcg_synchronize(self.h), "pcg_synchronize")

    def diag(self) -> Diagnostics:
        d = Diagnostics()
        self._check(self.lib.pcg_diag(self.h, ctypes.byref(d)), "pcg_diag")
        return d

    @property
    def time(self) -> float:
        return self.diag().time

    @property
    def removed(self) -> int:
        return int(self.diag().removed)

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.lib.pcg_get_stream(self.h, ctypes.byref(s)), "pcg_get_stream")
        return s.value or 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.pcg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
