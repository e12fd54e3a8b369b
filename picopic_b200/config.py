"""PiCoPiC.json for this library: the reference's configuration file
(src/cfg.cpp, schema in doc/PiCoPiC.json.md) read into a Domain, and a run
that writes its probes.

    cfg = config.load("PiCoPiC.json")
    d, slots = config.build_domain(cfg, precision="f32")
    config.run(cfg, d, slots, out_dir="data")      # probes as .npy under data/

What the reference fixes at compile time (pusher, current scheme,
collisions) are arguments here, as on the C ABI.  Differences from the
reference, by design:

* one domain: `geometry.domains_amount` is read and ignored (the reference
  splits the grid over OpenMP domains; here one GPU takes it whole);
* plasma species start uniform in the volume with Maxwellian velocities
  (pcg_seed_plasma) rather than the reference's initialisers
  (specieP.cpp:127-384), which place particles with weight proportional to
  r and scale |v| by a uniform draw;
* probes are written as .npy arrays, one per probe, at the path the
  reference gives its HDF5 dataset (cfg.cpp:204-272:
  <component>/[<specie>/]<shape>/<r0>-<r1>_<z0>-<z1>), frames stacked on
  the first axis, since no HDF5 library is available;
* external fields (`external_fields`) are read and ignored, as the
  reference's default build ignores them (configure.ac:84-85, 214-222:
  a development-only switch); with use_external_fields=True (the
  --external-fields switch) they are applied as the ENABLE_EXTERNAL_FIELDS
  build applies them (Domain.set_external_fields, pcg_set_external_fields).
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os

import numpy as np

from .domain import Domain, Geometry


@dataclasses.dataclass
class Probe:
    component: str     # "E/r", "H/phi", "J/z", "density", "temperature", "energy", "momentum/r", ...
    specie: str        # for the species components, else "unknown"
    shape: str         # "rec", "col", "row" or "dot"
    dims: tuple        # (r0, z0, r1, z1) in cells
    schedule: int      # every `schedule` steps
    path: str          # <component>/[<specie>/]<shape>/...


@dataclasses.dataclass
class RunConfig:
    geometry: Geometry
    t_end: float
    macro_amount: float
    beam_macro_ratio: float
    species: list      # dicts: name, charge, mass, density, temperature, macro_amount
    beams: list        # dicts: name ("beam_" + name), charge, mass, velocity, start_time, amount,
                       # distance, length, radius, density, profile, macro_amount
    probes: list
    data_root: str
    external_fields: dict
    raw: dict = dataclasses.field(default_factory=dict)  # the configuration as read, for the output metadata

    @property
    def steps(self) -> int:
        """Steps from start to end (the reference loops while current < end)."""
        g = self.geometry
        return int(np.ceil((self.t_end - g.t_start) / g.dt - 1e-9))


SPECIES_COMPONENTS = ("temperature", "energy", "momentum/r", "momentum/phi", "momentum/z", "density")


def _probe(o, nr, nz) -> Probe:
    """Cfg::init_probes (cfg.cpp:204-290)."""
    comp = o["component"]
    specie = o.get("specie", "unknown")
    shape = o["shape"]
    path = comp + "/"
    if comp in SPECIES_COMPONENTS:
        path += specie + "/"
    if shape == "rec":
        d = (int(o["start"]["r"]), int(o["start"]["z"]), int(o["end"]["r"]), int(o["end"]["z"]))
        path += f"rec/{d[0]}-{d[2]}_{d[1]}-{d[3]}"
    elif shape == "col":
        d = (0, 0, 0, int(o["z"]))
        path += f"col/{d[3]}"
    elif shape == "row":
        d = (0, 0, int(o["r"]), 0)
        path += f"row/{d[2]}"
    elif shape == "dot":
        d = (0, 0, int(o["r"]), int(o["z"]))
        path += f"dot/{d[2]}_{d[3]}"
    else:
        raise ValueError(f"unknown probe shape {shape!r}")
    if d[0] > d[2] or d[1] > d[3]:
        raise ValueError(f"incorrect probe {comp}/{shape} shape {d}")
    if d[2] > nr or d[3] > nz:
        raise ValueError(f"probe {comp}/{shape} {d} is out of the {nr} x {nz} grid")
    return Probe(comp, specie, shape, d, int(o["schedule"]), path)


def weight_macro_amount(nr, nz, dr, dz, n_species, beams, macro_amount, ratio):
    """Cfg::weight_macro_amount (cfg.cpp:489-571): every species gets
    cells x norm macroparticles and every beam (radius/dr) x
    (length x amount/dz) x norm x ratio, norm making the total macro_amount."""
    norm_sum = nr * nz * n_species
    for b in beams:
        norm_sum += (b["radius"] / dr) * (b["length"] * b["amount"] / dz) * ratio
    norm = macro_amount / norm_sum
    plasma = int(nr * nz * norm)
    beam = [int((b["radius"] / dr) * (b["length"] * b["amount"] / dz) * norm * ratio) for b in beams]
    return plasma, beam


def load(src) -> RunConfig:
    """A PiCoPiC.json file (path) or its parsed dict."""
    if isinstance(src, (str, os.PathLike)):
        with open(src) as f:
            src = json.load(f)
    g = src["geometry"]
    nr, nz = int(g["grid"]["radius"]), int(g["grid"]["longitude"])
    pml = g.get("pml", {})
    t = src["time"]
    geom = Geometry(nr, nz, float(g["size"]["radius"]), float(g["size"]["longitude"]), float(t["step"]),
                    t_start=float(t["start"]),
                    pml_size=(0, int(np.floor(pml.get("left_wall", 0) * nz)),
                              int(np.floor(pml.get("outer_wall", 0) * nr)),
                              int(np.floor(pml.get("right_wall", 0) * nz))),
                    pml_sigma=(float(pml.get("sigma_1", 0.0)), float(pml.get("sigma_2", 0.0))))
    species = []
    for o in src.get("particles", []):
        if any(s["name"] == o["name"] for s in species):
            raise ValueError(f"particle species name {o['name']!r} repeats")
        dens = o["density"]
        if isinstance(dens, dict):  # the documented left/right form; profiles are not supported
            dens = dens["left"]
        species.append(dict(name=o["name"], charge=int(o["charge"]), mass=int(o["mass"]),
                            density=float(dens), temperature=float(o["temperature"])))
    beams = []
    for o in src.get("beams", []):
        b = o["bunch"]
        name = "beam_" + o["name"]
        if any(x["name"] == name for x in beams):
            raise ValueError(f"beam name {o['name']!r} repeats")
        prof = b.get("profile", {})
        beams.append(dict(name=name, charge=int(o["charge"]), mass=int(o["mass"]),
                          start_time=float(o["start_time"]), velocity=float(o["velocity"]),
                          amount=int(b["amount"]), distance=float(b["distance"]), length=float(b["length"]),
                          radius=float(b["radius"]), density=float(b["density"]),
                          profile=(prof.get("radial", "rectangle"), prof.get("longitudinal", "rectangle"))))
    macro = float(src["macro_amount"])
    ratio = float(src.get("beam_plasma_macro_size_ratio", 1))
    plasma_n, beam_n = weight_macro_amount(nr, nz, geom.dr, geom.dz, len(species), beams, macro, ratio)
    for s in species:
        s["macro_amount"] = plasma_n
    for b, n in zip(beams, beam_n):
        b["macro_amount"] = n
    data = src.get("data", {})
    probes = [_probe(o, nr, nz) for o in data.get("probes", [])]
    ext = src.get("external_fields", {})
    return RunConfig(geom, float(t["end"]), macro, ratio, species, beams, probes,
                     data.get("data_root", "./"), ext, raw=src)


class _Spec:
    def __init__(self, name, charge, mass, id, beam=None):
        self.name, self.charge, self.mass, self.id, self.beam = name, charge, mass, id, beam


def _id(name: str) -> int:
    """A species id from its name (stable, 16 bits; the reference hashes the
    name with a salt, algo::common::hash_from_string)."""
    h = 2166136261
    for ch in name.encode():
        h = ((h ^ ch) * 16777619) & 0xFFFFFFFF
    return h & 0xFFFF


def build_domain(cfg: RunConfig, pusher="borisrel", current="vb", precision="f32", quirks="reference",
                 seed=0, device=0, use_external_fields=False, plasma="maxwellian"):
    """A Domain with the configuration's species (seeded) and beams.  Returns
    (domain, {name: slot}).

    plasma: "maxwellian" seeds each species on the device (r = R sqrt(U),
    equal weights, a Maxwellian at the configured temperature);
    "reference" builds on the host the particles the reference's own
    Domain::distribute makes (picopic_b200.initial: flat placement and
    weights bit for bit, its thermal velocity distribution)."""
    if plasma not in ("maxwellian", "reference"):
        raise ValueError(f"plasma initialiser {plasma!r}: 'maxwellian' or 'reference'")
    d = Domain(cfg.geometry, pusher=pusher, current=current, precision=precision, quirks=quirks, seed=seed,
               device=device)
    if use_external_fields:  # the reference's ENABLE_EXTERNAL_FIELDS build (cfg.cpp:454-487)
        ef = cfg.external_fields
        e, m = ef.get("electric", {}), ef.get("magnetic", {})
        d.set_external_fields(e.get("formfactor", "none"), e.get("params", []),
                              m.get("formfactor", "none"), m.get("params", []))
    slots = {}
    for s in cfg.species:
        slots[s["name"]] = d.add(_Spec(s["name"], s["charge"], s["mass"], _id(s["name"])),
                                 capacity=s["macro_amount"] + 16)
    for b in cfg.beams:
        if b["profile"] != ("rectangle", "rectangle"):
            raise NotImplementedError(f"beam profile {b['profile']}: the reference parses it but injects "
                                      "a rectangular bunch (beamP.cpp:100-145); use pcg_set_beam_profile")
        beam = dict(macro_amount=b["macro_amount"], start_time=b["start_time"], radius=b["radius"],
                    density=b["density"], amount=b["amount"], length=b["length"], distance=b["distance"],
                    velocity=b["velocity"])
        slots[b["name"]] = d.add(_Spec(b["name"], b["charge"], b["mass"], _id(b["name"]), beam=beam),
                                 capacity=b["macro_amount"] + 4096)
    g = cfg.geometry
    for k, s in enumerate(cfg.species):
        if plasma == "reference":
            from . import initial
            d.set_particles(slots[s["name"]], *initial.reference_plasma(
                s["macro_amount"], g.nr, g.nz, g.dr, g.dz, s["density"], s["temperature"], s["mass"],
                seed=seed * 1000 + k))
        else:
            d.seed_plasma(slots[s["name"]], s["macro_amount"], s["density"], s["temperature"], seed + k)
    return d, slots


def _frame(d, slots, p: Probe):
    """The probed grid of one frame: nodes [r0, r1) x [z0, z1) of the
    component (a column, row or dot for the other shapes)."""
    comp = p.component
    if comp.split("/")[0] in ("E", "H", "J"):
        field, axis = comp.split("/")
        # H probes read field_h_at_et, as OutController does (outController.cpp:151-297)
        prefix = {"E": "e", "H": "hat", "J": "j"}[field]
        grid = d.get_field(f"{prefix}_{axis}")
    else:
        slot = slots[p.specie]
        base = comp.split("/")[0]
        m = d.species_map(slot, base)
        grid = m[{"r": 0, "phi": 1, "z": 2}[comp.split("/")[1]]] if base == "momentum" else m
    g = grid[2:-2, 2:-2]  # interior nodes, index (r, z)
    r0, z0, r1, z1 = p.dims
    if p.shape == "rec":
        return g[r0:r1, z0:z1]
    if p.shape == "col":
        return g[:, z1]
    if p.shape == "row":
        return g[r1, :]
    return g[r1, z1]


def run(cfg: RunConfig, d, slots, steps=None, out_dir=None, log=print, attrs=None):
    """Step the domain `steps` times (default: to the configured end time),
    recording every probe on its schedule; writes <out_dir>/<probe path>.npy
    (frames x probe shape) with the layout of the reference's data.h5 in
    <out_dir>/data.h5.json (h5layout: the root attributes `attrs`, by
    default those of the relativistic Boris / VB float build) and returns
    {path: array}.

    The schedule is the reference's: its main loop (PiCoPiC.cpp:326-347)
    runs a step and then the writers while the clock still reads the step's
    start time t, and a probe writes when ceil(t / dt) is a multiple of its
    schedule (outController.cpp:341-351), t accumulated by repeated
    additions of dt.  So frame j is the state after schedule * j + 1 steps."""
    n = cfg.steps if steps is None else int(steps)
    g = cfg.geometry
    frames = {p.path: [] for p in cfg.probes}
    t = g.t_start
    for _ in range(n):
        d.step(1)
        ts = int(np.ceil(t / g.dt))
        for p in cfg.probes:
            if ts % p.schedule == 0:
                frames[p.path].append(np.array(_frame(d, slots, p)))
        t += g.dt
    d.synchronize()
    out = {path: np.stack(f) if f else np.zeros((0,)) for path, f in frames.items()}
    if out_dir:
        from . import h5layout
        h5layout.write_tree(out_dir, out, attrs if attrs is not None else h5layout.root_attributes(cfg.raw))
        log(f"{n} steps, {len(out)} probes written under {out_dir}")
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description="run a PiCoPiC.json configuration on the GPU")
    ap.add_argument("config")
    ap.add_argument("--steps", type=int, default=None, help="default: to the configured end time")
    ap.add_argument("--out", default=None, help="default: the configuration's data_root")
    ap.add_argument("--pusher", default="borisrel", choices=["boris", "borisadaptive", "borisrel", "vay", "hc"])
    ap.add_argument("--current", default="vb", choices=["vb", "zigzag"])
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--quirks", default="reference", choices=["reference", "fixed"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--plasma", default="maxwellian", choices=["maxwellian", "reference"],
                    help="plasma initial condition: device Maxwellian, or the reference's own")
    ap.add_argument("--external-fields", action="store_true",
                    help="apply the configuration's external_fields (the reference's ENABLE_EXTERNAL_FIELDS build)")
    a = ap.parse_args(argv)
    cfg = load(a.config)
    d, slots = build_domain(cfg, a.pusher, a.current, a.precision, a.quirks, a.seed,
                            use_external_fields=a.external_fields, plasma=a.plasma)
    from . import h5layout
    attrs = h5layout.root_attributes(cfg.raw, a.pusher, a.current, a.precision, a.quirks, a.plasma)
    run(cfg, d, slots, a.steps, a.out or cfg.data_root, attrs=attrs)


if __name__ == "__main__":
    main()
