"""ctypes harness over the CPU oracle and the compiled reference.

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import this module.  The product
(``picopic_b200``) never does.

Both back ends expose the same calls (``*_create``, ``*_add_species``,
``*_set_particles``, ``*_get_particles``, ``*_set_field``,
``*_get_field``, ``*_stage``, ``*_step``):

* :class:`OracleSim` loads ``oracle/liboracle.so``, the plain-C restatement
  in ``oracle/pic_oracle.c``;
* :class:`RefSim` loads ``oracle/_ref/libpicopic_ref_<pusher>_<current>.so``,
  the reference's own hot-path sources compiled by ``oracle/Makefile.ref``
  with the driver ``oracle/ref_driver.cpp``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF_ROOT_FILE = os.path.join(HERE, "_ref", "reference_root")
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

PUSHERS = {"boris": 0, "borisadaptive": 1, "borisrel": 2, "vay": 3, "hc": 4}
CURRENTS = {"vb": 0, "zigzag": 1}
QUIRKS = {"reference": 0, "fixed": 1}

# Stage numbers: the Domain methods in SMB / main-loop order.
STAGES = ["inject", "field_e", "field_h", "push", "dump_old", "move", "pos_rz", "reflect",
          "vel_rz", "bind", "collect", "reset_current", "current", "advance_time"]
STAGE = {name: i for i, name in enumerate(STAGES)}

# Field slots: E(r,phi,z), H, H_at_et, J, sigma.
FIELDS = ["e_r", "e_phi", "e_z", "h_r", "h_phi", "h_z", "hat_r", "hat_phi", "hat_z",
          "j_r", "j_phi", "j_z"]
FIELD = {name: i for i, name in enumerate(FIELDS)}

_D = ctypes.c_double
_PD = ctypes.POINTER(ctypes.c_double)
_PLL = ctypes.POINTER(ctypes.c_longlong)
_PI = ctypes.POINTER(ctypes.c_int)


def build_oracle(force: bool = False) -> str:
    """Compile oracle/pic_oracle.c into oracle/liboracle.so with gcc."""
    src = os.path.join(HERE, "pic_oracle.c")
    if force or not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-std=c11", "-O2", "-fPIC", "-ffp-contract=off", "-shared",
                               "-o", ORACLE_SO, src, "-lm"])
    return ORACLE_SO


def reference_root() -> str | None:
    """The reference checkout: $PICOPIC_REFERENCE, else the checkout the last
    build_reference compiled (recorded in oracle/_ref/reference_root); None
    when neither names a directory with the reference's sources."""
    root = os.environ.get("PICOPIC_REFERENCE")
    if not root and os.path.exists(REF_ROOT_FILE):
        with open(REF_ROOT_FILE) as f:
            root = f.read().strip()
    return root if root and os.path.isdir(os.path.join(root, "src")) else None


def build_reference(root: str | None = None, jobs: int = 8) -> bool:
    """Compile the reference hot path (oracle/Makefile.ref) from the checkout
    `root` (default: reference_root()); False when there is none."""
    root = root or reference_root()
    if not root or not os.path.isdir(os.path.join(root, "src")):
        return False
    subprocess.check_call(["make", "-s", "-f", os.path.join("oracle", "Makefile.ref"),
                           f"REF={root}", f"-j{jobs}"], cwd=REPO)
    os.makedirs(REF_DIR, exist_ok=True)
    with open(REF_ROOT_FILE, "w") as f:
        f.write(os.path.abspath(root) + "\n")
    return True


def reference_available(pusher: str = "borisrel", current: str = "vb", perf: bool = False,
                        extf: bool = False) -> bool:
    return os.path.exists(_ref_path(pusher, current, perf, extf))


def _ref_path(pusher: str, current: str, perf: bool = False, extf: bool = False) -> str:
    tag = "perf_" if perf else "extf_" if extf else ""
    return os.path.join(REF_DIR, f"libpicopic_ref_{tag}{pusher}_{current}.so")


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_PD)


@dataclass
class SpeciesSpec:
    """One particle species (SpecieP) or beam (BeamP) as the reference configures it."""
    name: str
    charge: float          # electron charges
    mass: float            # electron masses
    id: int = 0
    beam: dict | None = None   # BeamP parameters: macro_amount, start_time, radius, density,
                               # amount, length, distance, velocity


@dataclass
class GridSpec:
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


class _Sim:
    prefix = ""

    def _bind(self, lib):
        p = self.prefix
        f = getattr(lib, p + "add_species")
        f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, _D, _D]
        f.restype = ctypes.c_int
        f = getattr(lib, p + "add_beam")
        f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, _D, _D, ctypes.c_uint,
                      _D, _D, _D, _D, _D, _D, _D]
        f.restype = ctypes.c_int
        f = getattr(lib, p + "set_particles")
        f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t] + [_PD] * 6
        f.restype = ctypes.c_int
        f = getattr(lib, p + "count")
        f.argtypes = [ctypes.c_void_p, ctypes.c_int]
        f.restype = ctypes.c_long
        f = getattr(lib, p + "get_particles")
        f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t] + [_PD] * 8 + [_PLL] * 2
        f.restype = ctypes.c_int
        for name in ("set_field", "get_field"):
            f = getattr(lib, p + name)
            f.argtypes = [ctypes.c_void_p, ctypes.c_int, _PD]
            f.restype = ctypes.c_int
        for name in ("stage", "step"):
            f = getattr(lib, p + name)
            f.argtypes = [ctypes.c_void_p, ctypes.c_int]
            f.restype = ctypes.c_int
        f = getattr(lib, p + "species_map")
        f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _PD]
        f.restype = ctypes.c_int
        f = getattr(lib, p + "time")
        f.argtypes = [ctypes.c_void_p]
        f.restype = _D
        f = getattr(lib, p + "removed")
        f.argtypes = [ctypes.c_void_p]
        f.restype = ctypes.c_long
        f = getattr(lib, p + "destroy")
        f.argtypes = [ctypes.c_void_p]
        f.restype = None

    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def add(self, sp: SpeciesSpec) -> int:
        name = sp.name.encode()
        if sp.beam is None:
            return self._fn("add_species")(self.h, sp.id, name, sp.charge, sp.mass)
        b = sp.beam
        return self._fn("add_beam")(self.h, sp.id, name, sp.charge, sp.mass,
                                    int(b["macro_amount"]), b["start_time"], b["radius"],
                                    b["density"], b["amount"], b["length"], b["distance"],
                                    b["velocity"])

    def set_particles(self, sid: int, r, z, vr, vphi, vz, w):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (r, z, vr, vphi, vz, w)]
        n = arrs[0].size
        rc = self._fn("set_particles")(self.h, sid, n, *[_dp(a) for a in arrs])
        assert rc == 0, rc

    def count(self, sid: int) -> int:
        return int(self._fn("count")(self.h, sid))

    def get_particles(self, sid: int) -> dict:
        n = self.count(sid)
        out = {k: np.zeros(max(n, 1)) for k in ("r", "z", "vr", "vphi", "vz", "w", "r_old", "z_old")}
        cr = np.zeros(max(n, 1), dtype=np.int64)
        cz = np.zeros(max(n, 1), dtype=np.int64)
        rc = self._fn("get_particles")(self.h, sid, max(n, 1), *[_dp(out[k]) for k in
                                       ("r", "z", "vr", "vphi", "vz", "w", "r_old", "z_old")],
                                       cr.ctypes.data_as(_PLL), cz.ctypes.data_as(_PLL))
        assert rc == 0, rc
        out = {k: v[:n] for k, v in out.items()}
        out["cell_r"] = cr[:n]
        out["cell_z"] = cz[:n]
        return out

    def set_field(self, which, arr: np.ndarray):
        idx = FIELD[which] if isinstance(which, str) else which
        a = np.ascontiguousarray(arr, dtype=np.float64)
        assert a.shape == self.grid.shape
        assert self._fn("set_field")(self.h, idx, _dp(a)) == 0

    def get_field(self, which) -> np.ndarray:
        idx = FIELD[which] if isinstance(which, str) else which
        a = np.zeros(self.grid.shape)
        assert self._fn("get_field")(self.h, idx, _dp(a)) == 0
        return a

    def fields(self) -> dict:
        return {name: self.get_field(name) for name in FIELDS}

    MAPS = {"density": 0, "temperature": 1, "energy": 2, "momentum": 3}

    def species_map(self, sid: int, which: str) -> np.ndarray:
        """SpecieP::calc_<which> of species sid (specieP.cpp:665-839): a
        (nr+4, nz+4) grid, or (3, nr+4, nz+4) for "momentum"."""
        k = self.MAPS[which]
        out = np.zeros((3 if k == 3 else 1,) + self.grid.shape)
        rc = self._fn("species_map")(self.h, sid, k, _dp(out))
        assert rc == 0, f"species_map rc {rc}"
        return out if k == 3 else out[0]

    def set_external_fields(self, electric="none", e_params=(), magnetic="none", m_params=()) -> int:
        """ExternalFields' formfactors and params (externalFields.cpp); the
        reference library must be the ENABLE_EXTERNAL_FIELDS build (extf)."""
        f = self._fn("set_external_fields")
        f.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _PD, ctypes.c_int, ctypes.c_char_p, _PD, ctypes.c_int]
        f.restype = ctypes.c_int
        ep = np.ascontiguousarray(e_params, dtype=np.float64).reshape(-1)
        mp = np.ascontiguousarray(m_params, dtype=np.float64).reshape(-1)
        return int(f(self.h, electric.encode(), _dp(ep) if ep.size else None, ep.size,
                     magnetic.encode(), _dp(mp) if mp.size else None, mp.size))

    def stage(self, name) -> int:
        idx = STAGE[name] if isinstance(name, str) else name
        return self._fn("stage")(self.h, idx)

    def step(self, n: int = 1) -> int:
        return self._fn("step")(self.h, n)

    @property
    def time(self) -> float:
        return float(self._fn("time")(self.h))

    @property
    def removed(self) -> int:
        return int(self._fn("removed")(self.h))

    def close(self):
        if getattr(self, "h", None):
            self._fn("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _make_arrays(grid: GridSpec):
    pml = (ctypes.c_int * 4)(*[int(x) for x in grid.pml_size])
    sig = (ctypes.c_double * 2)(*[float(x) for x in grid.pml_sigma])
    return pml, sig


class OracleSim(_Sim):
    """The plain-C restatement (oracle/pic_oracle.c)."""
    prefix = "orc_"
    _lib = None

    def __init__(self, grid: GridSpec, pusher="borisrel", current="vb", quirks="reference"):
        if OracleSim._lib is None:
            lib = ctypes.CDLL(build_oracle())
            lib.orc_create.restype = ctypes.c_void_p
            lib.orc_create.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _PI, _PD,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int]
            lib.orc_set_rng.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64]
            lib.orc_error_count.argtypes = [ctypes.c_void_p]
            lib.orc_error_count.restype = ctypes.c_long
            lib.orc_philox_uniform.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64,
                                               ctypes.c_uint32, ctypes.c_int]
            lib.orc_philox_uniform.restype = _D
            lib.orc_philox4x32_10.argtypes = [ctypes.POINTER(ctypes.c_uint32)] * 3
            lib.orc_collide.argtypes = [ctypes.c_void_p, ctypes.c_int]
            lib.orc_collide.restype = ctypes.c_long
            lib.orc_collide_ta77s.argtypes = [ctypes.c_void_p, ctypes.c_int]
            lib.orc_collide_ta77s.restype = ctypes.c_long
            lib.orc_collide_sk98.argtypes = [ctypes.c_void_p, ctypes.c_int]
            lib.orc_collide_sk98.restype = ctypes.c_long
            self._bind(lib)
            OracleSim._lib = lib
        self.lib = OracleSim._lib
        self.grid = grid
        pml, sig = _make_arrays(grid)
        h = self.lib.orc_create(grid.nr, grid.nz, grid.radius, grid.longitude, grid.dt,
                                grid.t_start, pml, sig, PUSHERS[pusher], CURRENTS[current],
                                QUIRKS[quirks])
        assert h, "orc_create failed"
        self.h = ctypes.c_void_p(h)

    def set_rng(self, kind: str, seed: int):
        self.lib.orc_set_rng(self.h, {"mt19937": 0, "philox": 1}[kind], seed)

    def collide(self, shuffle: bool = False, scheme: str = "p12") -> int:
        """One binary-collision pass (scheme "p12": Perez 2012, "ta77s":
        Takizuka-Abe with the weighted correction, "sk98": the relativistic
        CM-frame scheme); returns the pair calls."""
        f = {"p12": self.lib.orc_collide, "ta77s": self.lib.orc_collide_ta77s,
             "sk98": self.lib.orc_collide_sk98}[scheme]
        return int(f(self.h, int(shuffle)))

    @property
    def errors(self) -> int:
        return int(self.lib.orc_error_count(self.h))


class RefSim(_Sim):
    """The reference's own sources compiled with oracle/Makefile.ref."""
    prefix = "ref_"
    _libs: dict = {}

    def __init__(self, grid: GridSpec, pusher="borisrel", current="vb", perf=False, extf=False):
        path = _ref_path(pusher, current, perf, extf)
        if path not in RefSim._libs:
            lib = ctypes.CDLL(path)
            lib.ref_create.restype = ctypes.c_void_p
            lib.ref_create.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _PI, _PD]
            lib.ref_seed.argtypes = [ctypes.c_uint]
            lib.ref_error_count.restype = ctypes.c_long
            lib.ref_collide.argtypes = [ctypes.c_void_p]
            lib.ref_collide.restype = ctypes.c_long
            lib.ref_collide_ta77s.argtypes = [ctypes.c_void_p]
            lib.ref_collide_ta77s.restype = ctypes.c_long
            lib.ref_collide_sk98.argtypes = [ctypes.c_void_p]
            lib.ref_collide_sk98.restype = ctypes.c_long
            lib.ref_add_plasma.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, _D, _D,
                                           ctypes.c_uint, _D, _D]
            lib.ref_distribute.argtypes = [ctypes.c_void_p]
            self._bind(lib)
            RefSim._libs[path] = lib
        self.lib = RefSim._libs[path]
        self.grid = grid
        pml, sig = _make_arrays(grid)
        h = self.lib.ref_create(grid.nr, grid.nz, grid.radius, grid.longitude, grid.dt,
                                grid.t_start, pml, sig)
        assert h, "ref_create failed"
        self.h = ctypes.c_void_p(h)

    def seed(self, s: int):
        """Seed the reference's global std::mt19937 (rand.cpp:25)."""
        self.lib.ref_seed(s)

    def add_plasma(self, sp: SpeciesSpec, macro_amount: int, density: float, temperature: float) -> int:
        """A species the reference fills itself at distribute()."""
        return self.lib.ref_add_plasma(self.h, sp.id, sp.name.encode(), sp.charge, sp.mass,
                                       int(macro_amount), density, temperature)

    def distribute(self):
        """Domain::distribute (domain.cpp:86-94): the reference's own flat
        placement, weights and thermal velocities for every plasma species."""
        rc = self.lib.ref_distribute(self.h)
        assert rc == 0, rc

    def collide(self, scheme: str = "p12") -> int:
        """One CollisionsP12 pass without its time-seeded shuffle (returns ncol),
        or one CollisionsTA77S / CollisionsSK98 pass likewise (returns 0: they
        keep no count)."""
        if scheme == "ta77s":
            return int(self.lib.ref_collide_ta77s(self.h))
        if scheme == "sk98":
            return int(self.lib.ref_collide_sk98(self.h))
        return int(self.lib.ref_collide(self.h))

    @property
    def errors(self) -> int:
        return int(self.lib.ref_error_count())


SMB_LIB = os.path.join(REF_DIR, "libpicopic_ref_smb_borisrel_vb.so")


def smb_available() -> bool:
    return os.path.exists(SMB_LIB)


class SmbSim:
    """The reference's own scheduler (src/SMB.cpp, unmodified, release flags,
    OpenMP over its domains) driven by oracle/ref_smb.cpp: relativistic
    Boris and Villasenor-Buneman.  Species and beams are added before
    build(); distribute() places every domain's plasma with the reference's
    own initialiser."""
    _lib = None
    FIELDS = ["e_r", "e_phi", "e_z", "hat_r", "hat_phi", "hat_z", "j_r", "j_phi", "j_z"]

    def __init__(self, grid: GridSpec, r_domains: int, z_domains: int):
        if SmbSim._lib is None:
            lib = ctypes.CDLL(SMB_LIB)
            lib.smb_new.restype = ctypes.c_void_p
            lib.smb_new.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, _D, ctypes.c_int, ctypes.c_int, _PI, _PD]
            lib.smb_add_species.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_char_p, ctypes.c_int,
                                            ctypes.c_uint, _D, _D, _D]
            lib.smb_add_beam.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_char_p, ctypes.c_int,
                                         ctypes.c_uint, _D, _D, _D, _D, ctypes.c_int, _D, _D, _D]
            lib.smb_build.argtypes = [ctypes.c_void_p]
            lib.smb_distribute.argtypes = [ctypes.c_void_p]
            lib.smb_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
            lib.smb_particles.argtypes = [ctypes.c_void_p]
            lib.smb_particles.restype = ctypes.c_long
            lib.smb_get_field.argtypes = [ctypes.c_void_p, ctypes.c_int, _PD]
            lib.smb_threads.restype = ctypes.c_int
            lib.smb_seed.argtypes = [ctypes.c_uint]
            SmbSim._lib = lib
        self.lib = SmbSim._lib
        self.grid = grid
        pml, sig = _make_arrays(grid)
        h = self.lib.smb_new(grid.nr, grid.nz, grid.radius, grid.longitude, grid.dt, r_domains, z_domains, pml, sig)
        assert h, "smb_new refused the decomposition (domains 1 or even per axis)"
        self.h = ctypes.c_void_p(h)

    def seed(self, s: int):
        """Seed the reference's global std::mt19937 (rand.cpp:25)."""
        self.lib.smb_seed(s)

    def add_species(self, sp: SpeciesSpec, macro_amount: float, density: float, temperature: float):
        assert self.lib.smb_add_species(self.h, sp.id, sp.name.encode(), int(sp.charge), int(sp.mass),
                                        float(macro_amount), density, temperature) == 0

    def add_beam(self, sp: SpeciesSpec):
        b = sp.beam
        assert self.lib.smb_add_beam(self.h, sp.id, sp.name.encode(), int(sp.charge), int(sp.mass),
                                     float(b["macro_amount"]), b["start_time"], b["radius"], b["density"],
                                     int(b["amount"]), b["length"], b["distance"], b["velocity"]) == 0

    def build(self):
        assert self.lib.smb_build(self.h) == 0

    def distribute(self):
        assert self.lib.smb_distribute(self.h) == 0

    def step(self, n: int = 1) -> int:
        return self.lib.smb_step(self.h, n)

    def particles(self) -> int:
        return int(self.lib.smb_particles(self.h))

    def threads(self) -> int:
        return int(self.lib.smb_threads())

    def get_field(self, which) -> np.ndarray:
        a = np.zeros(self.grid.shape)
        assert self.lib.smb_get_field(self.h, self.FIELDS.index(which), _dp(a)) == 0
        return a
