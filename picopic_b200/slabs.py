"""One run split along z into slabs, each slab an ordinary domain.

The reference splits its grid into domains (src/PiCoPiC.cpp:212-234, the
SMB grid of src/SMB.cpp:49-176) that step side by side and, after each
field update and deposit, add or copy the two-cell overlaps of their grids
(SMB::field_e_overlay, field_h_overlay, current_overlay, SMB.cpp:566-1229)
and hand particles that left a domain to its neighbour
(SMB::particles_runaway_collector, SMB.cpp:194-564).

Here a slab is a whole domain of its own (a :class:`picopic_b200.Domain`
on a GPU, or any object with the same methods) over its cells k0 <= k < k1
plus ``ghost`` cells on each side that has a neighbour.  The slab runs
unchanged kernels: its ends that are not the run's ends behave as walls,
which corrupts the ghost cells nearest to them, but within one step the
fields and particles of a cell depend only on cells two or three away, so
with ghost >= 4 the slab's own cells come out as the undivided run's do
(to the order of floating-point sums).  After every step the ghost cells
are overwritten from the slabs that own them: the twelve field arrays (E,
the time-centred H, H at integer time, J) column by column, and the
particles: a slab keeps the particles whose z lies in its own cells and
takes copies of its neighbours' particles in its ghost cells.  A particle
moves less than a cell per step, so a particle that crosses into a
neighbour was already there as a copy, pushed with the same fields; the
slab that owns its new position keeps it.

Only the end slabs keep the run's PML at their outer ends and only the
first injects beams (at z = 0).  :class:`SlabGroup` holds every slab in
one process (several domains on one GPU, or one per GPU); :class:`SlabRank`
holds one slab per process and exchanges the ghost strips with its
neighbours through ``torch.distributed`` point-to-point messages of host
tensors (a gloo group).
"""
from __future__ import annotations

import dataclasses

import numpy as np

FIELDS = ["e_r", "e_phi", "e_z", "h_r", "h_phi", "h_z", "hat_r", "hat_phi", "hat_z",
          "j_r", "j_phi", "j_z"]
PARTICLE_KEYS = ("r", "z", "vr", "vphi", "vz", "w")


@dataclasses.dataclass(frozen=True)
class Slab:
    """Slab `index` of `count`: its own cells [k0, k1) along z and the cells
    [e0, e1) its domain covers (its own plus the ghost cells)."""
    index: int
    count: int
    k0: int
    k1: int
    e0: int
    e1: int

    @property
    def first(self):
        return self.index == 0

    @property
    def last(self):
        return self.index == self.count - 1

    @property
    def nz(self):
        return self.e1 - self.e0


def plan(nz: int, count: int, ghost: int = 6) -> list:
    """Slabs of nearly equal length over nz cells."""
    if count < 1 or nz < count:
        raise ValueError(f"{count} slabs of a {nz}-cell grid")
    if ghost < 4:
        raise ValueError("the ghost width must cover the cells a step depends on: at least 4")
    bounds = [round(nz * s / count) for s in range(count + 1)]
    out = []
    for s in range(count):
        k0, k1 = bounds[s], bounds[s + 1]
        if s > 0 and k1 - k0 < ghost:
            raise ValueError(f"slab {s} has {k1 - k0} cells, fewer than the ghost width {ghost}")
        out.append(Slab(s, count, k0, k1, max(0, k0 - ghost), min(nz, k1 + ghost)))
    return out


def slab_geometry(grid, slab: Slab):
    """The geometry of a slab's domain: its cells along z, the run's radius,
    and the run's PML at the ends it shares with the run (pml_size as the
    reference orders it: [1] the z = 0 end, [2] the outer radius, [3] z = L)."""
    pml = list(grid.pml_size)
    if not slab.first:
        pml[1] = 0
    if not slab.last:
        pml[3] = 0
    if (slab.first and pml[1] > slab.k1 - slab.k0) or (slab.last and pml[3] > slab.k1 - slab.k0):
        raise ValueError("an end slab must hold the PML of its end")
    return dataclasses.replace(grid, nz=slab.nz, longitude=slab.nz * grid.dz, pml_size=tuple(pml))


def _owned(z, slab: Slab, dz):
    lo = -np.inf if slab.first else slab.k0 * dz
    hi = np.inf if slab.last else slab.k1 * dz
    return (z >= lo) & (z < hi)


def _strip(p, lo, hi):
    """The particles (global z) with lo <= z < hi."""
    m = (p["z"] >= lo) & (p["z"] < hi)
    return {k: p[k][m] for k in PARTICLE_KEYS}


def _cat(parts):
    return {k: np.concatenate([p[k] for p in parts]) for k in PARTICLE_KEYS}


class _SlabEngine:
    """A slab's domain with global coordinates on the outside."""

    def __init__(self, grid, slab: Slab, engine, species_count):
        self.grid, self.slab, self.engine, self.nsp = grid, slab, engine, species_count
        self.z0 = slab.e0 * grid.dz  # global z of the domain's z = 0

    # particles in global z
    def particles(self, slot):
        p = self.engine.get_particles(slot)
        out = {k: np.asarray(p[k], dtype=np.float64) for k in PARTICLE_KEYS}
        out["z"] = out["z"] + self.z0
        return out

    def set_particles(self, slot, p):
        self.engine.set_particles(slot, p["r"], p["z"] - self.z0, p["vr"], p["vphi"], p["vz"], p["w"])

    # field columns: global node k is local column k - e0 + 2
    def local(self, name):
        return self.engine.get_field(name)

    def col(self, k):
        return k - self.slab.e0 + 2


def _ghost_widths(slabs):
    """(left ghost, right ghost) cell counts of each slab."""
    return [(s.k0 - s.e0, s.e1 - s.k1) for s in slabs]


class SlabGroup:
    """Every slab of the run in this process.

    make_engine(geometry, slab) returns a domain for the slab's geometry
    with the run's species added in the same order (a beam with its
    injection in the first slab only, plain in the others); the group sets
    its particles and fields from global arrays and steps all slabs."""

    def __init__(self, grid, count, make_engine, species_count, ghost=6):
        self.grid = grid
        self.slabs = plan(grid.nz, count, ghost)
        self.widths = _ghost_widths(self.slabs)
        self.nsp = species_count
        self.parts = [_SlabEngine(grid, s, make_engine(slab_geometry(grid, s), s), species_count)
                      for s in self.slabs]

    # -- set-up from global data ------------------------------------------------------
    def set_particles(self, slot, r, z, vr, vphi, vz, w):
        p = {"r": np.asarray(r, float), "z": np.asarray(z, float), "vr": np.asarray(vr, float),
             "vphi": np.asarray(vphi, float), "vz": np.asarray(vz, float), "w": np.asarray(w, float)}
        for se in self.parts:
            s, dz = se.slab, self.grid.dz
            lo = -np.inf if s.first else s.e0 * dz
            hi = np.inf if s.last else s.e1 * dz
            se.set_particles(slot, _strip(p, lo, hi))

    def set_field(self, name, a):
        """A global (nr+4) x (nz+4) array: each domain gets its columns, with
        the halo columns the global array has (zeros beyond it)."""
        a = np.asarray(a, dtype=np.float64)
        for se in self.parts:
            s = se.slab
            loc = np.zeros((a.shape[0], s.nz + 4))
            for lc in range(s.nz + 4):
                gk = lc - 2 + s.e0 + 2  # global array column
                if 0 <= gk < a.shape[1]:
                    loc[:, lc] = a[:, gk]
            se.engine.set_field(name, loc)

    # -- stepping ------------------------------------------------------------------------
    def step(self, n=1):
        for _ in range(n):
            for se in self.parts:
                se.engine.step(1)
            self.exchange()

    def exchange(self):
        dz = self.grid.dz
        fields = [{f: se.local(f) for f in FIELDS} for se in self.parts]
        owned = []
        for se in self.parts:
            slots = []
            for t in range(self.nsp):
                p = se.particles(t)
                m = _owned(p["z"], se.slab, dz)
                slots.append({k: p[k][m] for k in PARTICLE_KEYS})
            owned.append(slots)
        for i, se in enumerate(self.parts):
            s = se.slab
            lw, rw = self.widths[i]
            # fields: ghost columns from the owners
            for f in FIELDS:
                a = fields[i][f]
                if lw:
                    src = self.parts[i - 1]
                    a[:, se.col(s.e0):se.col(s.k0)] = fields[i - 1][f][:, src.col(s.e0):src.col(s.k0)]
                if rw:
                    src = self.parts[i + 1]
                    a[:, se.col(s.k1):se.col(s.e1)] = fields[i + 1][f][:, src.col(s.k1):src.col(s.e1)]
                se.engine.set_field(f, a)
            # particles: own ones, then copies of the neighbours' in the ghost cells
            for t in range(self.nsp):
                parts = [owned[i][t]]
                if lw:
                    parts.append(_strip(owned[i - 1][t], s.e0 * dz, s.k0 * dz))
                if rw:
                    parts.append(_strip(owned[i + 1][t], s.k1 * dz, s.e1 * dz))
                se.set_particles(t, _cat(parts))

    # -- global views ------------------------------------------------------------------
    def get_field(self, name):
        """The run's (nr+4) x (nz+4) array from the slabs' own columns (and
        the end slabs' outer halo columns)."""
        out = np.zeros((self.grid.nr + 4, self.grid.nz + 4))
        for se in self.parts:
            s = se.slab
            a = se.local(name)
            lo = s.k0 - (2 if s.first else 0)
            hi = s.k1 + (2 if s.last else 0)
            out[:, lo + 2:hi + 2] = a[:, se.col(lo):se.col(hi)]
        return out

    def get_particles(self, slot):
        """The run's particles of a species: each slab's own (global z)."""
        parts = []
        for se in self.parts:
            p = se.particles(slot)
            m = _owned(p["z"], se.slab, self.grid.dz)
            parts.append({k: p[k][m] for k in PARTICLE_KEYS})
        return _cat(parts)


class SlabRank:
    """One slab per process: rank r of a torch.distributed group (host
    tensors: a gloo group) holds slab r and exchanges the ghost strips
    with ranks r - 1 and r + 1 after every step.  Every rank calls the same
    methods in the same order."""

    def __init__(self, grid, make_engine, species_count, group=None, ghost=6):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.rank, self.size = dist.get_rank(group), dist.get_world_size(group)
        self.grid = grid
        self.slabs = plan(grid.nz, self.size, ghost)
        self.widths = _ghost_widths(self.slabs)
        self.slab = self.slabs[self.rank]
        self.nsp = species_count
        self.se = _SlabEngine(grid, self.slab, make_engine(slab_geometry(grid, self.slab), self.slab),
                              species_count)

    # point-to-point of numpy arrays (shape known to both sides)
    def _send(self, a, peer):
        import torch
        self.dist.send(torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)), dst=peer, group=self.group)

    def _recv(self, shape, peer):
        import torch
        t = torch.empty(shape, dtype=torch.float64)
        self.dist.recv(t, src=peer, group=self.group)
        return t.numpy()

    def _send_particles(self, p, peer):
        self._send(np.array([p["r"].size], dtype=np.float64), peer)
        if p["r"].size:
            self._send(np.stack([p[k] for k in PARTICLE_KEYS]), peer)

    def _recv_particles(self, peer):
        n = int(self._recv((1,), peer)[0])
        if n == 0:
            return {k: np.zeros(0) for k in PARTICLE_KEYS}
        a = self._recv((len(PARTICLE_KEYS), n), peer)
        return {k: a[q] for q, k in enumerate(PARTICLE_KEYS)}

    def set_particles(self, slot, r, z, vr, vphi, vz, w):
        """Global arrays (the same on every rank): the slab keeps its own and ghost ones."""
        s, dz = self.slab, self.grid.dz
        p = {"r": np.asarray(r, float), "z": np.asarray(z, float), "vr": np.asarray(vr, float),
             "vphi": np.asarray(vphi, float), "vz": np.asarray(vz, float), "w": np.asarray(w, float)}
        lo = -np.inf if s.first else s.e0 * dz
        hi = np.inf if s.last else s.e1 * dz
        self.se.set_particles(slot, _strip(p, lo, hi))

    def set_field(self, name, a):
        s = self.slab
        loc = np.zeros((a.shape[0], s.nz + 4))
        for lc in range(s.nz + 4):
            gk = lc + s.e0
            if 0 <= gk < a.shape[1]:
                loc[:, lc] = a[:, gk]
        self.se.engine.set_field(name, loc)

    def step(self, n=1):
        for _ in range(n):
            self.se.engine.step(1)
            self.exchange()

    def exchange(self):
        s, se, dz = self.slab, self.se, self.grid.dz
        lw, rw = self.widths[self.rank]
        fields = {f: se.local(f) for f in FIELDS}
        owned = []
        for t in range(self.nsp):
            p = se.particles(t)
            m = _owned(p["z"], s, dz)
            owned.append({k: p[k][m] for k in PARTICLE_KEYS})
        # the strips each neighbour needs: its ghost columns are these own columns
        left, right = self.rank - 1, self.rank + 1
        nl = self.widths[left][1] if not s.first else 0    # the left slab's right ghost width
        nr = self.widths[right][0] if not s.last else 0    # the right slab's left ghost width
        rows = self.grid.nr + 4
        # even ranks send first, odd ranks receive first: no two ranks wait on each other
        def to_left():
            for f in FIELDS:
                self._send(fields[f][:, se.col(s.k0):se.col(s.k0 + nl)], left)
            for t in range(self.nsp):
                self._send_particles(_strip(owned[t], s.k0 * dz, (s.k0 + nl) * dz), left)

        def to_right():
            for f in FIELDS:
                self._send(fields[f][:, se.col(s.k1 - nr):se.col(s.k1)], right)
            for t in range(self.nsp):
                self._send_particles(_strip(owned[t], (s.k1 - nr) * dz, s.k1 * dz), right)

        got_left = got_right = None

        def from_left():
            f_ = {f: self._recv((rows, lw), left) for f in FIELDS}
            return f_, [self._recv_particles(left) for _ in range(self.nsp)]

        def from_right():
            f_ = {f: self._recv((rows, rw), right) for f in FIELDS}
            return f_, [self._recv_particles(right) for _ in range(self.nsp)]

        # phase 1: left-to-right along the chain; phase 2: right-to-left
        if self.rank % 2 == 0:
            if not s.last:
                to_right()
            if not s.first:
                got_left = from_left()
            if not s.first:
                to_left()
            if not s.last:
                got_right = from_right()
        else:
            if not s.first:
                got_left = from_left()
            if not s.last:
                to_right()
            if not s.last:
                got_right = from_right()
            if not s.first:
                to_left()
        for f in FIELDS:
            a = fields[f]
            if got_left is not None:
                a[:, se.col(s.e0):se.col(s.k0)] = got_left[0][f]
            if got_right is not None:
                a[:, se.col(s.k1):se.col(s.e1)] = got_right[0][f]
            se.engine.set_field(f, a)
        for t in range(self.nsp):
            parts = [owned[t]]
            if got_left is not None:
                parts.append(got_left[1][t])
            if got_right is not None:
                parts.append(got_right[1][t])
            se.set_particles(t, _cat(parts))

    def own_field_columns(self, name):
        """This slab's own columns of a field (the end slabs with their outer halo):
        (first global node, array)."""
        s, se = self.slab, self.se
        lo = s.k0 - (2 if s.first else 0)
        hi = s.k1 + (2 if s.last else 0)
        return lo, se.local(name)[:, se.col(lo):se.col(hi)]

    def own_particles(self, slot):
        p = self.se.particles(slot)
        m = _owned(p["z"], self.slab, self.grid.dz)
        return {k: p[k][m] for k in PARTICLE_KEYS}
