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
particles.  Each species has two slots in a slab's domain: the particles
the slab owns and the ghost copies of its neighbours' particles, pushed
alongside (with the same fields, so they deposit the same currents into
the own cells near the boundary).  After a step the owner hands the own
particles that left its cells to the neighbour (a particle moves less than
a cell per step, so only to a neighbour) and then sends copies of the own
particles in the neighbours' ghost cells, which replace their ghost slots.

Only the end slabs keep the run's PML at their outer ends and only the
first injects beams (at z = 0).  :class:`SlabGroup` holds every slab in
one process (several domains on one GPU, or one per GPU); :class:`SlabRank`
holds one slab per process and exchanges the strips with its neighbours
through ``torch.distributed`` point-to-point messages of host tensors (a
gloo group).
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


@dataclasses.dataclass(frozen=True)
class GhostSpecies:
    """The ghost copies of a species in a slab's domain: the species'
    charge and mass, no injection (what ``add`` of a domain reads)."""
    name: str
    charge: float
    mass: float
    id: int = 0
    capacity: int | None = None
    beam: None = None


def _owned(z, slab: Slab, dz):
    lo = -np.inf if slab.first else slab.k0 * dz
    hi = np.inf if slab.last else slab.k1 * dz
    return (z >= lo) & (z < hi)


def _strip(p, lo, hi):
    """The particles (global z) with lo <= z < hi."""
    m = (p["z"] >= lo) & (p["z"] < hi)
    return {k: p[k][m] for k in PARTICLE_KEYS}


def _cat(parts):
    parts = [p for p in parts if p is not None]
    if not parts:
        return {k: np.zeros(0) for k in PARTICLE_KEYS}
    return {k: np.concatenate([p[k] for p in parts]) for k in PARTICLE_KEYS}


def _empty():
    return {k: np.zeros(0) for k in PARTICLE_KEYS}


class _SlabEngine:
    """A slab's domain with global coordinates on the outside.

    Species slot t < nsp holds the particles the slab owns (z in its own
    cells, as this domain computes z); slot nsp + t holds the copies of the
    neighbours' particles of species t in the ghost cells, replaced at every
    exchange.  A particle's owner alone decides where it goes after a step,
    with one computation of its z for both the hand-over and the keep, so
    no particle is lost or doubled at a slab boundary, however close to it.
    Band selections and column copies go through the domain's own
    ``export_range``/``keep_range``/``get_field_columns``/
    ``set_field_columns`` where it has them (a GPU domain: only the strips
    cross to the host), else through whole-array copies."""

    def __init__(self, grid, slab: Slab, engine, species_count):
        self.grid, self.slab, self.engine, self.nsp = grid, slab, engine, species_count
        dz = grid.dz
        self.z0 = slab.e0 * dz  # global z of the domain's z = 0
        # own cells in the domain's coordinates
        self.lo = -np.inf if slab.first else (slab.k0 - slab.e0) * dz
        self.hi = np.inf if slab.last else (slab.k1 - slab.e0) * dz

    # -- band selections, in the domain's coordinates --------------------------------
    def _export(self, slot, lo, hi):
        e = self.engine
        if hasattr(e, "export_range"):
            p = e.export_range(slot, lo, hi)
        else:
            q = e.get_particles(slot)
            z = np.asarray(q["z"], dtype=np.float64)
            m = (z >= lo) & (z < hi)
            p = {k: np.asarray(q[k], dtype=np.float64)[m] for k in PARTICLE_KEYS}
        out = {k: np.asarray(p[k], dtype=np.float64) for k in PARTICLE_KEYS}
        out["z"] = out["z"] + self.z0
        return out

    def _keep(self, slot, lo, hi):
        e = self.engine
        if hasattr(e, "keep_range"):
            e.keep_range(slot, lo, hi)
            return
        q = e.get_particles(slot)
        z = np.asarray(q["z"], dtype=np.float64)
        m = (z >= lo) & (z < hi)
        e.set_particles(slot, *[np.asarray(q[k], dtype=np.float64)[m] for k in PARTICLE_KEYS])

    def _put(self, slot, p, append):
        arrs = [p[k] for k in PARTICLE_KEYS]
        arrs[1] = p["z"] - self.z0
        e = self.engine
        if not append:
            e.set_particles(slot, *arrs)
        elif arrs[0].size:
            if hasattr(e, "export_range"):  # a domain with pcg_append_species
                e.set_particles(slot, *arrs, append=True)
            else:
                q = e.get_particles(slot)
                e.set_particles(slot, *[np.concatenate([np.asarray(q[k], dtype=np.float64), a])
                                        for k, a in zip(PARTICLE_KEYS, arrs)])

    # -- the particle hand-over ---------------------------------------------------------
    def migrants(self, t):
        """Own particles that left the own cells (to the left, to the right),
        global z; they are removed here."""
        s = self.slab
        left = None if s.first else self._export(t, -np.inf, self.lo)
        right = None if s.last else self._export(t, self.hi, np.inf)
        if not (s.first and s.last):
            self._keep(t, self.lo, self.hi)
        return left, right

    def take(self, t, parts):
        """Append the migrants that neighbours handed over."""
        self._put(t, _cat(parts), append=True)

    def strips(self, t, nl, nr):
        """Copies of the own particles in the neighbours' ghost cells: the
        first nl own cells (and anything further left) and the last nr."""
        s, dz = self.slab, self.grid.dz
        left = None if s.first else self._export(t, -np.inf, (s.k0 + nl - s.e0) * dz)
        right = None if s.last else self._export(t, (s.k1 - nr - s.e0) * dz, np.inf)
        return left, right

    def set_ghosts(self, t, parts):
        self._put(self.nsp + t, _cat(parts), append=False)

    def own(self, t):
        return self._export(t, -np.inf, np.inf)

    # -- field columns: global node k is local column k - e0 + 2 -----------------------
    def col(self, k):
        return k - self.slab.e0 + 2

    def columns(self, name, k0, k1):
        e = self.engine
        if hasattr(e, "get_field_columns"):
            return e.get_field_columns(name, self.col(k0), self.col(k1))
        return np.asarray(e.get_field(name))[:, self.col(k0):self.col(k1)].copy()

    def set_columns(self, name, k0, a):
        e = self.engine
        if hasattr(e, "set_field_columns"):
            e.set_field_columns(name, self.col(k0), a)
            return
        full = np.array(e.get_field(name), dtype=np.float64)
        full[:, self.col(k0):self.col(k0) + a.shape[1]] = a
        e.set_field(name, full)

    def field_strips(self, nl, nr):
        """The own columns of every field that the neighbours hold as ghosts."""
        s = self.slab
        left = None if s.first else {f: self.columns(f, s.k0, s.k0 + nl) for f in FIELDS}
        right = None if s.last else {f: self.columns(f, s.k1 - nr, s.k1) for f in FIELDS}
        return left, right

    def set_ghost_fields(self, left, right):
        s = self.slab
        for f in FIELDS:
            if left is not None:
                self.set_columns(f, s.e0, left[f])
            if right is not None:
                self.set_columns(f, s.k1, right[f])

    # -- set-up from global data ----------------------------------------------------------
    def set_particles(self, t, p):
        """Global particles: the own ones and the ghost copies."""
        s, dz = self.slab, self.grid.dz
        m = _owned(p["z"], s, dz)
        g = ~m & (p["z"] >= s.e0 * dz) & (p["z"] < s.e1 * dz)
        self._put(t, {k: p[k][m] for k in PARTICLE_KEYS}, append=False)
        self._put(self.nsp + t, {k: p[k][g] for k in PARTICLE_KEYS}, append=False)

    def set_field(self, name, a):
        """The domain's columns of a global (nr+4) x (nz+4) array (its halo
        columns where the global array has them, zeros beyond)."""
        s = self.slab
        loc = np.zeros((a.shape[0], s.nz + 4))
        for lc in range(s.nz + 4):
            gk = lc + s.e0  # global array column
            if 0 <= gk < a.shape[1]:
                loc[:, lc] = a[:, gk]
        self.engine.set_field(name, loc)


def _ghost_widths(slabs):
    """(left ghost, right ghost) cell counts of each slab."""
    return [(s.k0 - s.e0, s.e1 - s.k1) for s in slabs]


def _add_ghosts(engine, species, capacity):
    for sp in species:
        engine.add(GhostSpecies(sp.name + ".ghost", sp.charge, sp.mass, getattr(sp, "id", 0), capacity))


class SlabGroup:
    """Every slab of the run in this process.

    make_engine(geometry, slab) returns a domain for the slab's geometry
    with the run's species added in the given order (a beam with its
    injection in the first slab only, plain in the others); the group adds
    the ghost species after them, sets the slabs' particles and fields from
    global arrays and steps all slabs."""

    def __init__(self, grid, count, make_engine, species, ghost=6, ghost_capacity=None, on_device=None):
        self.grid = grid
        self.slabs = plan(grid.nz, count, ghost)
        self.widths = _ghost_widths(self.slabs)
        self.nsp = len(species)
        self.parts = []
        for s in self.slabs:
            e = make_engine(slab_geometry(grid, s), s)
            _add_ghosts(e, species, ghost_capacity)
            self.parts.append(_SlabEngine(grid, s, e, self.nsp))
        # device to device (GPU domains: pcg_transfer_species_range and
        # pcg_copy_field_columns, a peer copy between GPUs), else through the host
        can = all(hasattr(se.engine, "transfer_bands") and hasattr(se.engine, "copy_field_columns")
                  for se in self.parts)
        if on_device and not can:
            raise ValueError("the slabs' engines have no device-to-device exchange")
        self.on_device = can if on_device is None else bool(on_device)

    # -- set-up from global data ------------------------------------------------------
    def set_particles(self, slot, r, z, vr, vphi, vz, w):
        p = {"r": np.asarray(r, float), "z": np.asarray(z, float), "vr": np.asarray(vr, float),
             "vphi": np.asarray(vphi, float), "vz": np.asarray(vz, float), "w": np.asarray(w, float)}
        for se in self.parts:
            se.set_particles(slot, p)

    def set_field(self, name, a):
        a = np.asarray(a, dtype=np.float64)
        for se in self.parts:
            se.set_field(name, a)

    # -- stepping ------------------------------------------------------------------------
    def step(self, n=1):
        for _ in range(n):
            for se in self.parts:
                se.engine.step(1)
            self.exchange()

    def _neighbour_widths(self, i):
        s = self.slabs[i]
        nl = 0 if s.first else self.widths[i - 1][1]  # the left slab's right ghost width
        nr = 0 if s.last else self.widths[i + 1][0]   # the right slab's left ghost width
        return nl, nr

    def exchange(self):
        if self.on_device:
            self._exchange_on_device()
            return
        last = len(self.parts) - 1
        # 1. owners hand over the particles that left their cells
        mig = [[se.migrants(t) for t in range(self.nsp)] for se in self.parts]
        for i, se in enumerate(self.parts):
            for t in range(self.nsp):
                se.take(t, [mig[i - 1][t][1] if i > 0 else None, mig[i + 1][t][0] if i < last else None])
        # 2. ghost columns and ghost particles from the owners
        fs, ps = [], []
        for i, se in enumerate(self.parts):
            nl, nr = self._neighbour_widths(i)
            fs.append(se.field_strips(nl, nr))
            ps.append([se.strips(t, nl, nr) for t in range(self.nsp)])
        for i, se in enumerate(self.parts):
            se.set_ghost_fields(fs[i - 1][1] if i > 0 else None, fs[i + 1][0] if i < last else None)
            for t in range(self.nsp):
                se.set_ghosts(t, [ps[i - 1][t][1] if i > 0 else None, ps[i + 1][t][0] if i < last else None])

    def _exchange_on_device(self):
        """The same exchange with the strips moved between the domains on the
        device (one band transfer call, one host wait, per slab and phase);
        only the particle counts reach the host.  The slabs go in order: a
        slab's hand-over sees the migrants its left neighbour has just
        appended and passes on any that lie outside its own cells."""
        last, dz, inf = len(self.parts) - 1, self.grid.dz, np.inf
        for i, se in enumerate(self.parts):
            s = se.slab
            bands = []
            for t in range(self.nsp):
                if not s.first:
                    nb = self.parts[i - 1]
                    bands.append((t, -inf, se.lo, nb.z0 - se.z0, nb.engine, t, True))
                if not s.last:
                    nb = self.parts[i + 1]
                    bands.append((t, se.hi, inf, nb.z0 - se.z0, nb.engine, t, True))
            se.engine.transfer_bands(bands)
            if not (s.first and s.last):
                for t in range(self.nsp):
                    se.engine.keep_range(t, se.lo, se.hi)
        for i, se in enumerate(self.parts):
            s = se.slab
            lw, rw = self.widths[i]
            if i > 0:  # left ghost columns: global nodes [e0, k0) of the left slab
                src = self.parts[i - 1]
                src.engine.copy_field_columns(src.col(s.e0), src.col(s.k0), se.engine, se.col(s.e0))
            if i < last:
                src = self.parts[i + 1]
                src.engine.copy_field_columns(src.col(s.k1), src.col(s.e1), se.engine, se.col(s.k1))
        # ghost particles: slab i sends to i - 1 (after i - 2 has replaced that
        # slab's ghosts: append) and to i + 1 (the first to reach it: replace)
        for i, se in enumerate(self.parts):
            s = se.slab
            bands = []
            for t in range(self.nsp):
                if i > 0:  # the left slab's right ghost cells: our first cells
                    dst = self.parts[i - 1]
                    hi = (s.k0 + self.widths[i - 1][1] - s.e0) * dz
                    bands.append((t, -inf, hi, dst.z0 - se.z0, dst.engine, self.nsp + t, i - 1 > 0))
                if i < last:  # the right slab's left ghost cells: our last cells
                    dst = self.parts[i + 1]
                    lo = (s.k1 - self.widths[i + 1][0] - s.e0) * dz
                    bands.append((t, lo, inf, dst.z0 - se.z0, dst.engine, self.nsp + t, False))
            se.engine.transfer_bands(bands)

    # -- global views ------------------------------------------------------------------
    def get_field(self, name):
        """The run's (nr+4) x (nz+4) array from the slabs' own columns (and
        the end slabs' outer halo columns)."""
        out = np.zeros((self.grid.nr + 4, self.grid.nz + 4))
        for se in self.parts:
            s = se.slab
            lo = s.k0 - (2 if s.first else 0)
            hi = s.k1 + (2 if s.last else 0)
            out[:, lo + 2:hi + 2] = se.columns(name, lo, hi)
        return out

    def get_particles(self, slot):
        """The run's particles of a species: each slab's own (global z)."""
        return _cat([se.own(slot) for se in self.parts])


class SlabRank:
    """One slab per process: rank r of a torch.distributed group holds slab
    r and exchanges the migrants and the ghost strips with ranks r - 1 and
    r + 1 after every step.  Every rank calls the same methods in the same
    order.  Over a gloo group the strips travel as host tensors; over an
    NCCL group, with GPU domains (``export_range_device`` and the other
    device-buffer methods of :class:`picopic_b200.Domain`), they stay on
    the GPUs: band exports and column copies into CUDA tensors, NCCL
    point-to-point sends between the ranks' GPUs."""

    def __init__(self, grid, make_engine, species, group=None, ghost=6, ghost_capacity=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.rank, self.size = dist.get_rank(group), dist.get_world_size(group)
        self.grid = grid
        self.slabs = plan(grid.nz, self.size, ghost)
        self.widths = _ghost_widths(self.slabs)
        self.slab = self.slabs[self.rank]
        self.nsp = len(species)
        e = make_engine(slab_geometry(grid, self.slab), self.slab)
        _add_ghosts(e, species, ghost_capacity)
        self.se = _SlabEngine(grid, self.slab, e, self.nsp)
        on_gpu = dist.get_backend(group) == "nccl" and hasattr(e, "export_range_device")
        self.device = e.torch_device if on_gpu else None

    # point-to-point of float64 arrays (shape known to both sides): numpy
    # arrays through host tensors, or CUDA tensors in place
    def _send(self, a, peer):
        import torch
        if self.device is not None:
            t = a if torch.is_tensor(a) else torch.as_tensor(np.asarray(a, dtype=np.float64), device=self.device)
            self.dist.send(t.contiguous(), dst=peer, group=self.group)
        else:
            self.dist.send(torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)), dst=peer, group=self.group)

    def _recv(self, shape, peer):
        import torch
        t = torch.empty(shape, dtype=torch.float64, device=self.device or "cpu")
        self.dist.recv(t, src=peer, group=self.group)
        return t if self.device is not None else t.numpy()

    def _send_particles(self, p, peer):
        """A particle set: a dict of arrays, or a (6, n) CUDA tensor."""
        n = p.shape[1] if self.device is not None else p["r"].size
        self._send(np.array([n], dtype=np.float64), peer)
        if n:
            self._send(p if self.device is not None else np.stack([p[k] for k in PARTICLE_KEYS]), peer)

    def _recv_particles(self, peer):
        n = int(self._recv((1,), peer)[0])
        if self.device is not None:
            return self._recv((len(PARTICLE_KEYS), n), peer) if n else None
        if n == 0:
            return _empty()
        a = self._recv((len(PARTICLE_KEYS), n), peer)
        return {k: a[q] for q, k in enumerate(PARTICLE_KEYS)}

    def _swap(self, send_left, send_right, recv_left, recv_right):
        """One exchange with both neighbours: even ranks send first, odd
        ranks receive first, so no two ranks wait on each other."""
        s = self.slab
        left, right = self.rank - 1, self.rank + 1
        got_l = got_r = None
        if self.rank % 2 == 0:
            if not s.last:
                send_right(right)
            if not s.first:
                got_l = recv_left(left)
            if not s.first:
                send_left(left)
            if not s.last:
                got_r = recv_right(right)
        else:
            if not s.first:
                got_l = recv_left(left)
            if not s.last:
                send_right(right)
            if not s.last:
                got_r = recv_right(right)
            if not s.first:
                send_left(left)
        return got_l, got_r

    def set_particles(self, slot, r, z, vr, vphi, vz, w):
        """Global arrays (the same on every rank): the slab keeps its own and ghost ones."""
        p = {"r": np.asarray(r, float), "z": np.asarray(z, float), "vr": np.asarray(vr, float),
             "vphi": np.asarray(vphi, float), "vz": np.asarray(vz, float), "w": np.asarray(w, float)}
        self.se.set_particles(slot, p)

    def set_field(self, name, a):
        self.se.set_field(name, np.asarray(a, dtype=np.float64))

    def step(self, n=1):
        for _ in range(n):
            self.se.engine.step(1)
            self.exchange()

    def exchange(self):
        if self.device is not None:
            self._exchange_on_device()
            return
        s, se, nsp = self.slab, self.se, self.nsp
        lw, rw = self.widths[self.rank]
        rows = self.grid.nr + 4
        # 1. migrants
        mig = [se.migrants(t) for t in range(nsp)]
        got_l, got_r = self._swap(
            lambda peer: [self._send_particles(mig[t][0], peer) for t in range(nsp)],
            lambda peer: [self._send_particles(mig[t][1], peer) for t in range(nsp)],
            lambda peer: [self._recv_particles(peer) for _ in range(nsp)],
            lambda peer: [self._recv_particles(peer) for _ in range(nsp)])
        for t in range(nsp):
            se.take(t, [got_l[t] if got_l else None, got_r[t] if got_r else None])
        # 2. ghost columns and ghost particles
        nl = 0 if s.first else self.widths[self.rank - 1][1]
        nr = 0 if s.last else self.widths[self.rank + 1][0]
        fl, fr = se.field_strips(nl, nr)
        ps = [se.strips(t, nl, nr) for t in range(nsp)]

        def send(fields, side):
            def go(peer):
                for f in FIELDS:
                    self._send(fields[f], peer)
                for t in range(nsp):
                    self._send_particles(ps[t][side], peer)
            return go

        def recv(width):
            def go(peer):
                f_ = {f: self._recv((rows, width), peer) for f in FIELDS}
                return f_, [self._recv_particles(peer) for _ in range(nsp)]
            return go

        got_l, got_r = self._swap(send(fl, 0), send(fr, 1), recv(lw), recv(rw))
        se.set_ghost_fields(got_l[0] if got_l else None, got_r[0] if got_r else None)
        for t in range(nsp):
            se.set_ghosts(t, [got_l[1][t] if got_l else None, got_r[1][t] if got_r else None])

    def _exchange_on_device(self):
        """The exchange with CUDA tensors: the same two rounds (migrants, then
        ghost columns and ghost particles), z shifted on the GPU."""
        import torch
        s, se, nsp, e = self.slab, self.se, self.nsp, self.se.engine
        lw, rw = self.widths[self.rank]
        rows, dz, inf = self.grid.nr + 4, self.grid.dz, np.inf

        def out(t):  # domain z to global z
            if t is not None and t.shape[1]:
                t[1] += se.z0
            return t

        def into(parts, slot, append):  # global z to domain z, then import
            parts = [q for q in parts if q is not None and q.shape[1]]
            t = torch.cat(parts, dim=1) if parts else torch.zeros((6, 0), dtype=torch.float64, device=self.device)
            t[1] -= se.z0
            if t.shape[1] or not append:
                e.set_particles_device(slot, t, append=append)

        mig = []
        for t in range(nsp):
            left = None if s.first else out(e.export_range_device(t, -inf, se.lo))
            right = None if s.last else out(e.export_range_device(t, se.hi, inf))
            if not (s.first and s.last):
                e.keep_range(t, se.lo, se.hi)
            mig.append((left, right))
        got_l, got_r = self._swap(
            lambda peer: [self._send_particles(mig[t][0], peer) for t in range(nsp)],
            lambda peer: [self._send_particles(mig[t][1], peer) for t in range(nsp)],
            lambda peer: [self._recv_particles(peer) for _ in range(nsp)],
            lambda peer: [self._recv_particles(peer) for _ in range(nsp)])
        for t in range(nsp):
            into([got_l[t] if got_l else None, got_r[t] if got_r else None], t, append=True)
        nl = 0 if s.first else self.widths[self.rank - 1][1]
        nr = 0 if s.last else self.widths[self.rank + 1][0]
        fl = None if s.first else {f: e.get_field_columns_device(f, se.col(s.k0), se.col(s.k0 + nl)) for f in FIELDS}
        fr = None if s.last else {f: e.get_field_columns_device(f, se.col(s.k1 - nr), se.col(s.k1)) for f in FIELDS}
        ps = [(None if s.first else out(e.export_range_device(t, -inf, (s.k0 + nl - s.e0) * dz)),
               None if s.last else out(e.export_range_device(t, (s.k1 - nr - s.e0) * dz, inf)))
              for t in range(nsp)]

        def send(fields, side):
            def go(peer):
                for f in FIELDS:
                    self._send(fields[f], peer)
                for t in range(nsp):
                    self._send_particles(ps[t][side], peer)
            return go

        def recv(width):
            def go(peer):
                f_ = {f: self._recv((rows, width), peer) for f in FIELDS}
                return f_, [self._recv_particles(peer) for _ in range(nsp)]
            return go

        got_l, got_r = self._swap(send(fl, 0), send(fr, 1), recv(lw), recv(rw))
        for f in FIELDS:
            if got_l is not None:
                e.set_field_columns_device(f, se.col(s.e0), got_l[0][f])
            if got_r is not None:
                e.set_field_columns_device(f, se.col(s.k1), got_r[0][f])
        for t in range(nsp):
            into([got_l[1][t] if got_l else None, got_r[1][t] if got_r else None], nsp + t, append=False)

    def own_field_columns(self, name):
        """This slab's own columns of a field (the end slabs with their outer halo):
        (first global node, array)."""
        s = self.slab
        lo = s.k0 - (2 if s.first else 0)
        hi = s.k1 + (2 if s.last else 0)
        return lo, self.se.columns(name, lo, hi)

    def own_particles(self, slot):
        return self.se.own(slot)
