"""Band-of-z particle selection and field column copies (pcg_export_species_range,
pcg_keep_species_range, pcg_get_field_columns, pcg_set_field_columns) on
both particle layouts, against the whole-array exports of the same domain.

The band export must return exactly the particles of the whole export with
lo <= z < hi (the same z: bit-equal), the keep must leave exactly those
(the complement of the two side bands, so a hand-over neither loses nor
doubles a particle), and an append beyond the capacity must succeed once
the dead slots of a keep are reclaimed.
"""
import numpy as np
import pytest

from tests.cases import ELECTRONS, particles, random_fields, small_grid

pytestmark = pytest.mark.gpu

KEYS = ("r", "z", "vr", "vphi", "vz", "w")


def _domain(grid, precision, cap=20000):
    from picopic_b200 import Domain
    d = Domain(grid, pusher="borisrel", current="vb", precision=precision, seed=7)
    d.add(ELECTRONS, capacity=cap)
    return d


def _sorted(p):
    order = np.lexsort((p["vz"], p["r"], p["z"]))
    return {k: np.asarray(p[k])[order] for k in KEYS}


def _equal(a, b):
    a, b = _sorted(a), _sorted(b)
    assert a["r"].size == b["r"].size
    for k in KEYS:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_band_export_and_keep_split_the_particles(precision):
    grid = small_grid(nr=16, nz=96)
    d = _domain(grid, precision)
    p = particles(grid, 12000, 11)
    d.set_particles(0, *p)
    for name, a in random_fields(grid, 2).items():
        d.set_field(name, a)
    d.step(3)  # float layout: tile-sorted, with dead slots of the runaways
    whole = d.get_particles(0)
    z = whole["z"]
    lo, hi = 31 * grid.dz, 64.5 * grid.dz
    band = d.export_range(0, lo, hi)
    m = (z >= lo) & (z < hi)
    _equal(band, {k: whole[k][m] for k in KEYS})
    left, right = d.export_range(0, -np.inf, lo), d.export_range(0, hi, np.inf)
    assert left["r"].size + band["r"].size + right["r"].size == z.size
    assert d.export_range(0, hi, lo)["r"].size == 0
    d.keep_range(0, lo, hi)
    assert d.count(0) == m.sum()
    _equal(d.get_particles(0), {k: whole[k][m] for k in KEYS})
    # the kept particles step on: the same as a domain given only them
    ref = _domain(grid, precision)
    ref.set_particles(0, *[whole[k][m] for k in KEYS])
    for name in random_fields(grid, 2):
        ref.set_field(name, d.get_field(name))
    d.step(2)
    ref.step(2)
    a, b = _sorted(d.get_particles(0)), _sorted(ref.get_particles(0))
    assert a["r"].size == b["r"].size
    tol = 1e-12 if precision == "f64" else 1e-6  # the deposit adds in another order
    for k in KEYS:
        np.testing.assert_allclose(a[k], b[k], rtol=0, atol=tol * np.abs(b[k]).max(), err_msg=k)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_append_reclaims_dead_slots_before_giving_up(precision):
    grid = small_grid(nr=16, nz=96)
    d = _domain(grid, precision, cap=4000)
    p = particles(grid, 4000, 5)
    d.set_particles(0, *p)
    d.keep_range(0, 0.0, grid.longitude / 2)
    live = int((p[1] < grid.longitude / 2).sum())  # no count(): it would compact
    extra = particles(grid, 4000 - live, 6)
    d.set_particles(0, *extra, append=True)
    assert d.count(0) == 4000
    from picopic_b200._ffi import PcgError
    with pytest.raises(PcgError):
        d.set_particles(0, *particles(grid, 1, 7), append=True)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_field_columns(precision):
    grid = small_grid(nr=16, nz=96)
    d = _domain(grid, precision)
    fields = random_fields(grid, 4)
    for name, a in fields.items():
        d.set_field(name, a)
    rng = np.random.default_rng(1)
    for name, a in fields.items():
        whole = d.get_field(name)
        for c0, c1 in ((0, 5), (40, 52), (grid.nz - 2, grid.nz + 4)):
            np.testing.assert_array_equal(d.get_field_columns(name, c0, c1), whole[:, c0:c1])
        new = rng.normal(size=(grid.nr + 4, 7))
        d.set_field_columns(name, 20, new)
        expect = whole.copy()
        expect[:, 20:27] = new if precision == "f64" else new.astype(np.float32)
        np.testing.assert_array_equal(d.get_field(name), expect)
    from picopic_b200._ffi import PcgError
    with pytest.raises(PcgError):
        d.get_field_columns("e_r", 90, grid.nz + 5)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_transfer_between_domains_on_the_device(precision):
    """A band of one domain appended to (or replacing) another domain's species
    with z shifted, device to device: the same particles as the band's host
    export, shifted; and the source keeps all of its own."""
    grid = small_grid(nr=16, nz=96)
    src, dst = _domain(grid, precision), _domain(grid, precision)
    src.set_particles(0, *particles(grid, 6000, 21))
    dst.set_particles(0, *particles(grid, 500, 22))
    for name, a in random_fields(grid, 3).items():
        src.set_field(name, a)
    src.step(2)
    before = dst.get_particles(0)
    lo, hi, shift = 60 * grid.dz, np.inf, 50 * grid.dz
    band = src.export_range(0, lo, hi)
    n_src = src.count(0)
    assert src.transfer_range(0, lo, hi, shift, dst, 0, append=True) == band["r"].size > 0
    assert src.count(0) == n_src
    got = dst.get_particles(0)
    expect = {k: np.concatenate([before[k], band[k] - (shift if k == "z" else 0.0)]) for k in KEYS}
    a, b = _sorted(got), _sorted(expect)
    assert a["r"].size == b["r"].size
    for k in KEYS:  # the float layout re-splits z into cell and offset: within its rounding
        np.testing.assert_allclose(a[k], b[k], rtol=0, atol=(0 if precision == "f64" else 1e-7) * np.abs(b[k]).max(),
                                   err_msg=k)
    assert src.transfer_range(0, -np.inf, 10 * grid.dz, 0.0, dst, 0, append=False) == dst.count(0)
    if precision == "f64":  # a replacement: exactly the band
        _equal(dst.get_particles(0), src.export_range(0, -np.inf, 10 * grid.dz))
    # the destination steps on with what it received
    dst.step(1)
    assert dst.count(0) > 0


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_field_columns_between_domains_on_the_device(precision):
    grid = small_grid(nr=16, nz=96)
    src, dst = _domain(grid, precision), _domain(grid, precision)
    fa, fb = random_fields(grid, 8), random_fields(grid, 9)
    for name in fa:
        src.set_field(name, fa[name])
        dst.set_field(name, fb[name])
    src.copy_field_columns(10, 17, dst, 60)
    src.copy_field_columns(30, 32, dst, 0, which="j_z")
    for name in fa:
        a, b = src.get_field(name), _get_expected(fb[name], precision)
        b[:, 60:67] = a[:, 10:17]
        if name == "j_z":
            b[:, 0:2] = a[:, 30:32]
        np.testing.assert_array_equal(dst.get_field(name), b, err_msg=name)
    from picopic_b200._ffi import PcgError
    with pytest.raises(PcgError):
        src.copy_field_columns(90, grid.nz + 4, dst, 95)


def _get_expected(a, precision):
    return a.copy() if precision == "f64" else a.astype(np.float32).astype(np.float64)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_device_buffers(precision):
    """The particle and column calls with CUDA tensors in place of host arrays
    (what an NCCL exchange sends) give what the host arrays give."""
    import torch
    grid = small_grid(nr=16, nz=96)
    src, dst = _domain(grid, precision), _domain(grid, precision)
    src.set_particles(0, *particles(grid, 5000, 31))
    for name, a in random_fields(grid, 5).items():
        src.set_field(name, a)
    src.step(2)
    lo, hi = 20 * grid.dz, 41 * grid.dz
    t = src.export_range_device(0, lo, hi)
    assert t.is_cuda and t.shape[0] == 6
    band = src.export_range(0, lo, hi)
    _equal({k: t[q].cpu().numpy() for q, k in enumerate(KEYS)}, band)
    dst.set_particles_device(0, t)
    _equal(dst.export_range(0, -np.inf, np.inf), dst.get_particles(0))
    assert dst.count(0) == band["r"].size
    dst.set_particles_device(0, t[:, :7], append=True)
    assert dst.count(0) == band["r"].size + 7
    c = src.get_field_columns_device("e_z", 30, 45)
    np.testing.assert_array_equal(c.cpu().numpy(), src.get_field_columns("e_z", 30, 45))
    dst.set_field_columns_device("h_phi", 3, c)
    np.testing.assert_array_equal(dst.get_field_columns("h_phi", 3, 18), c.cpu().numpy())
    empty = src.export_range_device(0, hi, lo)
    assert empty.shape == (6, 0)
    torch.cuda.synchronize()


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_transfer_bands_in_one_call(precision):
    """Several bands of one source to two destinations in one call: each band
    selected from the source as it was at the call, imported in band order
    (the first band to a slot replaces, the next appends)."""
    grid = small_grid(nr=16, nz=96)
    src, a, b = (_domain(grid, precision) for _ in range(3))
    src.set_particles(0, *particles(grid, 6000, 41))
    a.set_particles(0, *particles(grid, 300, 42))
    b.set_particles(0, *particles(grid, 300, 43))
    src.step(1)
    dz = grid.dz
    bands = [(0, -np.inf, 20 * dz, 0.0, a, 0, False),
             (0, 70 * dz, np.inf, 10 * dz, b, 0, True),
             (0, 20 * dz, 40 * dz, -5 * dz, a, 0, True)]
    expect_a = [src.export_range(0, -np.inf, 20 * dz), src.export_range(0, 20 * dz, 40 * dz)]
    expect_a[1]["z"] = expect_a[1]["z"] + 5 * dz
    before_b = b.get_particles(0)
    band_b = src.export_range(0, 70 * dz, np.inf)
    band_b["z"] = band_b["z"] - 10 * dz
    counts = src.transfer_bands(bands)
    assert counts == [expect_a[0]["r"].size, band_b["r"].size, expect_a[1]["r"].size]
    tol = 0 if precision == "f64" else 1e-7
    for got, parts in ((a.get_particles(0), expect_a), (b.get_particles(0), [before_b, band_b])):
        x, y = _sorted(got), _sorted({k: np.concatenate([p[k] for p in parts]) for k in KEYS})
        assert x["r"].size == y["r"].size
        for k in KEYS:
            np.testing.assert_allclose(x[k], y[k], rtol=0, atol=tol * np.abs(y[k]).max(), err_msg=k)
    from picopic_b200._ffi import PcgError
    with pytest.raises(PcgError):  # a band into the source itself
        src.transfer_bands([(0, 0.0, dz, 0.0, src, 0, True)])
