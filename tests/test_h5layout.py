"""The probe output tree against the layout of the reference's data.h5.

run() writes every probe as <root>/<path>.npy and data.h5.json beside them
(picopic_b200/h5layout.py).  Here a tree is written for the probes of a small
PiCoPiC.json (fake frames of the right shapes, no GPU) and read back the way
the reference's Python reader reads data.h5 (lib/python/picopic/h5_reader.py
and reader.py): the configuration from the root attribute `metadata`, a
rectangle from the dataset at Reader.__path__ indexed by frame.  The layout
records what OutEngineHDF5 creates: an unlimited frame axis and one-frame
chunks (outEngineHDF5.cpp:119-150), and the root attributes of
write_metadata (outEngineHDF5.cpp:268-389).
"""
import json
import os

import numpy as np
import pytest

from picopic_b200 import config, h5layout

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT_ATTRS = ("metadata", "software", "softwareVersion", "softwareBuildFlags", "softwareDependencies",
              "softwareConfigDebug", "softwareConfigIEEE", "softwareConfigCurrentDeposition",
              "softwareConfigFieldSolver", "softwareConfigParticlesPusher",
              "softwareConfigPlasmaVelocityDistribution", "softwareConfigPlasmaSpatialDistribution", "comment")


def reader_path(component, p_type, shape):
    """Reader.__path__ of the reference's reader (lib/python/picopic/reader.py:51-63)
    for a rectangle, shape = [r0, z0, r1, z1]."""
    assert p_type == "rec"
    return "/{}/{}/{}-{}_{}-{}".format(component, p_type, shape[0], shape[2], shape[1], shape[3])


def frame_shape(p):
    r0, z0, r1, z1 = p.dims
    return {"rec": (r1 - r0, z1 - z0), "col": None, "row": None, "dot": ()}[p.shape]


@pytest.fixture
def tree(tmp_path):
    cfg = config.load(os.path.join(HERE, "golden", "configs", "small.json"))
    nr, nz = cfg.geometry.nr, cfg.geometry.nz
    rng = np.random.default_rng(3)
    frames = 4
    data = {}
    for p in cfg.probes:
        shape = {"rec": frame_shape(p), "col": (nr,), "row": (nz,), "dot": ()}[p.shape]
        data[p.path] = rng.normal(size=(frames,) + tuple(shape))
    attrs = h5layout.root_attributes(cfg.raw, "vay", "zigzag", "f32", "fixed")
    h5layout.write_tree(str(tmp_path), data, attrs)
    return cfg, data, h5layout.Tree(str(tmp_path))


def test_root_attributes_and_metadata(tree):
    cfg, _, f = tree
    attrs = f["/"].attrs
    for k in ROOT_ATTRS:
        assert k in attrs, k
    meta = json.loads(attrs.get("metadata"))  # h5_reader.py:50
    assert meta["geometry"] == cfg.raw["geometry"]
    assert meta["build_options"]["particles_pusher"] == "vay"
    assert meta["build_options"]["current_deposition"] == "zigzag"
    assert attrs["softwareConfigFieldSolver"] == "yee"


def test_reader_finds_every_rectangle_by_its_path(tree):
    cfg, data, f = tree
    recs = [p for p in cfg.probes if p.shape == "rec"]
    assert recs
    for p in recs:
        comp = p.path.split("/rec/")[0]
        path = reader_path(comp, "rec", list(p.dims))
        for number in range(data[p.path].shape[0]):
            frame = f[path][number]  # H5Reader.rec, h5_reader.py:79-93
            assert frame.shape == frame_shape(p)
            assert np.array_equal(frame, data[p.path][number])


def test_every_probe_has_the_data_h5_layout(tree):
    cfg, data, f = tree
    for p in cfg.probes:
        lay = f.layout(p.path)
        a = data[p.path]
        assert lay["shape"] == list(a.shape)
        assert lay["maxshape"][0] is None and lay["maxshape"][1:] == list(a.shape[1:])
        assert lay["chunks"] == [1] + list(a.shape[1:])
        assert lay["dtype"] == "<f8"
        assert np.array_equal(np.asarray(f[p.path]), a)
    # groups list their members as h5py's do
    top = {p.path.split("/")[0] for p in cfg.probes}
    assert set(f["/"].keys()) == top


def test_to_hdf5_needs_h5py(tree, tmp_path):
    try:
        import h5py  # noqa: F401
    except ImportError:
        with pytest.raises(ImportError):
            h5layout.to_hdf5(str(tmp_path))
        return
    cfg, data, _ = tree
    dst = h5layout.to_hdf5(str(tmp_path))
    with h5py.File(dst, "r") as f:
        assert json.loads(f["/"].attrs["metadata"])["geometry"] == cfg.raw["geometry"]
        for path, a in data.items():
            assert np.array_equal(f[path][...], a) and f[path].maxshape[0] is None
