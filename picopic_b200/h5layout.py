"""The reference's HDF5 output layout, kept without an HDF5 library.

PiCoPiC writes one file, ``data.h5`` under the configuration's data root
(OutWriter, src/outWriter.cpp:49-100, through OutEngineHDF5,
src/outEngine/outEngineHDF5.cpp:52-389):

* one dataset of doubles per probe at ``/<component>/[<specie>/]<shape>/...``
  (the path Cfg::init_probes builds, src/cfg.cpp:204-290), frames on the
  first axis, which is unlimited, in chunks of one frame
  (OutEngineHDF5::create_dataset, outEngineHDF5.cpp:119-150);
* attributes of the root group (OutEngineHDF5::write_metadata,
  outEngineHDF5.cpp:268-389): ``metadata`` (the configuration as JSON, with
  the ``build_options`` object Cfg adds, src/cfg.cpp:60-121), ``software``,
  ``softwareVersion``, ``softwareBuildFlags``, ``softwareDependencies``,
  ``softwareConfigDebug``, ``softwareConfigIEEE``,
  ``softwareConfigCurrentDeposition``, ``softwareConfigFieldSolver``,
  ``softwareConfigParticlesPusher``,
  ``softwareConfigPlasmaVelocityDistribution``,
  ``softwareConfigPlasmaSpatialDistribution`` and ``comment``.

There is no HDF5 library in this build environment, so :func:`write_tree`
stores each dataset as ``<root>/<path>.npy`` and writes ``data.h5.json``
beside them: the root attributes and, per dataset, its path, shape,
maximum shape, chunk shape, type and ``.npy`` file.  :class:`Tree` opens
that tree with the part of h5py's ``File`` interface that the reference's
reader uses (``f['/'].attrs.get('metadata')``, ``f[path][frame]``,
``f[group].keys()``, lib/python/picopic/h5_reader.py:41-170), and
:func:`to_hdf5` writes the real ``data.h5`` from it where h5py is installed.
"""
from __future__ import annotations

import json
import os

import numpy as np

SIDECAR = "data.h5.json"
H5_NAME = "data.h5"
PUSHER_NAMES = {"boris": "boris classic", "borisadaptive": "boris adaptive", "borisrel": "boris relativistic",
                "vay": "vay", "hc": "higuera-cary"}
CURRENT_NAMES = {"vb": "villasenor-buneman", "zigzag": "zigzag"}
VERSION = "1.0"
BUILD_FLAGS = "nvcc -gencode arch=compute_100a,code=sm_100a -O3"


def root_attributes(raw_config: dict, pusher="borisrel", current="vb", precision="f32", quirks="reference",
                    plasma="maxwellian") -> dict:
    """The root attributes OutEngineHDF5::write_metadata writes, for a run
    of the given switches (the reference fixes them at compile time)."""
    cfg = json.loads(json.dumps(raw_config or {}))
    build = {"package_version": VERSION, "debug": False, "ieee": precision == "f64" and quirks == "reference",
             "plasma_spatial_distribution": "flat" if plasma == "reference" else "random",
             "plasma_velocity_distribution": "thermal", "particles_pusher": PUSHER_NAMES[pusher],
             "current_deposition": CURRENT_NAMES[current], "maxwell_solver": "yee", "build_flags": BUILD_FLAGS,
             "precision": precision, "quirks": quirks}
    cfg["build_options"] = build
    return {
        "metadata": json.dumps(cfg),
        "software": "picopic_b200",
        "softwareVersion": VERSION,
        "softwareBuildFlags": BUILD_FLAGS,
        "softwareDependencies": "CUDA runtime (static), NVIDIA driver",
        "softwareConfigDebug": False,
        "softwareConfigIEEE": build["ieee"],
        "softwareConfigCurrentDeposition": build["current_deposition"],
        "softwareConfigFieldSolver": build["maxwell_solver"],
        "softwareConfigParticlesPusher": build["particles_pusher"],
        "softwareConfigPlasmaVelocityDistribution": build["plasma_velocity_distribution"],
        "softwareConfigPlasmaSpatialDistribution": build["plasma_spatial_distribution"],
        "comment": str(cfg.get("comment", "")),
    }


def write_tree(root: str, datasets: dict, attrs: dict) -> str:
    """Write every dataset (path -> array of frames) as <root>/<path>.npy
    and the layout in <root>/data.h5.json; returns the sidecar's path."""
    os.makedirs(root, exist_ok=True)
    entries = {}
    for path, a in datasets.items():
        a = np.asarray(a, dtype=np.float64)
        rel = path.strip("/") + ".npy"
        dst = os.path.join(root, rel)
        os.makedirs(os.path.dirname(dst), exist_ok=True)
        np.save(dst, a)
        shape = list(a.shape) if a.ndim else [0]
        entries["/" + path.strip("/")] = {"shape": shape, "maxshape": [None] + shape[1:],
                                         "chunks": [1] + shape[1:], "dtype": "<f8", "npy": rel}
    side = os.path.join(root, SIDECAR)
    with open(side, "w") as f:
        json.dump({"file": H5_NAME, "attributes": attrs, "datasets": entries}, f, indent=1)
    return side


class _Attrs(dict):
    pass


class _Group:
    def __init__(self, tree, path):
        self._tree, self.name = tree, path
        self.attrs = _Attrs(tree._attrs if path == "/" else {})

    def keys(self):
        pre = self.name.rstrip("/") + "/"
        return sorted({p[len(pre):].split("/")[0] for p in self._tree._datasets if p.startswith(pre)})

    def __getitem__(self, key):
        return self._tree[self.name.rstrip("/") + "/" + str(key).strip("/")]


class Tree:
    """Read access to a tree written by :func:`write_tree`, in the shape of
    h5py's File: ``tree['/'].attrs``, ``tree[dataset_path]`` (an array whose
    first axis is the frame), ``tree[group_path].keys()``."""

    def __init__(self, path: str):
        root = path if os.path.isdir(path) else os.path.dirname(path)
        with open(os.path.join(root, SIDECAR)) as f:
            meta = json.load(f)
        self.root = root
        self._attrs = meta["attributes"]
        self._datasets = meta["datasets"]

    def __getitem__(self, path):
        path = "/" + str(path).strip("/") if path != "/" else "/"
        if path in self._datasets:
            return np.load(os.path.join(self.root, self._datasets[path]["npy"]), mmap_mode="r")
        if path == "/" or any(p.startswith(path + "/") for p in self._datasets):
            return _Group(self, path)
        raise KeyError(path)

    def layout(self, path):
        """shape, maxshape, chunks and dtype of a dataset, as data.h5 has them."""
        return self._datasets["/" + str(path).strip("/")]

    def close(self):
        pass


def to_hdf5(root: str, dst: str | None = None) -> str:
    """Write <root>/data.h5 (or dst) from the tree: every dataset with an
    unlimited first axis and one-frame chunks, the root attributes.  Needs
    h5py, which this build environment does not have."""
    try:
        import h5py
    except ImportError as e:
        raise ImportError("to_hdf5 needs h5py; the tree and data.h5.json hold the same data and layout") from e
    tree = Tree(root)
    dst = dst or os.path.join(root, H5_NAME)
    with h5py.File(dst, "w") as f:
        for k, v in tree._attrs.items():
            f.attrs[k] = v
        for path, meta in tree._datasets.items():
            a = np.asarray(tree[path])
            f.create_dataset(path, data=a, maxshape=tuple(meta["maxshape"]),
                             chunks=tuple(meta["chunks"]) if a.size else None)
    return dst
