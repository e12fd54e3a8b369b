"""The C-ABI library loads and exports every entry point include/pcg.h declares.

No compute call is made here (this runs on machines without a GPU).
"""
import ctypes
import os
import re

from picopic_b200 import _ffi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(REPO, "include", header)).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(pcg_\w+)\s*\(", text, re.M)))


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(_ffi.LIB_PATH)
    names = _declared("pcg.h")
    assert len(names) >= 17
    for name in names:
        assert hasattr(lib, name), name


def test_binding_covers_header():
    assert set(_declared("pcg.h")) <= set(_ffi.SIGNATURES)


def test_abi_version_without_device():
    lib = _ffi.load()
    assert lib.pcg_abi_version() == 1


def test_missing_library_fails_loudly(tmp_path):
    import pytest
    saved = _ffi._lib
    _ffi._lib = None
    try:
        with pytest.raises(ImportError):
            _ffi.load(str(tmp_path / "libpcg.so"))
    finally:
        _ffi._lib = saved


def test_null_handles_are_rejected_without_a_device():
    """Every entry point checks its handle and pointers before any device
    call: a null handle returns PCG_ERR_ARG (-1), also here without a GPU."""
    lib = _ffi.load()
    null = None
    calls = [
        ("pcg_step", (null, 1)), ("pcg_collide", (null, null)), ("pcg_diag", (null, null)),
        ("pcg_set_tiling", (null, 0, 0, 0)), ("pcg_tile_sort", (null, 0, null, null)),
        ("pcg_species_map", (null, 0, 0, null)), ("pcg_set_collision_scheme", (null, 0)),
        ("pcg_set_collision_crowding", (null, 0)),
        ("pcg_set_collisions", (null, 0)), ("pcg_collide_learned", (null, null, null)),
        ("pcg_count", (null, 0, null)), ("pcg_node_charge", (null, null)), ("pcg_stage", (null, 0)),
        ("pcg_synchronize", (null,)), ("pcg_get_stream", (null, null)), ("pcg_set_field", (null, 0, null)),
        ("pcg_export_field", (null, 0, null)), ("pcg_ensemble_create", (null, 0, 1, null)),
        ("pcg_ensemble_step", (null, 1, null)), ("pcg_ensemble_autotune", (null, 1, null)),
        ("pcg_ensemble_destroy", (null,)), ("pcg_ensemble_set_graph", (null, 1)),
        ("pcg_ensemble_graph_info", (null, null, null)),
    ]
    for name, args in calls:
        assert getattr(lib, name)(*args) == -1, name
