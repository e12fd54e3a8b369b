"""picopic_b200 — B200-native PiCoPiC per-timestep PIC loop.

The compute lives in ``libpcg.so`` (CUDA, sm_100a) behind the C ABI of
``include/pcg.h``; :class:`Domain` drives it from Python with the method
names of the reference's ``Domain`` façade.
"""
from ._ffi import PcgError, load  # noqa: F401
from .domain import FIELDS, STAGES, Domain, Geometry  # noqa: F401

__all__ = ["Domain", "Geometry", "PcgError", "FIELDS", "STAGES", "load"]
