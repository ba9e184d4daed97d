"""B200-native elastic-wave solver: a drop-in for the SeisWave Lab Seis3D solver path.

The solver itself is CUDA (csrc/, built into libseis3d_b200.so); this package is the
host-side mirror of the reference API over its C ABI (include/seis3d_capi.h).
"""
from . import capi
from .seis3d import (InvalidArgument, LogicError, Session, SolverError, default_context, default_source,
                     estimate_memory3D, make_cpml_coefficients3D, make_view_layout3D, validate_context3D)

__all__ = ["capi", "InvalidArgument", "LogicError", "Session", "SolverError", "default_context", "default_source",
           "estimate_memory3D", "make_cpml_coefficients3D", "make_view_layout3D", "validate_context3D"]
