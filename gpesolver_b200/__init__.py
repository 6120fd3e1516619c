"""gpesolver_b200: B200-native backend for GPESolver's solver/ hot path.

The numerical work lives in the CUDA library ``libgpe_b200.so`` (C ABI in
include/gpe_b200.h, sources in gpesolver_b200/csrc).  This package holds the
build recipe, a ctypes binding, the host-side parameter layer and a Python
mirror of the reference's solver interface.
"""
from .capi import GpeError  # noqa: F401
from .params import PhysicalParameters, initial_psi, load_params, params_from_json, potential  # noqa: F401
from .batch import B200Batch  # noqa: F401
from .solver import B200GrossPitaevskiSolver, BECEnergies, make_gpe_params, make_init_params  # noqa: F401

__all__ = [
    "GpeError",
    "PhysicalParameters",
    "B200GrossPitaevskiSolver",
    "B200Batch",
    "make_init_params",
    "BECEnergies",
    "initial_psi",
    "potential",
    "load_params",
    "params_from_json",
    "make_gpe_params",
]
