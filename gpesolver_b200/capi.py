"""ctypes binding of the gpe_b200 C ABI (include/gpe_b200.h).

The shared library is the in-tree ``gpesolver_b200/libgpe_b200.so``.  Loading
fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpe_b200.so")

GPE_OK = 0
GPE_ERR_ARG = 1
GPE_ERR_SIZE = 2
GPE_ERR_CUDA = 3
GPE_ERR_STATE = 4
GPE_ERR_NUMERIC = 5
GPE_ERR_NOMEM = 6

GPE_PREC_C64 = 0
GPE_PREC_C128 = 1

ERR_NAMES = {1: "GPE_ERR_ARG", 2: "GPE_ERR_SIZE", 3: "GPE_ERR_CUDA", 4: "GPE_ERR_STATE",
             5: "GPE_ERR_NUMERIC", 6: "GPE_ERR_NOMEM"}


class GpeError(RuntimeError):
    """A failed gpe_* call (the reference throws std::runtime_error in these places)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


class gpe_params(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
        ("m", ctypes.c_double), ("n_atoms", ctypes.c_double),
        ("add", ctypes.c_double), ("cdd", ctypes.c_double), ("ggp11", ctypes.c_double),
        ("gamma", ctypes.c_double), ("w_15", ctypes.c_double),
        ("real_time_dt", ctypes.c_double), ("imag_time_dt", ctypes.c_double),
        ("const_edd", ctypes.c_int),
        ("edd", ctypes.c_double), ("edd_start", ctypes.c_double), ("edd_stop", ctypes.c_double),
        ("iter_real", ctypes.c_long),
        ("precision", ctypes.c_int), ("device", ctypes.c_int), ("schedule", ctypes.c_int),
    ]

GPE_SCHED_AUTO = 0
GPE_SCHED_SPLIT = 1


class gpe_init_params(ctypes.Structure):
    _fields_ = [
        ("omega_x", ctypes.c_double), ("omega_y", ctypes.c_double), ("omega_z", ctypes.c_double),
        ("aa", ctypes.c_double), ("b", ctypes.c_double), ("dd", ctypes.c_double),
        ("n_gauss_max", ctypes.c_int),
        ("bec_droplets_x", ctypes.c_int), ("bec_droplets_y", ctypes.c_int), ("bec_droplets_z", ctypes.c_int),
    ]


class gpe_warm_config(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("levels", ctypes.c_int), ("channels", ctypes.c_int * 8),
        ("hidden", ctypes.c_int), ("n_inputs", ctypes.c_int), ("max_batch", ctypes.c_int),
    ]


# GPE_POT_* (registration order of the reference's potentials) and GPE_INIT_*.
POTENTIAL_IDS = {"HARMONIC": 0, "MEXICAN": 1, "MEXICAN_FREE": 2, "CYLINDRICAL": 3, "FREE": 4,
                 "MEXICAN_ASYMETRIC": 5, "MEXICAN_ASYMETRIC_FREE": 6}
INIT_IDS = {"COS": 0, "GAUSS": 1, "MULTIPLE_GAUSS": 2, "SETUP_GAUSS": 3}


_dp = ctypes.POINTER(ctypes.c_double)
_lib = None

# Every entry point declared in include/gpe_b200.h: (name, restype, argtypes).
SIGNATURES = [
    ("gpe_last_error", ctypes.c_char_p, []),
    ("gpe_abi_version", ctypes.c_int, []),
    ("gpe_params_derive", ctypes.c_int, [ctypes.POINTER(gpe_params)]),
    ("gpe_params_edd_at", ctypes.c_int, [ctypes.POINTER(gpe_params), ctypes.c_long, _dp]),
    ("gpe_create", ctypes.c_int, [ctypes.POINTER(gpe_params), ctypes.POINTER(ctypes.c_void_p)]),
    ("gpe_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("gpe_set_stream", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("gpe_get_stream", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    ("gpe_synchronize", ctypes.c_int, [ctypes.c_void_p]),
    ("gpe_load_psi", ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_size_t]),
    ("gpe_import_psi", ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_size_t]),
    ("gpe_load_potential", ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_size_t]),
    ("gpe_export_psi", ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_size_t]),
    ("gpe_export_fi3d", ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_size_t]),
    ("gpe_load_fi3d", ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_size_t]),
    ("gpe_export_psi_async", ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_size_t]),
    ("gpe_export_wait", ctypes.c_int, [ctypes.c_void_p]),
    ("gpe_calc_fi3d", ctypes.c_int, [ctypes.c_void_p]),
    ("gpe_imag_iter_linear_step", ctypes.c_int, [ctypes.c_void_p]),
    ("gpe_imag_iter_nonlinear_step", ctypes.c_int, [ctypes.c_void_p]),
    ("gpe_calc_norm", ctypes.c_int, [ctypes.c_void_p, _dp]),
    ("gpe_normalize", ctypes.c_int, [ctypes.c_void_p]),
    ("gpe_real_fft_potential_half_step", ctypes.c_int, [ctypes.c_void_p]),
    ("gpe_real_fft_kinetic_step", ctypes.c_int, [ctypes.c_void_p]),
    ("gpe_calc_energy", ctypes.c_int, [ctypes.c_void_p, _dp]),
    ("gpe_set_coeffs", ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]),
    ("gpe_imag_steps", ctypes.c_int, [ctypes.c_void_p, ctypes.c_long]),
    ("gpe_imag_steps_energies", ctypes.c_int, [ctypes.c_void_p, ctypes.c_long, ctypes.c_int, _dp]),
    ("gpe_real_steps", ctypes.c_int, [ctypes.c_void_p, ctypes.c_long, ctypes.c_long]),
    ("gpe_launch_count", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
    ("gpe_x_tiles", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    ("gpe_time_kernel", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp]),
    ("gpe_kernel_name", ctypes.c_char_p, [ctypes.c_int]),
    ("gpe_plane_kernel_name", ctypes.c_char_p, [ctypes.c_void_p]),
    ("gpe_init_potential", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(gpe_init_params)]),
    ("gpe_init_psi", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(gpe_init_params)]),
    ("gpe_export_potential", ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_size_t]),
    ("gpe_batch_create", ctypes.c_int,
     [ctypes.POINTER(gpe_params), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("gpe_batch_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("gpe_batch_member", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("gpe_batch_set_stream", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("gpe_batch_imag_steps", ctypes.c_int, [ctypes.c_void_p, ctypes.c_long]),
    ("gpe_warm_create", ctypes.c_int,
     [ctypes.POINTER(gpe_warm_config), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("gpe_warm_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("gpe_warm_num_weights", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t)]),
    ("gpe_warm_set_weights", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    ("gpe_warm_get_weights", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    ("gpe_warm_init_weights", ctypes.c_int, [ctypes.c_void_p, ctypes.c_ulonglong]),
    ("gpe_warm_forward", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    ("gpe_warm_gradients", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
      ctypes.POINTER(ctypes.c_double)]),
    ("gpe_warm_train_step", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_float,
      ctypes.POINTER(ctypes.c_double)]),
    ("gpe_export_amplitude_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    ("gpe_load_amplitude_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    ("gpe_calc_fi3d_noalloc", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
      ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p]),
]

GPE_NOALLOC_SCRATCH_BYTES = 16 << 20

KERNELS = ["DIP_Z_FWD", "DIP_Y_FWD", "DIP_X", "DIP_Y_INV", "DIP_Z_INV", "KIN_Z_FWD", "KIN_Y_FWD",
           "KIN_X", "KIN_Y_INV", "KIN_Z_INV", "PHASE", "IT_UPDATE", "F_X", "F_YINV", "F_Z", "F_YFWD",
           "F_XK", "F_XD", "F_YZ"]


def lib() -> ctypes.CDLL:
    """Load libgpe_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m gpesolver_b200.build` "
                "(the solver has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != GPE_OK:
        raise GpeError(rc, lib().gpe_last_error().decode(errors="replace"))


def dptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_dp)
