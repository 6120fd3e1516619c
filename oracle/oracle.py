"""Python bindings of the oracle libraries -- TEST INFRASTRUCTURE ONLY.

Two CPU FP64 implementations of GPESolver's solver hot path live under oracle/:

* ``libgpe_oracle.so``: the project's plain-C restatement (gpe_oracle.c), each
  function citing the reference file:line it restates;
* ``_ref/libgpe_ref.so``: the reference's own unmodified CPU sources compiled in
  place (oracle/Makefile) around a small harness (ref_harness.cpp).

``_ref/libgpe_adapter.so`` (and ``_ref/libgpe_adapter_fused.so``) link the
reference's own base class and driver with the B200 adapter
(gpesolver_b200/adapter) instead of its CPU backend: the GPU tests use them to run
the reference's control flow on the B200 backend.

Both use the FP64 FFTW-API shim in oracle/fftw_shim because FFTW3 is not in this
image.  Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline
import this module; the product path never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libgpe_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libgpe_ref.so")
ADAPTER_SO = os.path.join(HERE, "_ref", "libgpe_adapter.so")
ADAPTER_FUSED_SO = os.path.join(HERE, "_ref", "libgpe_adapter_fused.so")
# calc_strategy of solve() (src/parameters/complex_param.hpp:14-20).
STRATEGIES = {"IT": 0, "RT": 1, "FS": 2}

# Potential ids in the reference's registration order (src/parameters/potentials.hpp:76-157).
POTENTIALS = {
    "HARMONIC": 0,
    "MEXICAN": 1,
    "MEXICAN_FREE": 2,
    "CYLINDRICAL": 3,
    "FREE": 4,
    "MEXICAN_ASYMETRIC": 5,
    "MEXICAN_ASYMETRIC_FREE": 6,
}
# InitializationOption (src/parameters/complex_param.hpp:57-97); file-based
# strategies are handled by the caller (load_buffer).
INITS = {"COS": 0, "GAUSS": 1, "MULTIPLE_GAUSS": 2, "SETUP_GAUSS": 3}

_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def build(ref: bool = True) -> None:
    """Build the oracle libraries with oracle/Makefile (the reference only if its
    sources are present)."""
    targets = ["libgpe_oracle.so"]
    if ref and os.path.isdir(os.environ.get("GPE_REFERENCE_DIR", "/root/reference") + "/src"):
        targets.append("ref")
        if os.path.exists(os.path.join(os.path.dirname(HERE), "gpesolver_b200", "libgpe_b200.so")):
            targets.append("adapter")
        targets.append("refgpu")
    subprocess.check_call(["make", "-s", "-C", HERE] + targets)


class Params(ctypes.Structure):
    """Mirror of gpeo_params (oracle/gpe_oracle.h)."""

    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
        ("m", ctypes.c_double), ("n_atoms", ctypes.c_double),
        ("omega_x", ctypes.c_double), ("omega_y", ctypes.c_double), ("omega_z", ctypes.c_double),
        ("dd", ctypes.c_double),
        ("const_edd", ctypes.c_int),
        ("edd", ctypes.c_double), ("edd_start", ctypes.c_double), ("edd_stop", ctypes.c_double),
        ("iter_imag", ctypes.c_long), ("iter_real", ctypes.c_long),
        ("real_time_dt", ctypes.c_double), ("imag_time_dt", ctypes.c_double),
        ("fftw_n_threads", ctypes.c_int),
        ("aa", ctypes.c_double), ("b", ctypes.c_double), ("dxdydz", ctypes.c_double),
        ("add", ctypes.c_double), ("cdd", ctypes.c_double), ("ggp11", ctypes.c_double),
        ("gamma", ctypes.c_double), ("w_15", ctypes.c_double),
    ]


class RefConfig(ctypes.Structure):
    """Mirror of gperef_config (oracle/ref_harness.cpp): gpe_params.json units."""

    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx_nm", ctypes.c_double), ("dy_nm", ctypes.c_double), ("dz_nm", ctypes.c_double),
        ("m_da", ctypes.c_double), ("n_atoms", ctypes.c_double),
        ("omega_x_hz", ctypes.c_double), ("omega_y_hz", ctypes.c_double),
        ("omega_z_hz", ctypes.c_double), ("dd_nm", ctypes.c_double),
        ("const_edd", ctypes.c_int), ("edd", ctypes.c_double),
        ("edd_start", ctypes.c_double), ("edd_stop", ctypes.c_double),
        ("iter_imag", ctypes.c_long), ("iter_real", ctypes.c_long),
        ("init_strategy", ctypes.c_int), ("n_gauss_max", ctypes.c_int),
        ("bec_droplets_x", ctypes.c_int), ("bec_droplets_y", ctypes.c_int),
        ("bec_droplets_z", ctypes.c_int), ("fftw_n_threads", ctypes.c_int),
        ("pote_key", ctypes.c_char * 32),
    ]


def default_config(**kw) -> dict:
    """A gpe_params.json-like dict (file units: nm, Da, Hz) with the README's values."""
    cfg = dict(nx=64, ny=64, nz=16, dx=120.0, dy=120.0, dz=600.0, m=163.929, n_atoms=2e4,
               omega_x=60.0, omega_y=60.0, omega_z=120.0, dd=1500.0, edd=1.5,
               edd_start=None, edd_stop=None, iter_imag=1000, iter_real=10000,
               init_strategy="GAUSS", initial_maximas=2, bec_droplets_x=3, bec_droplets_y=3,
               bec_droplets_z=2, pote_strategy="HARMONIC", fftw_n_threads=4)
    cfg.update(kw)
    return cfg


# ---------------------------------------------------------------------------
# The plain-C restatement
# ---------------------------------------------------------------------------
_olib = None


def olib():
    global _olib
    if _olib is None:
        L = ctypes.CDLL(ORACLE_SO)
        for name in ["gpeo_len_nm_to_au", "gpeo_len_au_to_nm", "gpeo_mass_da_to_au",
                     "gpeo_freq_hz_to_au", "gpeo_ene_au_to_mev"]:
            getattr(L, name).restype = ctypes.c_double
            getattr(L, name).argtypes = [ctypes.c_double]
        L.gpeo_create.restype = ctypes.c_void_p
        L.gpeo_create.argtypes = [ctypes.POINTER(Params)]
        L.gpeo_destroy.argtypes = [ctypes.c_void_p]
        L.gpeo_solver_params.restype = ctypes.POINTER(Params)
        L.gpeo_solver_params.argtypes = [ctypes.c_void_p]
        for name in ["gpeo_psi", "gpeo_psii", "gpeo_fi3d", "gpeo_pote"]:
            getattr(L, name).restype = _dp
            getattr(L, name).argtypes = [ctypes.c_void_p]
        L.gpeo_calc_norm.restype = ctypes.c_double
        L.gpeo_calc_norm.argtypes = [ctypes.c_void_p]
        for name in ["gpeo_calc_fi3d", "gpeo_imag_iter_linear_step", "gpeo_imag_iter_nonlinear_step",
                     "gpeo_normalize", "gpeo_real_fft_potential_half_step",
                     "gpeo_real_fft_kinetic_step", "gpeo_imag_time_iter", "gpeo_real_time_iter"]:
            getattr(L, name).argtypes = [ctypes.c_void_p]
        L.gpeo_imag_steps.argtypes = [ctypes.c_void_p, ctypes.c_long]
        L.gpeo_real_steps.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_long]
        L.gpeo_calc_energy.argtypes = [ctypes.c_void_p, _dp]
        L.gpeo_load_buffer.argtypes = [ctypes.c_void_p, _dp]
        L.gpeo_load_pote.argtypes = [ctypes.c_void_p, _dp]
        L.gpeo_potential.argtypes = [ctypes.POINTER(Params), ctypes.c_int, _dp]
        L.gpeo_init_psi.argtypes = [ctypes.POINTER(Params), ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
        L.gpeo_coords.argtypes = [ctypes.POINTER(Params), _dp, _dp, _dp]
        L.gpeo_init_parameters.argtypes = [ctypes.POINTER(Params)]
        L.gpeo_update_edd.argtypes = [ctypes.POINTER(Params), ctypes.c_uint]
        L.gpeo_default_dt.argtypes = [ctypes.POINTER(Params)]
        _olib = L
    return _olib


def make_params(cfg: dict) -> Params:
    """gpe_params.json units -> atomic units, as FileManager::load_* does
    (src/filemanager/file_manager.cpp:468-541), then init_parameters."""
    L = olib()
    p = Params()
    p.nx, p.ny, p.nz = cfg["nx"], cfg["ny"], cfg["nz"]
    p.dx = L.gpeo_len_nm_to_au(cfg["dx"])
    p.dy = L.gpeo_len_nm_to_au(cfg["dy"])
    p.dz = L.gpeo_len_nm_to_au(cfg["dz"])
    p.m = L.gpeo_mass_da_to_au(cfg["m"])
    p.n_atoms = cfg["n_atoms"]
    p.omega_x = L.gpeo_freq_hz_to_au(cfg["omega_x"])
    p.omega_y = L.gpeo_freq_hz_to_au(cfg["omega_y"])
    p.omega_z = L.gpeo_freq_hz_to_au(cfg["omega_z"])
    p.dd = L.gpeo_len_nm_to_au(cfg["dd"])
    if cfg.get("edd") is not None:
        p.const_edd, p.edd = 1, cfg["edd"]
    else:
        p.const_edd = 0
        p.edd_start, p.edd_stop = cfg["edd_start"], cfg["edd_stop"]
        p.edd = cfg["edd_start"]
    p.iter_imag, p.iter_real = cfg["iter_imag"], cfg["iter_real"]
    p.fftw_n_threads = cfg.get("fftw_n_threads", 4)
    L.gpeo_default_dt(ctypes.byref(p))
    L.gpeo_init_parameters(ctypes.byref(p))
    return p


def potential(p: Params, name: str) -> np.ndarray:
    V = np.zeros(p.nx * p.ny * p.nz)
    rc = olib().gpeo_potential(ctypes.byref(p), POTENTIALS[name], _ptr(V))
    assert rc == 0
    return V


def initial_psi(p: Params, cfg: dict) -> np.ndarray:
    psi = np.zeros(2 * p.nx * p.ny * p.nz)
    rc = olib().gpeo_init_psi(ctypes.byref(p), INITS[cfg["init_strategy"]],
                              cfg.get("initial_maximas", 2), cfg.get("bec_droplets_x", 1),
                              cfg.get("bec_droplets_y", 1), cfg.get("bec_droplets_z", 1), _ptr(psi))
    assert rc == 0
    return psi


def as_complex(flat: np.ndarray, p) -> np.ndarray:
    return flat.view(np.complex128).reshape(p.nx, p.ny, p.nz)


class OracleSolver:
    """The restated CPU backend: same calls as CpuGrossPitaevskiSolver."""

    def __init__(self, cfg: dict, load_initial: bool = True):
        L = olib()
        self.cfg = cfg
        self.params = make_params(cfg)
        self.h = L.gpeo_create(ctypes.byref(self.params))
        self.n = self.params.nx * self.params.ny * self.params.nz
        if load_initial:
            self.load_pote(potential(self.params, cfg["pote_strategy"]))
            self.load_buffer(initial_psi(self.params, cfg))

    def close(self):
        if self.h:
            olib().gpeo_destroy(self.h)
            self.h = None

    __del__ = close

    @property
    def p(self) -> Params:
        return olib().gpeo_solver_params(self.h).contents

    def load_buffer(self, psi_c128_flat: np.ndarray):
        a = np.ascontiguousarray(psi_c128_flat, dtype=np.float64)
        olib().gpeo_load_buffer(self.h, _ptr(a))

    def load_pote(self, V: np.ndarray):
        a = np.ascontiguousarray(V, dtype=np.float64)
        olib().gpeo_load_pote(self.h, _ptr(a))

    def change_potential(self, name: str):
        self.load_pote(potential(self.p, name))

    def psi(self) -> np.ndarray:
        return np.ctypeslib.as_array(olib().gpeo_psi(self.h), shape=(2 * self.n,)).copy()

    def fi3d(self) -> np.ndarray:
        return np.ctypeslib.as_array(olib().gpeo_fi3d(self.h), shape=(self.n,)).copy()

    def pote(self) -> np.ndarray:
        return np.ctypeslib.as_array(olib().gpeo_pote(self.h), shape=(self.n,)).copy()

    def calc_fi3d(self):
        olib().gpeo_calc_fi3d(self.h)

    def calc_norm(self) -> float:
        return olib().gpeo_calc_norm(self.h)

    def normalize(self):
        olib().gpeo_normalize(self.h)

    def imag_steps(self, k: int):
        olib().gpeo_imag_steps(self.h, k)

    def real_steps(self, k: int, first_iter: int = 0):
        olib().gpeo_real_steps(self.h, k, first_iter)

    def potential_half_step(self):
        olib().gpeo_real_fft_potential_half_step(self.h)

    def kinetic_step(self):
        olib().gpeo_real_fft_kinetic_step(self.h)

    def imag_linear_step(self):
        olib().gpeo_imag_iter_linear_step(self.h)

    def imag_nonlinear_step(self):
        olib().gpeo_imag_iter_nonlinear_step(self.h)

    def energy(self) -> np.ndarray:
        out = np.zeros(6)
        olib().gpeo_calc_energy(self.h, _ptr(out))
        return out


# ---------------------------------------------------------------------------
# The compiled reference (oracle/_ref/libgpe_ref.so)
# ---------------------------------------------------------------------------
_rlib = None


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def rlib():
    global _rlib
    if _rlib is None:
        L = ctypes.CDLL(REF_SO)
        L.gperef_create.argtypes = [ctypes.POINTER(RefConfig)]
        L.gperef_last_error.restype = ctypes.c_char_p
        L.gperef_norm.restype = ctypes.c_double
        for name in ["gperef_export_psi", "gperef_export_fi3d", "gperef_export_pote",
                     "gperef_energy", "gperef_load_psi", "gperef_load_pote",
                     "gperef_coefficients", "gperef_peek_psi"]:
            getattr(L, name).argtypes = [_dp]
        L.gperef_imag_steps.argtypes = [ctypes.c_long]
        L.gperef_real_steps.argtypes = [ctypes.c_long, ctypes.c_long]
        L.gperef_update_edd.argtypes = [ctypes.c_long]
        L.gperef_change_potential.argtypes = [ctypes.c_char_p]
        L.gperef_op.argtypes = [ctypes.c_int]
        L.gperef_solve.argtypes = [ctypes.c_int]
        for name in ("gperef_save_binary", "gperef_save_text", "gperef_save_pote_text"):
            getattr(L, name).argtypes = [ctypes.c_char_p]
        L.gperef_load_binary.argtypes = [ctypes.c_char_p, _dp]
        L.gperef_checkpoints.restype = ctypes.c_long
        L.gperef_saved_energies.restype = ctypes.c_long
        L.gperef_saved_energies.argtypes = [_dp, ctypes.c_long]
        _rlib = L
    return _rlib


REF_OPS = {"calc_fi3d": 0, "imag_iter_linear_step": 1, "imag_iter_nonlinear_step": 2,
           "calc_norm": 3, "normalize": 4, "real_fft_potential_half_step": 5,
           "real_fft_kinetic_step": 6, "calc_energy": 7}


def ref_config(cfg: dict, load_initial: bool = True) -> RefConfig:
    """gperef_config from a gpe_params.json-style dict (default_config())."""
    c = RefConfig()
    c.nx, c.ny, c.nz = cfg["nx"], cfg["ny"], cfg["nz"]
    c.dx_nm, c.dy_nm, c.dz_nm = cfg["dx"], cfg["dy"], cfg["dz"]
    c.m_da, c.n_atoms = cfg["m"], cfg["n_atoms"]
    c.omega_x_hz, c.omega_y_hz, c.omega_z_hz = cfg["omega_x"], cfg["omega_y"], cfg["omega_z"]
    c.dd_nm = cfg["dd"]
    if cfg.get("edd") is not None:
        c.const_edd, c.edd = 1, cfg["edd"]
    else:
        c.const_edd, c.edd_start, c.edd_stop = 0, cfg["edd_start"], cfg["edd_stop"]
    c.iter_imag, c.iter_real = cfg["iter_imag"], cfg["iter_real"]
    c.init_strategy = INITS[cfg["init_strategy"]] if load_initial else 4
    c.n_gauss_max = cfg.get("initial_maximas", 2)
    c.bec_droplets_x = cfg.get("bec_droplets_x", 1)
    c.bec_droplets_y = cfg.get("bec_droplets_y", 1)
    c.bec_droplets_z = cfg.get("bec_droplets_z", 1)
    c.fftw_n_threads = cfg.get("fftw_n_threads", 4)
    c.pote_key = cfg["pote_strategy"].encode()
    return c


class RefSolver:
    """The reference's own CpuGrossPitaevskiSolver, driven through the harness.

    The reference keeps its parameters in process-wide singletons, so only one
    RefSolver is live at a time."""

    def __init__(self, cfg: dict, load_initial: bool = True):
        L = rlib()
        c = ref_config(cfg, load_initial)
        rc = L.gperef_create(ctypes.byref(c))
        if rc != 0:
            raise RuntimeError(L.gperef_last_error().decode())
        self.cfg = cfg
        self.shape = (cfg["nx"], cfg["ny"], cfg["nz"])
        self.n = cfg["nx"] * cfg["ny"] * cfg["nz"]

    def close(self):
        rlib().gperef_destroy()

    def coefficients(self) -> dict:
        out = np.zeros(15)
        rlib().gperef_coefficients(_ptr(out))
        keys = ["m", "dx", "dy", "dz", "cdd", "ggp11", "gamma", "w_15", "aa", "b", "dd",
                "omega_x", "omega_y", "omega_z", "edd"]
        return dict(zip(keys, out))

    def psi(self) -> np.ndarray:
        out = np.zeros(2 * self.n)
        rlib().gperef_peek_psi(_ptr(out))
        return out

    def fi3d(self) -> np.ndarray:
        out = np.zeros(self.n)
        rlib().gperef_export_fi3d(_ptr(out))
        return out

    def pote(self) -> np.ndarray:
        out = np.zeros(self.n)
        rlib().gperef_export_pote(_ptr(out))
        return out

    def load_buffer(self, psi):
        a = np.ascontiguousarray(psi, dtype=np.float64)
        rlib().gperef_load_psi(_ptr(a))

    def load_pote(self, V):
        a = np.ascontiguousarray(V, dtype=np.float64)
        rlib().gperef_load_pote(_ptr(a))

    def change_potential(self, name: str):
        rc = rlib().gperef_change_potential(name.encode())
        assert rc == 0

    def op(self, name: str):
        rlib().gperef_op(REF_OPS[name])

    def norm(self) -> float:
        return rlib().gperef_norm()

    def imag_steps(self, k: int):
        rlib().gperef_imag_steps(k)

    def real_steps(self, k: int, first_iter: int = 0):
        rlib().gperef_real_steps(k, first_iter)

    def energy(self) -> np.ndarray:
        out = np.zeros(6)
        rlib().gperef_energy(_ptr(out))
        return out

    def solve(self, strategy: str):
        """AbstractGrossPitaevskiSolver::solve with calc_strategy IT / RT / FS."""
        rc = rlib().gperef_solve(STRATEGIES[strategy])
        if rc != 0:
            raise RuntimeError(rlib().gperef_last_error().decode())

    def checkpoints(self) -> int:
        return rlib().gperef_checkpoints()

    def saved_energies(self) -> np.ndarray:
        return _saved_energies(rlib().gperef_saved_energies)


    # the reference's FileManager (names without extension; energies into the
    # working directory's energy.gpe.dat)
    def save_binary(self, name: str):
        assert rlib().gperef_save_binary(name.encode()) == 0, rlib().gperef_last_error()

    def save_text(self, name: str):
        assert rlib().gperef_save_text(name.encode()) == 0, rlib().gperef_last_error()

    def save_pote_text(self, name: str):
        assert rlib().gperef_save_pote_text(name.encode()) == 0, rlib().gperef_last_error()

    def save_energies(self):
        assert rlib().gperef_save_energies() == 0, rlib().gperef_last_error()

    def load_binary(self, name: str) -> np.ndarray:
        out = np.zeros(2 * self.n)
        if rlib().gperef_load_binary(name.encode(), _ptr(out)) != 0:
            raise RuntimeError(rlib().gperef_last_error().decode())
        return out


def _saved_energies(fn) -> np.ndarray:
    n = fn(None, 0)
    out = np.zeros((max(n, 0), 6))
    if n > 0:
        fn(_ptr(out), n)
    return out


_alibs: dict = {}


def alib(fused: bool = False):
    path = ADAPTER_FUSED_SO if fused else ADAPTER_SO
    if path not in _alibs:
        L = ctypes.CDLL(path)
        L.gpeadp_create.argtypes = [ctypes.POINTER(RefConfig), ctypes.c_int]
        L.gpeadp_last_error.restype = ctypes.c_char_p
        L.gpeadp_imag_steps.argtypes = [ctypes.c_long]
        L.gpeadp_real_steps.argtypes = [ctypes.c_long, ctypes.c_long]
        L.gpeadp_solve.argtypes = [ctypes.c_int]
        L.gpeadp_export_psi.argtypes = [_dp]
        L.gpeadp_energy.argtypes = [_dp]
        L.gpeadp_checkpoints.restype = ctypes.c_long
        L.gpeadp_saved_energies.restype = ctypes.c_long
        L.gpeadp_saved_energies.argtypes = [_dp, ctypes.c_long]
        _alibs[path] = L
    return _alibs[path]


class AdapterSolver:
    """The reference's own AbstractGrossPitaevskiSolver code driving the B200
    backend through gpesolver_b200/adapter (B200GrossPitaevskiSolver).

    ``fused`` selects the build with GPE_B200_FUSED_LOOPS (calc_initial_state /
    calc_evolution run as fused device calls).  Needs a GPU."""

    def __init__(self, cfg: dict, precision: int = 0, fused: bool = False):
        self.L = alib(fused)
        rc = self.L.gpeadp_create(ctypes.byref(ref_config(cfg)), precision)
        if rc != 0:
            raise RuntimeError(self.L.gpeadp_last_error().decode())
        self.n = cfg["nx"] * cfg["ny"] * cfg["nz"]

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.L.gpeadp_last_error().decode())

    def close(self):
        self.L.gpeadp_destroy()

    def imag_steps(self, k: int):
        self._check(self.L.gpeadp_imag_steps(k))

    def real_steps(self, k: int, first_iter: int = 0):
        self._check(self.L.gpeadp_real_steps(k, first_iter))

    def solve(self, strategy: str):
        self._check(self.L.gpeadp_solve(STRATEGIES[strategy]))

    def psi(self) -> np.ndarray:
        out = np.zeros(2 * self.n)
        self._check(self.L.gpeadp_export_psi(_ptr(out)))
        return out

    def energy(self) -> np.ndarray:
        out = np.zeros(6)
        self._check(self.L.gpeadp_energy(_ptr(out)))
        return out

    def checkpoints(self) -> int:
        return self.L.gpeadp_checkpoints()

    def saved_energies(self) -> np.ndarray:
        return _saved_energies(self.L.gpeadp_saved_energies)


# ---------------------------------------------------------------------------
# The reference's GPU backend (cuFFT FP64), for timing beside this project
# ---------------------------------------------------------------------------
REFGPU_SO = os.path.join(HERE, "_ref", "libgpe_refgpu.so")
_rglib = None


def rglib():
    global _rglib
    if _rglib is None:
        L = ctypes.CDLL(REFGPU_SO)
        L.gperefgpu_create.argtypes = [ctypes.POINTER(RefConfig)]
        L.gperefgpu_last_error.restype = ctypes.c_char_p
        L.gperefgpu_imag_steps.argtypes = [ctypes.c_long]
        L.gperefgpu_real_steps.argtypes = [ctypes.c_long, ctypes.c_long]
        L.gperefgpu_change_potential.argtypes = [ctypes.c_char_p]
        L.gperefgpu_export_psi.argtypes = [_dp]
        L.gperefgpu_energy.argtypes = [_dp]
        _rglib = L
    return _rglib


class RefGpuSolver:
    """The reference's own GpuGrossPitaevskiSolver (its CUDA kernels and cuFFT
    FP64), driven through its base-class iterations.  Needs a GPU."""

    def __init__(self, cfg: dict):
        L = rglib()
        if L.gperefgpu_create(ctypes.byref(ref_config(cfg))) != 0:
            raise RuntimeError(L.gperefgpu_last_error().decode())
        self.n = cfg["nx"] * cfg["ny"] * cfg["nz"]

    def close(self):
        rglib().gperefgpu_destroy()

    def imag_steps(self, k: int):
        assert rglib().gperefgpu_imag_steps(k) == 0

    def real_steps(self, k: int, first_iter: int = 0):
        assert rglib().gperefgpu_real_steps(k, first_iter) == 0

    def change_potential(self, key: str):
        assert rglib().gperefgpu_change_potential(key.encode()) == 0

    def psi(self) -> np.ndarray:
        out = np.zeros(2 * self.n)
        rglib().gperefgpu_export_psi(_ptr(out))
        return out

    def energy(self) -> np.ndarray:
        out = np.zeros(6)
        rglib().gperefgpu_energy(_ptr(out))
        return out



# ---------------------------------------------------------------------------
# Speed of the FP64 FFTW-API shim beside numpy / scipy pocketfft
# ---------------------------------------------------------------------------
def shim_fft_seconds(shape=(256, 256, 64), threads: int = 1, reps: int = 3) -> float:
    """Seconds for one r2c + c2r pair of `shape` through the FP64 FFTW-API shim
    (the padded dipolar transform pair the reference runs every calc_fi3d,
    src/solver/fft_solvers/cpu/fftw_poisson_solver.cpp:51-96), best of `reps`."""
    import time

    L = ctypes.CDLL(ORACLE_SO)
    L.fftw_plan_dft_r2c_3d.restype = ctypes.c_void_p
    L.fftw_plan_dft_r2c_3d.argtypes = [ctypes.c_int] * 3 + [_dp, _dp, ctypes.c_uint]
    L.fftw_plan_dft_c2r_3d.restype = ctypes.c_void_p
    L.fftw_plan_dft_c2r_3d.argtypes = [ctypes.c_int] * 3 + [_dp, _dp, ctypes.c_uint]
    L.fftw_execute.argtypes = [ctypes.c_void_p]
    L.fftw_destroy_plan.argtypes = [ctypes.c_void_p]
    L.fftw_plan_with_nthreads.argtypes = [ctypes.c_int]
    L.fftw_plan_with_nthreads(threads)
    n0, n1, n2 = shape
    x = np.random.default_rng(0).standard_normal(n0 * n1 * n2)
    spec = np.zeros(2 * n0 * n1 * (n2 // 2 + 1))
    back = np.zeros_like(x)
    fwd = L.fftw_plan_dft_r2c_3d(n0, n1, n2, _ptr(x), _ptr(spec), 0)
    inv = L.fftw_plan_dft_c2r_3d(n0, n1, n2, _ptr(spec), _ptr(back), 0)
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        L.fftw_execute(fwd)
        L.fftw_execute(inv)
        best = min(best, time.perf_counter() - t0)
    L.fftw_destroy_plan(fwd)
    L.fftw_destroy_plan(inv)
    return best


def fft_backend_check(shape=(256, 256, 64), threads: int = 1, reps: int = 3) -> dict:
    """The shim's r2c + c2r time for `shape` beside numpy's pocketfft (one
    thread) and scipy's pocketfft with `threads` workers, FP64, same host: how
    the CPU baseline's FFT compares with a production FFT library."""
    import time

    x = np.random.default_rng(0).standard_normal(shape)

    def best(fn):
        t = float("inf")
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            t = min(t, time.perf_counter() - t0)
        return t

    out = {"shape": list(shape), "threads": threads,
           "shim_r2c_c2r_s": shim_fft_seconds(shape, threads, reps),
           "shim_r2c_c2r_s_1_thread": shim_fft_seconds(shape, 1, reps),
           "numpy_pocketfft_r2c_c2r_s_1_thread": best(lambda: np.fft.irfftn(np.fft.rfftn(x), s=shape))}
    try:
        import scipy.fft as sf

        out["scipy_pocketfft_r2c_c2r_s"] = best(lambda: sf.irfftn(sf.rfftn(x, workers=threads), s=shape,
                                                                  workers=threads))
    except ImportError:
        pass
    return out
