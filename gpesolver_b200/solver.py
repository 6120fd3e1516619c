"""The B200 backend behind GPESolver's solver interface, for Python callers.

``B200GrossPitaevskiSolver`` exposes the members of the reference's
AbstractGrossPitaevskiSolver (src/solver/solver.hpp:17-72) with the same names
and meaning -- load_buffer / load_pote / export_data, the pure virtuals
(calc_fi3d, imag_iter_linear_step, imag_iter_nonlinear_step, calc_norm,
normalize, real_fft_potential_half_step, real_fft_kinetic_step, calc_energy),
the iteration bodies imag_time_iter / real_time_iter and the solve() driver --
on top of the C ABI in include/gpe_b200.h.  Errors raise GpeError (a
RuntimeError), where the reference throws std::runtime_error.

Every numerical operation runs in libgpe_b200.so on the GPU; this module only
moves host buffers and sequences calls.
"""
from __future__ import annotations

import ctypes
import dataclasses
from collections import namedtuple
from typing import Callable, Optional

import numpy as np

from . import capi
from .params import PhysicalParameters

BECEnergies = namedtuple("BECEnergies", "e_kin e_pot e_int e_ext e_bmf e_total")

PRECISIONS = {"c64": capi.GPE_PREC_C64, "c128": capi.GPE_PREC_C128}


def make_gpe_params(p: PhysicalParameters, precision: str = "c64", device: int = 0,
                    schedule: str = "auto") -> capi.gpe_params:
    """Fill the C ABI's gpe_params from the PhysicalParameters fields."""
    g = capi.gpe_params()
    g.nx, g.ny, g.nz = p.nx, p.ny, p.nz
    g.dx, g.dy, g.dz = p.dx, p.dy, p.dz
    g.m, g.n_atoms = p.m, p.n_atoms
    g.add, g.cdd, g.ggp11, g.gamma, g.w_15 = p.add, p.cdd, p.ggp11, p.gamma, p.w_15
    g.real_time_dt, g.imag_time_dt = p.real_time_dt, p.imag_time_dt
    g.const_edd = 1 if p.const_edd else 0
    g.edd, g.edd_start, g.edd_stop = p.edd, p.edd_start, p.edd_stop
    g.iter_real = max(int(p.iter_real), 1)
    g.precision = PRECISIONS[precision]
    g.device = device
    g.schedule = {"auto": capi.GPE_SCHED_AUTO, "split": capi.GPE_SCHED_SPLIT}[schedule]
    return g


def make_init_params(p: PhysicalParameters) -> capi.gpe_init_params:
    """gpe_init_params: the fields the potentials and initialisers read."""
    g = capi.gpe_init_params()
    g.omega_x, g.omega_y, g.omega_z = p.omega_x, p.omega_y, p.omega_z
    g.aa, g.b, g.dd = p.aa, p.b, p.dd
    g.n_gauss_max = p.n_gauss_max
    g.bec_droplets_x, g.bec_droplets_y, g.bec_droplets_z = p.bec_droplets_x, p.bec_droplets_y, p.bec_droplets_z
    return g


class B200GrossPitaevskiSolver:
    @classmethod
    def _borrow(cls, handle: ctypes.c_void_p, params: PhysicalParameters, precision: str = "c64"):
        """A view of a handle owned elsewhere (a batch member): close() leaves it alone."""
        self = cls.__new__(cls)
        self.params = dataclasses.replace(params)
        self.precision = precision
        self._L = capi.lib()
        self._gp = None
        self._h = handle
        self._borrowed = True
        self.n = params.n
        self.xnorma = 0.0
        self.enes = []
        self.ene = None
        return self

    def __init__(self, params: PhysicalParameters, precision: str = "c64", device: int = 0,
                 schedule: str = "auto"):
        # the solver owns its parameters (real_steps advances edd on this copy,
        # as calc_evolution advances the reference's singleton)
        self.params = dataclasses.replace(params)
        self.precision = precision
        self._L = capi.lib()
        self._gp = make_gpe_params(params, precision, device, schedule)
        h = ctypes.c_void_p()
        capi.check(self._L.gpe_create(ctypes.byref(self._gp), ctypes.byref(h)))
        self._h = h
        self.n = params.n
        self.xnorma = 0.0
        self.enes: list[BECEnergies] = []
        self.ene: Optional[BECEnergies] = None

    # -- lifecycle ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_borrowed", False):
            self._h = None
            return
        if getattr(self, "_h", None):
            self._L.gpe_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_ptr: int) -> None:
        capi.check(self._L.gpe_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def synchronize(self) -> None:
        capi.check(self._L.gpe_synchronize(self._h))

    def launch_count(self) -> int:
        c = ctypes.c_longlong()
        capi.check(self._L.gpe_launch_count(self._h, ctypes.byref(c)))
        return c.value

    def x_tiles(self) -> tuple[int, int]:
        """Lines per CTA of the kinetic and dipolar x pencils picked by the
        autotuner for this grid (GPE_X_TILES="k,d" fixes them)."""
        k, d = ctypes.c_int(), ctypes.c_int()
        capi.check(self._L.gpe_x_tiles(self._h, ctypes.byref(k), ctypes.byref(d)))
        return k.value, d.value

    def plane_kernel(self) -> str:
        """The plane kernel of the middle real-time iterations ("k5_yz_pair",
        "k4_yz", or "" on grids without one)."""
        return self._L.gpe_plane_kernel_name(self._h).decode()

    # -- data in / out (solver.cpp:118-131, gpu_solver.cpp:136-155) -------
    def load_buffer(self, psi) -> None:
        a = _as_c128_flat(psi, self.n)
        capi.check(self._L.gpe_load_psi(self._h, capi.dptr(a), self.n))

    def import_data(self, psi) -> None:
        """import_data: psi and psii take the values as given (no normalisation)."""
        a = _as_c128_flat(psi, self.n)
        capi.check(self._L.gpe_import_psi(self._h, capi.dptr(a), self.n))

    def load_pote(self, V) -> None:
        a = np.ascontiguousarray(np.asarray(V, dtype=np.float64).reshape(-1))
        if a.size != self.n:
            raise capi.GpeError(capi.GPE_ERR_ARG, "bad potential import")
        capi.check(self._L.gpe_load_potential(self._h, capi.dptr(a), self.n))

    def init_pote(self, key: Optional[str] = None) -> None:
        """load_pote(init_pote()) with V computed on the device (FP64,
        bit-identical to the host potential)."""
        key = key or self.params.pote_key
        ip = make_init_params(self.params)
        capi.check(self._L.gpe_init_potential(self._h, capi.POTENTIAL_IDS[key], ctypes.byref(ip)))

    def init_buffer(self, strategy: Optional[str] = None) -> None:
        """load_buffer(psi_0) with psi_0 computed on the device from the
        initialisation strategy (COS, GAUSS, MULTIPLE_GAUSS, SETUP_GAUSS)."""
        strategy = strategy or self.params.init_strategy
        if strategy not in capi.INIT_IDS:
            raise capi.GpeError(capi.GPE_ERR_ARG, f"no device initialiser for {strategy}")
        ip = make_init_params(self.params)
        capi.check(self._L.gpe_init_psi(self._h, capi.INIT_IDS[strategy], ctypes.byref(ip)))

    def export_pote(self) -> np.ndarray:
        """The potential the solver holds (buf_data->pote), FP64."""
        out = np.zeros(self.n)
        capi.check(self._L.gpe_export_potential(self._h, capi.dptr(out), self.n))
        return out.reshape(self.params.shape)

    def export_data(self) -> np.ndarray:
        """psi as complex128 of shape (nx, ny, nz)."""
        out = np.zeros(2 * self.n)
        capi.check(self._L.gpe_export_psi(self._h, capi.dptr(out), self.n))
        return out.view(np.complex128).reshape(self.params.shape)

    def export_async(self, buf: np.ndarray) -> None:
        """Start copying psi (complex128, flat float64 view of 2n values) into
        `buf` (pinned host memory) without waiting; export_wait() completes it."""
        if buf.dtype != np.float64 or buf.size != 2 * self.n or not buf.flags["C_CONTIGUOUS"]:
            raise capi.GpeError(capi.GPE_ERR_ARG, "export buffer must be 2n contiguous float64")
        capi.check(self._L.gpe_export_psi_async(self._h, capi.dptr(buf), self.n))

    def export_wait(self) -> None:
        capi.check(self._L.gpe_export_wait(self._h))

    def export_fi3d(self) -> np.ndarray:
        out = np.zeros(self.n)
        capi.check(self._L.gpe_export_fi3d(self._h, capi.dptr(out), self.n))
        return out.reshape(self.params.shape)

    def load_fi3d(self, fi3d) -> None:
        """Sets the dipolar field that the next real-time iteration's first
        potential half step uses (a resumed run: the checkpoint's field)."""
        a = np.ascontiguousarray(np.asarray(fi3d, dtype=np.float64).reshape(-1))
        if a.size != self.n:
            raise capi.GpeError(capi.GPE_ERR_ARG, "bad fi3d import")
        capi.check(self._L.gpe_load_fi3d(self._h, capi.dptr(a), self.n))

    # -- the pure virtuals (solver.hpp:55-66) -------------------------------
    def calc_fi3d(self) -> None:
        capi.check(self._L.gpe_calc_fi3d(self._h))

    def imag_iter_linear_step(self) -> None:
        capi.check(self._L.gpe_imag_iter_linear_step(self._h))

    def imag_iter_nonlinear_step(self) -> None:
        capi.check(self._L.gpe_imag_iter_nonlinear_step(self._h))

    def calc_norm(self, to_host: bool = True) -> float:
        """xnorma; with to_host=False the reduction stays on the device."""
        if not to_host:
            capi.check(self._L.gpe_calc_norm(self._h, None))
            return self.xnorma
        x = ctypes.c_double()
        capi.check(self._L.gpe_calc_norm(self._h, ctypes.byref(x)))
        self.xnorma = x.value
        return self.xnorma

    def normalize(self) -> None:
        capi.check(self._L.gpe_normalize(self._h))

    def real_fft_potential_half_step(self) -> None:
        capi.check(self._L.gpe_real_fft_potential_half_step(self._h))

    def real_fft_kinetic_step(self) -> None:
        capi.check(self._L.gpe_real_fft_kinetic_step(self._h))

    def calc_energy(self) -> BECEnergies:
        out = np.zeros(6)
        capi.check(self._L.gpe_calc_energy(self._h, capi.dptr(out)))
        self.ene = BECEnergies(*out.tolist())
        self.enes.append(self.ene)
        return self.ene

    def set_coeffs(self, ggp11: float, gamma: float) -> None:
        capi.check(self._L.gpe_set_coeffs(self._h, ggp11, gamma))

    # -- iteration bodies (solver.cpp:99-112) -------------------------------
    def imag_time_iter(self) -> None:
        """One iteration through the individual virtuals (one call per virtual)."""
        self.calc_fi3d()
        self.imag_iter_linear_step()
        self.imag_iter_nonlinear_step()
        self.calc_norm(to_host=False)
        self.normalize()

    def real_time_iter(self) -> None:
        self.real_fft_potential_half_step()
        self.calc_fi3d()
        self.real_fft_kinetic_step()
        self.real_fft_potential_half_step()

    # -- fused iterations (CUDA-graph replays) ------------------------------
    def imag_steps(self, k: int) -> None:
        capi.check(self._L.gpe_imag_steps(self._h, int(k)))

    def imag_steps_energies(self, k: int, checks: int) -> np.ndarray:
        """`checks` rounds of k imaginary-time iterations; the total energy after
        each round (one host synchronisation for all of them)."""
        out = np.zeros(checks)
        capi.check(self._L.gpe_imag_steps_energies(self._h, int(k), int(checks), capi.dptr(out)))
        return out

    def real_steps(self, k: int, first_iter: int = 0) -> None:
        capi.check(self._L.gpe_real_steps(self._h, int(k), int(first_iter)))
        if not self.params.const_edd and k > 0:
            self.params.update_edd(first_iter + k - 1)

    # -- driver (AbstractGrossPitaevskiSolver::solve, solver.cpp:25-97) -----
    def solve(self, checkpoint: Optional[Callable[[str, int, np.ndarray], None]] = None,
              request_free_potential: Optional[Callable[[], np.ndarray]] = None,
              checkpointer=None, resume: Optional[dict] = None) -> None:
        """Runs the configured strategy with the reference's cadence
        (solver.cpp:25-97): energies and checkpoints after iterations 0, 100,
        200, ... (IT) and 0, 1000, ... (RT); the FS strategy switches to the free
        potential in between.

        checkpoint(phase, iteration, psi): called with psi on the host at every
        checkpoint (synchronous, as the reference's save_checkpoint).
        checkpointer: a checkpoint.Checkpointer instead -- the copy of psi
        overlaps the next iterations and the file is written in the background.
        resume: {"phase": "imag" | "real", "iteration": it} of a checkpoint whose
        psi has been loaded (load_buffer): the run continues after it, the edd
        ramp included.  A real-time record with "fi3d_file" (Checkpointer
        writes one) also restores the dipolar field the next iteration's first
        half step uses, so the resumed run repeats the uninterrupted one."""
        p = self.params

        def at_checkpoint(phase, it):
            if checkpointer is not None:
                checkpointer.checkpoint(phase, it)
            elif checkpoint:
                checkpoint(phase, it, self.export_data())
            self.calc_energy()

        def imag_phase(done):
            total = p.iter_imag + 1
            while done < total:
                k = 1 if done == 0 else min(100 - (done - 1) % 100, total - done)
                self.imag_steps(k)
                done += k
                it = done - 1
                if it % 100 == 0:
                    at_checkpoint("imag", it)

        def real_phase(done):
            total = p.iter_real + 1
            while done < total:
                k = 1 if done == 0 else min(1000 - (done - 1) % 1000, total - done)
                self.real_steps(k, done)
                done += k
                it = done - 1
                if it % 1000 == 0:
                    at_checkpoint("real", it)

        phase0, start = "imag", 0
        if resume is not None:
            phase0, start = resume["phase"], int(resume["iteration"]) + 1
        if p.calc_strategy in ("IT", "FS") and phase0 == "imag":
            imag_phase(start)
            start = 0
        if p.calc_strategy == "FS" and phase0 == "imag":
            # SimulationManager::request_free_potential (sim_manager.cpp:78-80):
            # the caller's potential, else MEXICAN_FREE computed on the device
            if request_free_potential is not None:
                self.load_pote(request_free_potential())
            else:
                self.init_pote("MEXICAN_FREE")
        if p.calc_strategy == "FS" and phase0 == "real":
            # resumed after the switch: the free potential again
            if request_free_potential is not None:
                self.load_pote(request_free_potential())
            else:
                self.init_pote("MEXICAN_FREE")
        if phase0 == "real" and resume.get("fi3d_file"):
            self.load_fi3d(np.fromfile(resume["fi3d_file"], dtype=np.float64))
        if p.calc_strategy in ("RT", "FS"):
            real_phase(start)
        if checkpointer is not None:
            checkpointer.close()


def _as_c128_flat(psi, n: int) -> np.ndarray:
    a = np.asarray(psi)
    if np.iscomplexobj(a):
        a = np.ascontiguousarray(a.reshape(-1), dtype=np.complex128).view(np.float64)
    else:
        a = np.ascontiguousarray(a.reshape(-1), dtype=np.float64)
    if a.size != 2 * n:
        raise capi.GpeError(capi.GPE_ERR_ARG, "bad wavefunction import")
    return a
