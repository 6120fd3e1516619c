"""Learned warm start for imaginary-time ground states.

``WarmStartNet`` wraps the network of include/gpe_b200.h (gpe_warm_*): from
the physical parameters of a solve (edd, n_atoms, omega_r, omega_z) it
predicts the ground-state amplitude |psi_0| on the solver grid, and
``predict_into`` loads that amplitude into a solver as its initial state
(load_buffer semantics, without a host round trip).  Imaginary time then
refines it to the same energy tolerance as a Gaussian start; plain
Gaussian-start imaginary time remains the fallback and the yardstick for the
prediction's error.

The training data are ground states that the plain method produces
(``ground_states``, batched with B200Batch); ``train`` runs Adam on them with
the network's own CUDA forward and backward kernels; ``time_to_ground_state``
measures iterations and seconds to a relative energy change below a tolerance,
with the energy checked every K iterations.

Device buffers (the training targets, the predicted amplitudes) are torch
tensors: torch is only the allocator here, every operation on them runs in
libgpe_b200.so.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import capi
from .batch import B200Batch
from .params import PhysicalParameters
from .solver import B200GrossPitaevskiSolver


@dataclass
class WarmConfig:
    nx: int = 128
    ny: int = 128
    nz: int = 32
    levels: int = 4
    channels: tuple = (32, 32, 16, 8, 8)
    hidden: int = 256
    n_inputs: int = 4
    max_batch: int = 8
    # normalisation of the inputs (centre, half range): edd, n_atoms, omega_r [Hz], omega_z / omega_r
    centre: tuple = (1.5, 3.0e4, 60.0, 2.5)
    half_range: tuple = (0.3, 2.0e4, 20.0, 1.5)


def hz(omega_au: float) -> float:
    """Frequency in Hz of an angular frequency in atomic units (UnitConverter)."""
    from .params import freq_hz_to_au

    return omega_au / freq_hz_to_au(1.0)


def features(p: PhysicalParameters, cfg: WarmConfig) -> np.ndarray:
    """Normalised network inputs of a solve: edd, n_atoms, omega_r, omega_z/omega_r."""
    wr = hz(p.omega_x)
    raw = (p.edd, p.n_atoms, wr, hz(p.omega_z) / wr)
    return np.array([(v - c) / h for v, c, h in zip(raw, cfg.centre, cfg.half_range)], dtype=np.float32)


def target_scale(p: PhysicalParameters) -> float:
    """Amplitudes are trained as |psi| sqrt(dV N): mean square 1 on every grid."""
    return math.sqrt(p.dx * p.dy * p.dz * p.n)


class WarmStartNet:
    def __init__(self, cfg: WarmConfig = WarmConfig(), device: int = 0, seed: int = 0):
        self.cfg = cfg
        self._L = capi.lib()
        c = capi.gpe_warm_config()
        c.nx, c.ny, c.nz, c.levels = cfg.nx, cfg.ny, cfg.nz, cfg.levels
        for s, ch in enumerate(cfg.channels):
            c.channels[s] = ch
        c.hidden, c.n_inputs, c.max_batch = cfg.hidden, cfg.n_inputs, cfg.max_batch
        h = ctypes.c_void_p()
        capi.check(self._L.gpe_warm_create(ctypes.byref(c), device, ctypes.byref(h)))
        self._h = h
        n = ctypes.c_size_t()
        capi.check(self._L.gpe_warm_num_weights(self._h, ctypes.byref(n)))
        self.n_weights = n.value
        capi.check(self._L.gpe_warm_init_weights(self._h, seed))
        self.device = device
        self._amp = None

    @property
    def n_voxels(self) -> int:
        return self.cfg.nx * self.cfg.ny * self.cfg.nz

    def close(self):
        if getattr(self, "_h", None):
            self._L.gpe_warm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- weights ------------------------------------------------------------
    def get_weights(self) -> np.ndarray:
        w = np.zeros(self.n_weights, dtype=np.float32)
        capi.check(self._L.gpe_warm_get_weights(self._h, w.ctypes.data, w.size))
        return w

    def set_weights(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, dtype=np.float32)
        capi.check(self._L.gpe_warm_set_weights(self._h, w.ctypes.data, w.size))

    def save(self, path: str) -> None:
        c = self.cfg
        np.savez(path, weights=self.get_weights().astype(np.float32), nx=c.nx, ny=c.ny, nz=c.nz,
                 levels=c.levels, channels=np.array(c.channels), hidden=c.hidden, n_inputs=c.n_inputs,
                 centre=np.array(c.centre), half_range=np.array(c.half_range))

    @classmethod
    def pretrained(cls, device: int = 0) -> "WarmStartNet":
        """The network trained at 128x128x32 on 2000 sweep ground states
        (bench.py --workload warmstart), stored as BF16 weights."""
        import os

        return cls.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                                     "warmstart_128x128x32.npz"), device)

    @classmethod
    def load(cls, path: str, device: int = 0, max_batch: int = 8) -> "WarmStartNet":
        with np.load(path) as f:
            cfg = WarmConfig(nx=int(f["nx"]), ny=int(f["ny"]), nz=int(f["nz"]), levels=int(f["levels"]),
                             channels=tuple(int(v) for v in f["channels"]), hidden=int(f["hidden"]),
                             n_inputs=int(f["n_inputs"]), max_batch=max_batch,
                             centre=tuple(float(v) for v in f["centre"]),
                             half_range=tuple(float(v) for v in f["half_range"]))
            net = cls(cfg, device)
            if "weights" in f.files:
                net.set_weights(f["weights"])
            else:  # BF16 bit patterns
                net.set_weights((f["weights_bf16"].astype(np.uint32) << 16).view(np.float32))
        return net

    # -- forward / training ---------------------------------------------------
    def forward(self, inputs: np.ndarray, out_ptr: int) -> None:
        x = np.ascontiguousarray(inputs, dtype=np.float32)
        capi.check(self._L.gpe_warm_forward(self._h, x.ctypes.data, x.shape[0], ctypes.c_void_p(out_ptr)))

    def gradients(self, inputs: np.ndarray, targets_ptr: int) -> tuple[float, np.ndarray]:
        x = np.ascontiguousarray(inputs, dtype=np.float32)
        g = np.zeros(self.n_weights, dtype=np.float32)
        loss = ctypes.c_double()
        capi.check(self._L.gpe_warm_gradients(self._h, x.ctypes.data, ctypes.c_void_p(targets_ptr), x.shape[0],
                                              g.ctypes.data, ctypes.byref(loss)))
        return loss.value, g

    def train_step(self, inputs: np.ndarray, targets_ptr: int, lr: float) -> float:
        x = np.ascontiguousarray(inputs, dtype=np.float32)
        loss = ctypes.c_double()
        capi.check(self._L.gpe_warm_train_step(self._h, x.ctypes.data, ctypes.c_void_p(targets_ptr), x.shape[0],
                                               ctypes.c_float(lr), ctypes.byref(loss)))
        return loss.value

    def predict_into(self, solver: B200GrossPitaevskiSolver) -> None:
        """Initial state of `solver` = the predicted amplitude for its parameters."""
        import torch

        if self._amp is None:
            self._amp = torch.empty(self.n_voxels, dtype=torch.float32, device=f"cuda:{self.device}")
        self.forward(features(solver.params, self.cfg)[None], self._amp.data_ptr())
        capi.check(self._L.gpe_load_amplitude_device(solver.handle, ctypes.c_void_p(self._amp.data_ptr()),
                                                     self.n_voxels))


def ground_states(params: Sequence[PhysicalParameters], iters: int, batch: int = 64, device: int = 0,
                  converge_tol: float | None = None, max_chunks: int = 8):
    """Amplitude targets (torch float32 on the device, one row per solve,
    scaled by target_scale) after imaginary time from each solve's Gaussian
    start, batched.  With converge_tol, every batch keeps stepping in chunks of
    `iters` iterations (at most max_chunks) until the total energy of every
    member changes by less than converge_tol (relative) over a chunk, so that
    the targets are ground states and not states still relaxing; without it,
    each member runs `iters` iterations.  Returns (targets, chunks run per
    batch)."""
    import torch

    n = params[0].n
    out = torch.empty((len(params), n), dtype=torch.float32, device=f"cuda:{device}")
    chunks = []
    for s in range(0, len(params), batch):
        chunk = params[s:s + batch]
        with B200Batch(chunk, device) as b:
            for m in b.members:
                m.init_pote()
                m.init_buffer("GAUSS")
            b.imag_steps(iters)
            done = 1
            if converge_tol is not None:
                e_prev = np.array([m.calc_energy().e_total for m in b.members])
                while done < max_chunks:
                    b.imag_steps(iters)
                    done += 1
                    e = np.array([m.calc_energy().e_total for m in b.members])
                    worst = float(np.max(np.abs(e - e_prev) / np.abs(e)))
                    e_prev = e
                    if worst < converge_tol:
                        break
            chunks.append(done)
            for r, m in enumerate(b.members):
                row = out[s + r]
                capi.check(capi.lib().gpe_export_amplitude_device(m.handle, ctypes.c_void_p(row.data_ptr()), n))
                row.mul_(target_scale(m.params))
    return out, chunks


def train(net: WarmStartNet, params: Sequence[PhysicalParameters], targets, epochs: int, batch: int,
          lr: float = 1e-3, lr_final: float = 1e-5, seed: int = 0, log=None) -> list[float]:
    """Adam over the training set with a cosine learning-rate schedule; returns
    the mean loss of every epoch."""
    X = np.stack([features(p, net.cfg) for p in params])
    rng = np.random.default_rng(seed)
    n = len(params)
    steps = epochs * max(1, n // batch)
    hist, step = [], 0
    for ep in range(epochs):
        order = rng.permutation(n)
        losses = []
        for s in range(0, n - batch + 1, batch):
            idx = order[s:s + batch]
            lr_t = lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * step / max(1, steps)))
            tb = targets[idx].contiguous()
            losses.append(net.train_step(X[idx], tb.data_ptr(), lr_t))
            step += 1
        hist.append(float(np.mean(losses)))
        if log:
            log(ep, hist[-1])
    return hist


def time_to_ground_state(solver: B200GrossPitaevskiSolver, tol: float = 1e-8, K: int = 10,
                         max_iters: int = 100000, checks_per_sync: int = 4) -> tuple[int, float, float]:
    """Imaginary-time iterations until the relative change of the total energy
    between two checks K iterations apart is below tol, the wall seconds until
    the host knows it, and the energy.  Energies of `checks_per_sync` checks are
    gathered on the device between host synchronisations (the iterations run
    past the converged check until the end of its round are not counted)."""
    t0 = time.perf_counter()
    e_prev = solver.calc_energy().e_total
    it = 0
    while it < max_iters:
        es = solver.imag_steps_energies(K, checks_per_sync)
        for e in es:
            it += K
            if abs(e - e_prev) < tol * abs(e):
                return it, time.perf_counter() - t0, float(e)
            e_prev = e
    return it, time.perf_counter() - t0, float(e_prev)
