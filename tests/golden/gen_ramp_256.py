"""Generates tests/golden/ramp_256x256x64_rt.npz: the reference's own FP64 run of
the precision study's first real-time iterations at 256 x 256 x 64, for
tests/test_ramp_accuracy.py.

Workload (the precision study): nx = ny = 256, nz = 64, dx = dy = 120 nm,
dz = 600 nm, Dy-164 (163.929 Da), n_atoms = 2e4, FREE potential (z-bound only),
SETUP_GAUSS with 3 x 3 x 2 droplets, edd ramped linearly from edd_start = 1.40
to edd_stop = 1.60 over iter_real = 20000 iterations (update_edd before each
iteration, src/solver/solver.cpp:75-77 and src/parameters/parameters.cpp:53),
real-time split-step iterations from the initial state
(src/solver/solver.cpp:107-112).  The fixture holds the first
RT_CHECKPOINTS[-1] iterations of the ramp.

The run is the reference's own CpuGrossPitaevskiSolver and FFTW solvers,
compiled unmodified by oracle/Makefile into oracle/_ref/libgpe_ref.so (with the
FP64 FFTW-API shim, FFTW3 being absent from this image): about 3 s per
iteration on 8 host threads.

psi itself (4.2 M points) would make a 34 MB file, so the fixture keeps, at
each checkpoint, two planes of it rounded to complex64 (~3e-8 relative, far
below the bounds the test holds the GPU path to) and the FP64 scalars:
  meta_grid, meta_steps      grid and checkpoints
  xy_<k>   psi[:, :, nz/2] after k real-time iterations (nx x ny)
  xz_<k>   psi[:, ny/2, :] after k real-time iterations (nx x nz)
  energy_<k>, norm_<k>       the six calc_energy terms and calc_norm (FP64)
  xy_0, xz_0, energy_0, norm_0   the same for the initial state

Run from the repository root (needs the reference sources to build the harness):

    make -C oracle ref && python tests/golden/gen_ramp_256.py
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ramp_256x256x64_rt.npz")
RT_CHECKPOINTS = (250, 500, 1000)


def config() -> dict:
    return O.default_config(nx=256, ny=256, nz=64, pote_strategy="FREE", init_strategy="SETUP_GAUSS",
                            bec_droplets_x=3, bec_droplets_y=3, bec_droplets_z=2, edd=None,
                            edd_start=1.40, edd_stop=1.60, iter_imag=0, iter_real=20000,
                            fftw_n_threads=os.cpu_count() or 4)


def planes(psi_flat: np.ndarray, shape) -> tuple[np.ndarray, np.ndarray]:
    nx, ny, nz = shape
    p = psi_flat.view(np.complex128).reshape(nx, ny, nz)
    return (np.ascontiguousarray(p[:, :, nz // 2]).astype(np.complex64),
            np.ascontiguousarray(p[:, ny // 2, :]).astype(np.complex64))


def main() -> None:
    O.build(ref=True)
    cfg = config()
    shape = (cfg["nx"], cfg["ny"], cfg["nz"])
    r = O.RefSolver(cfg)
    out = {"meta_grid": np.array(shape), "meta_steps": np.array(RT_CHECKPOINTS)}

    def save(k):
        out[f"xy_{k}"], out[f"xz_{k}"] = planes(r.psi(), shape)
        out[f"energy_{k}"] = r.energy()
        out[f"norm_{k}"] = np.array([r.norm()])

    save(0)
    t0 = time.time()
    done = 0
    for k in RT_CHECKPOINTS:
        r.real_steps(k - done, done)
        done = k
        save(k)
        np.savez_compressed(OUT, **out)  # partial results survive an interrupted run
        print(f"RT {k} done ({time.time() - t0:.0f} s)", flush=True)
    r.close()
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
