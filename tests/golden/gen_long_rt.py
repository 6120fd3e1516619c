"""Generates tests/golden/readme_fs_long_rt.npz: the reference's own FP64 run of
the README full simulation at 128 x 128 x 32, for the long-run accuracy test.

Workload (the reference README's gpe_params.json at 128 x 128 x 32): dx = dy =
120 nm, dz = 600 nm, Dy-164 (163.929 Da), n_atoms = 2e4, edd = 1.5, MEXICAN
potential with dd = 1500 nm, MULTIPLE_GAUSS with 2 maxima; 1000 imaginary-time
iterations, then the potential switches to MEXICAN_FREE (the FS strategy,
src/manager/sim_manager.cpp:78-80) and 10000 real-time split-step iterations
(src/solver/solver.cpp:72-112).

The run is the reference's own CpuGrossPitaevskiSolver and FFTW solvers,
compiled unmodified by oracle/Makefile into oracle/_ref/libgpe_ref.so (with the
FP64 FFTW-API shim, FFTW3 being absent from this image).  It takes about half an
hour on 8 host threads.

Saved (psi rounded to complex64 to keep the file small: the rounding is ~3e-8
relative, far below the 1e-5 bound the test holds the GPU path to):
  psi_it       psi after the 1000 imaginary-time iterations
  psi_rt_<k>   psi after k real-time iterations, k in RT_CHECKPOINTS
  energy_it, energy_rt_<k>   the six calc_energy terms (FP64)
  norm_it, norm_rt_<k>       calc_norm (FP64)

Run from the repository root (needs the reference sources to build the harness):

    make -C oracle ref && python tests/golden/gen_long_rt.py
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "readme_fs_long_rt.npz")
IT_STEPS = 1000
RT_CHECKPOINTS = (1000, 2000, 5000, 10000)


def config() -> dict:
    return O.default_config(nx=128, ny=128, nz=32, init_strategy="MULTIPLE_GAUSS", initial_maximas=2,
                            pote_strategy="MEXICAN", iter_imag=IT_STEPS, iter_real=RT_CHECKPOINTS[-1],
                            fftw_n_threads=os.cpu_count() or 4)


def c64(psi_flat: np.ndarray) -> np.ndarray:
    return psi_flat.view(np.complex128).astype(np.complex64)


def main() -> None:
    O.build(ref=True)
    cfg = config()
    r = O.RefSolver(cfg)
    out = {"meta_grid": np.array([cfg["nx"], cfg["ny"], cfg["nz"]]),
           "meta_steps": np.array([IT_STEPS] + list(RT_CHECKPOINTS))}
    t0 = time.time()
    r.imag_steps(IT_STEPS)
    out["psi_it"] = c64(r.psi())
    out["energy_it"] = r.energy()
    out["norm_it"] = np.array([r.norm()])
    print(f"IT done ({time.time() - t0:.0f} s)", flush=True)
    r.change_potential("MEXICAN_FREE")
    done = 0
    for k in RT_CHECKPOINTS:
        r.real_steps(k - done, done)
        done = k
        out[f"psi_rt_{k}"] = c64(r.psi())
        out[f"energy_rt_{k}"] = r.energy()
        out[f"norm_rt_{k}"] = np.array([r.norm()])
        print(f"RT {k} done ({time.time() - t0:.0f} s)", flush=True)
    r.close()
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
