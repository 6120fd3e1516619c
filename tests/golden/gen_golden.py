"""Generates the golden fixtures in tests/golden/ from the reference itself.

The reference publishes no numerical fixtures (its tests cover only GpuArray and
the JSON loader), so the golden vectors are outputs of the reference's own CPU
solver (CpuGrossPitaevskiSolver + FFTW solvers + DataInitializer + parameters),
compiled unmodified from its sources by oracle/Makefile into
oracle/_ref/libgpe_ref.so and driven through oracle/ref_harness.cpp.

Run from the repository root (needs the reference sources to build the harness):

    make -C oracle ref && python tests/golden/gen_golden.py [case ...]
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# name -> (config overrides, IT steps, optional potential switch, RT steps, RT first iter)
CASES = {
    "it_harmonic_gauss": (dict(nx=16, ny=12, nz=8, init_strategy="GAUSS", pote_strategy="HARMONIC"),
                          4, None, 3, 0),
    "fs_mexican_multigauss": (dict(nx=16, ny=16, nz=8, init_strategy="MULTIPLE_GAUSS",
                                   initial_maximas=2, pote_strategy="MEXICAN"),
                              5, "MEXICAN_FREE", 4, 0),
    "rt_free_setup_ramp": (dict(nx=12, ny=10, nz=6, init_strategy="SETUP_GAUSS", bec_droplets_x=2,
                                bec_droplets_y=2, bec_droplets_z=1, pote_strategy="FREE", edd=None,
                                edd_start=1.40, edd_stop=1.60, iter_real=10),
                           0, None, 5, 3),
    "it_cylindrical_cos": (dict(nx=10, ny=12, nz=8, init_strategy="COS", pote_strategy="CYLINDRICAL"),
                           3, None, 2, 0),
    "mixed_radix_harmonic": (dict(nx=12, ny=12, nz=6, init_strategy="GAUSS", pote_strategy="HARMONIC",
                                  omega_z=240.0),
                             2, None, 2, 0),
    "mexican_asym_three": (dict(nx=20, ny=16, nz=10, init_strategy="MULTIPLE_GAUSS", initial_maximas=3,
                                pote_strategy="MEXICAN_ASYMETRIC", dd=900.0),
                           3, "MEXICAN_ASYMETRIC_FREE", 2, 0),
    # Well-conditioned runs: on the cases above (the README's couplings on small
    # boxes) the imaginary-time state is a collapsing droplet whose real-time
    # phase reaches 5-80 rad per half step, and the FP64 reference itself turns
    # a 1e-7 change of its start into a much larger one within a few steps.  On
    # these (dilute states, contact-dominated or a loose trap) the phase stays
    # near 5e-3 rad and a 1e-7 change of the start stays 1e-7, so a complex64
    # result can be held to the per-call bound over tens of iterations.
    "well_harmonic_ramp": (dict(nx=32, ny=32, nz=16, init_strategy="GAUSS", pote_strategy="HARMONIC",
                                dx=200.0, dy=200.0, dz=800.0, edd=None, edd_start=0.70, edd_stop=0.80,
                                iter_real=200),
                           30, None, 60, 0),
    "well_mexican_free": (dict(nx=32, ny=32, nz=16, init_strategy="MULTIPLE_GAUSS", initial_maximas=2,
                               pote_strategy="MEXICAN", dx=250.0, dy=250.0, dz=800.0, n_atoms=5e3, edd=0.9),
                          20, "MEXICAN_FREE", 40, 0),
    "well_cylindrical_cos": (dict(nx=24, ny=20, nz=12, init_strategy="COS", pote_strategy="CYLINDRICAL",
                                  dx=250.0, dy=250.0, dz=800.0, n_atoms=5e3, edd=0.8),
                             10, None, 30, 0),
}

# The cases whose real-time phase a complex64 run can follow to the per-call bound.
WELL_CONDITIONED = ("well_harmonic_ramp", "well_mexican_free", "well_cylindrical_cos")


def config(name: str) -> dict:
    return O.default_config(**CASES[name][0])


def generate(name: str) -> dict:
    over, n_it, switch, n_rt, first = CASES[name]
    cfg = config(name)
    r = O.RefSolver(cfg)
    out = {"psi0": r.psi(), "pote0": r.pote(), "coef": np.array(list(r.coefficients().values()))}
    # single operations from the loaded state (copies of the solver are not
    # possible, so each op is applied in sequence)
    r.op("calc_fi3d")
    out["op_fi3d"] = r.fi3d()
    r.op("real_fft_potential_half_step")
    out["op_pot_half"] = r.psi()
    r.op("real_fft_kinetic_step")
    out["op_kinetic"] = r.psi()
    out["op_energy"] = r.energy()
    r.close()
    # full iterations from a fresh start
    r = O.RefSolver(cfg)
    if n_it:
        r.imag_steps(n_it)
        out["it_psi"] = r.psi()
        out["it_fi3d"] = r.fi3d()
        out["it_norm"] = np.array([r.norm()])
        out["it_energy"] = r.energy()
    if switch:
        r.change_potential(switch)
        out["pote1"] = r.pote()
    r.real_steps(n_rt, first)
    out["rt_psi"] = r.psi()
    out["rt_fi3d"] = r.fi3d()
    out["rt_energy"] = r.energy()
    r.close()
    out["meta"] = np.array([n_it, n_rt, first])
    return out


def main(names=None) -> None:
    O.build(ref=True)
    for name in names or CASES:
        data = generate(name)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **data)
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1:] or None)
