"""Known-answer tests that pin the physics of the solver path independently of
the oracle (GPU):

1. linear limit: with the contact, LHY and dipolar couplings switched off,
   imaginary time converges to the lowest eigenvalue of the finite-difference
   Hamiltonian the reference discretises (7-point Laplacian, Dirichlet walls,
   the HARMONIC trap as the initializer builds it), computed here from three
   1D tridiagonal eigenproblems;
2. real time is time-reversible and norm-conserving: the split step with the
   contact and LHY phases (solver.cpp:107-112) run for k steps with dt and
   then k steps with -dt returns to its start (the dipolar potential is off:
   the reference's second half step uses the phi of the first, which breaks
   exact reversal);
3. a plane wave of the periodic box evolves by the exact phase
   exp(-i t k^2 / 2m) under the split step (no potential, no coupling).

Both the fused schedule (plane kernel, kinetic increment form) and the split
schedule run, in complex64; the split schedule also in complex128.
"""
import numpy as np
import pytest
import scipy.linalg

import gpesolver_b200 as G
from oracle import oracle as O

from .helpers import gparams, rel_l2

pytestmark = pytest.mark.gpu

RUNS = [("c64", "auto"), ("c64", "split"), ("c128", "split")]


def linear_params(**kw):
    """Config 1's box and trap (64^2 x 16, HARMONIC 60/60/120 Hz), dipolar
    coupling off."""
    p = gparams(O.default_config(**kw))
    p.cdd = 0.0
    return p


def fd_ground_energy(p, V):
    """Lowest eigenvalue of -1/(2m) Laplacian_FD + V on the interior points
    (psi = 0 on the walls); V is separable: V[i,j,k] = V[i,c,c] + V[c,j,c] +
    V[c,c,k] with c = n/2, where every coordinate is 0."""
    V3 = np.asarray(V).reshape(p.nx, p.ny, p.nz)
    cx, cy, cz = p.nx // 2, p.ny // 2, p.nz // 2
    assert V3[cx, cy, cz] == 0.0
    e = 0.0
    for v1, d in ((V3[:, cy, cz], p.dx), (V3[cx, :, cz], p.dy), (V3[cx, cy, :], p.dz)):
        t = 1.0 / (2.0 * p.m * d * d)
        diag = 2.0 * t + v1[1:-1]
        off = np.full(diag.size - 1, -t)
        e += scipy.linalg.eigh_tridiagonal(diag, off, select="i", select_range=(0, 0),
                                           eigvals_only=True)[0]
    return e


@pytest.mark.parametrize("prec,sched", RUNS)
def test_linear_limit_reaches_fd_harmonic_ground_state(prec, sched):
    p = linear_params()
    V = G.potential(p)
    e0 = fd_ground_energy(p, V)
    # the discretisation is coarse (dz is 0.8 oscillator lengths), so the FD
    # eigenvalue sits near, not at, (wx + wy + wz) / 2
    assert abs(e0 / (0.5 * (p.omega_x + p.omega_y + p.omega_z)) - 1) < 0.05
    with G.B200GrossPitaevskiSolver(p, precision=prec, schedule=sched) as s:
        s.set_coeffs(0.0, 0.0)
        s.load_pote(V)
        s.load_buffer(G.initial_psi(p))
        s.imag_steps(20000)
        e = s.calc_energy()
        s.imag_steps(2000)
        e2 = s.calc_energy()
    assert e.e_int == 0.0 and e.e_ext == 0.0 and e.e_bmf == 0.0
    per_atom = e2.e_total / p.n_atoms
    tol = 1e-6 if prec == "c64" else 1e-10
    assert abs(e2.e_total - e.e_total) < tol * abs(e.e_total)  # converged
    assert abs(per_atom - e0) < tol * abs(e0), (per_atom, e0)


@pytest.mark.parametrize("prec,sched", RUNS)
def test_real_time_is_reversible_and_conserves_norm(prec, sched):
    p = linear_params()
    V = G.potential(p)
    k = 500
    with G.B200GrossPitaevskiSolver(p, precision=prec, schedule=sched) as s:
        s.load_pote(V)
        s.load_buffer(G.initial_psi(p))
        s.imag_steps(200)
        start = s.export_data()
        n0 = s.calc_norm()
        s.real_steps(k, 0)
        fwd = s.export_data()
        n1 = s.calc_norm()
    p.real_time_dt = -p.real_time_dt
    with G.B200GrossPitaevskiSolver(p, precision=prec, schedule=sched) as s:
        s.load_pote(V)
        s.import_data(fwd)
        s.real_steps(k, 0)
        back = s.export_data()
    moved = rel_l2(fwd, start)
    assert moved > 1e-2  # the state did evolve
    tol = 2e-5 if prec == "c64" else 1e-10
    assert rel_l2(back, start) < tol * max(1.0, moved)
    assert abs(n1 / n0 - 1) < (1e-6 if prec == "c64" else 1e-12)


@pytest.mark.parametrize("prec,sched", RUNS)
def test_plane_wave_evolves_by_the_exact_phase(prec, sched):
    p = linear_params()
    modes = (3, -2, 1)
    idx = np.meshgrid(np.arange(p.nx), np.arange(p.ny), np.arange(p.nz), indexing="ij")
    arg = sum(2 * np.pi * m * i / n for m, i, n in zip(modes, idx, (p.nx, p.ny, p.nz)))
    psi0 = np.exp(1j * arg).reshape(-1)
    psi0 /= np.sqrt(np.sum(np.abs(psi0) ** 2) * p.dx * p.dy * p.dz)
    k2 = sum((2 * np.pi * m / (n * d)) ** 2 for m, n, d in zip(modes, (p.nx, p.ny, p.nz), (p.dx, p.dy, p.dz)))
    steps = 1000
    with G.B200GrossPitaevskiSolver(p, precision=prec, schedule=sched) as s:
        s.set_coeffs(0.0, 0.0)
        s.load_pote(np.zeros(p.nx * p.ny * p.nz))
        s.import_data(psi0)
        s.real_steps(steps, 0)
        got = s.export_data()
    theta = -steps * p.real_time_dt * k2 / (2 * p.m)
    assert abs(theta) > 0.1  # a phase well above the tolerance
    want = psi0 * np.exp(1j * theta)
    assert rel_l2(got, want) < (1e-5 if prec == "c64" else 1e-11)
