"""The allocation-free dipolar entry point against the handle-based one.

gpe_calc_fi3d_noalloc exists for callers that cannot call cudaMalloc -- a host
framework that owns all device memory through its own allocator, or a loop that
must not add the device-wide synchronisation cudaMalloc/cudaFree can cause.  It
works in a fixed file-scope device array instead of allocating.  Here it is
called twice in a row, through the C ABI, on caller-owned device buffers, and
each result is compared with gpe_calc_fi3d + gpe_export_fi3d of a solver handle
given the same psi.  Tolerance: relative L2 1e-6 (both run the same FP32
kernels; only the twiddle and V_dd(k) tables are built on different processors).

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

import gpesolver_b200 as G
from gpesolver_b200 import capi
from oracle import oracle as O

from .helpers import gparams, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _normalised(p, psi_flat):
    z = psi_flat.view(np.complex128)
    return (z / np.sqrt(np.sum(np.abs(z) ** 2) * p.dx * p.dy * p.dz)).view(np.float64).copy()


def _handle_fi3d(p, psi_norm):
    with G.B200GrossPitaevskiSolver(p, precision="c64") as s:
        s.import_data(psi_norm)
        s.calc_fi3d()
        return s.export_fi3d().reshape(-1)


def _noalloc_fi3d(p, psi_norm, stream=None):
    import torch

    psi_dev = torch.from_numpy(psi_norm.view(np.complex128).astype(np.complex64)).cuda()
    fi_dev = torch.full((p.n,), float("nan"), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    stream = stream or torch.cuda.current_stream()
    rc = capi.lib().gpe_calc_fi3d_noalloc(
        ctypes.c_void_p(psi_dev.data_ptr()), ctypes.c_void_p(fi_dev.data_ptr()), p.nx, p.ny, p.nz,
        p.dx, p.dy, p.dz, p.n_atoms, ctypes.c_void_p(stream.cuda_stream))
    capi.check(rc)
    stream.synchronize()
    return fi_dev.cpu().numpy().astype(np.float64)


def test_noalloc_matches_handle_path_on_two_calls_in_a_row():
    cases = [
        O.default_config(nx=64, ny=64, nz=16, init_strategy="GAUSS", pote_strategy="HARMONIC"),
        O.default_config(nx=48, ny=40, nz=12, init_strategy="MULTIPLE_GAUSS", initial_maximas=3,
                         pote_strategy="MEXICAN"),
        # the README grid, the largest of the stated configurations that fits the array
        O.default_config(nx=128, ny=128, nz=32, init_strategy="MULTIPLE_GAUSS", initial_maximas=2,
                         pote_strategy="MEXICAN"),
    ]
    # the last call repeats the first grid after two others
    for cfg in cases + cases[:1]:
        p = gparams(cfg)
        psi = _normalised(p, G.initial_psi(p))
        want = _handle_fi3d(p, psi)
        got = _noalloc_fi3d(p, psi)
        assert np.all(np.isfinite(got))
        assert rel_l2(got, want) < TOL


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    psi = torch.zeros(2, dtype=torch.complex64, device="cuda")
    fi = torch.zeros(2, dtype=torch.float32, device="cuda")
    rc = capi.lib().gpe_calc_fi3d_noalloc(ctypes.c_void_p(psi.data_ptr()), ctypes.c_void_p(fi.data_ptr()),
                                          256, 256, 64, 1.0, 1.0, 1.0, 1.0, None)
    assert rc == capi.GPE_ERR_SIZE
    assert b"limit" in capi.lib().gpe_last_error()


def test_noalloc_calls_on_two_streams_in_turn():
    """Calls alternate between two streams (each finished before the next
    starts) over two grids; every result matches the handle path."""
    import torch

    a = gparams(O.default_config(nx=64, ny=64, nz=16, init_strategy="GAUSS", pote_strategy="HARMONIC"))
    b = gparams(O.default_config(nx=32, ny=48, nz=16, init_strategy="COS", pote_strategy="CYLINDRICAL"))
    psi = {id(p): _normalised(p, G.initial_psi(p)) for p in (a, b)}
    want = {id(p): _handle_fi3d(p, psi[id(p)]) for p in (a, b)}
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    for k, p in enumerate((a, b, b, a)):
        got = _noalloc_fi3d(p, psi[id(p)], streams[k % 2])
        assert rel_l2(got, want[id(p)]) < TOL
