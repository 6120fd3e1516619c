"""The reference's own GPU backend (GpuGrossPitaevskiSolver with its CUDA
kernels and FP64 cuFFT, compiled from its sources into oracle/_ref) runs on
this GPU and agrees with its CPU backend: it is the comparator bench.py times
beside this project's kernels.  Its potential half step also covers the last
boundary layer (cuda_kernels.cu:371), where psi is ~0, hence the tolerance."""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(O.REFGPU_SO) or not os.path.exists(O.REF_SO),
                                 reason="reference libraries not built")]


def test_reference_gpu_backend_matches_cpu_backend():
    cfg = O.default_config(nx=32, ny=32, nz=16, init_strategy="GAUSS", pote_strategy="HARMONIC")
    g = O.RefGpuSolver(cfg)
    try:
        g.imag_steps(5)
        g.real_steps(5, 0)
        got, eg = g.psi().view(np.complex128), g.energy()
    finally:
        g.close()
    r = O.RefSolver(cfg)
    try:
        r.imag_steps(5)
        r.real_steps(5, 0)
        want, er = r.psi().view(np.complex128).copy(), r.energy()
    finally:
        r.close()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-6
    np.testing.assert_allclose(eg, er, rtol=1e-6, atol=1e-6 * abs(er[5]))
