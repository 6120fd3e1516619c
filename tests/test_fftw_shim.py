"""The FP64 FFTW-API shim against numpy's pocketfft and analytic known answers.

The oracle (and the compiled reference in oracle/_ref) get their FFTs from this
shim, so its semantics are pinned here: unnormalised, forward sign -1, backward
+1, row-major, r2c half spectrum n0 x n1 x (n2/2+1), c2r Hermitian.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

SIZES = [(8, 6, 4), (16, 12, 8), (10, 14, 6), (7, 5, 9), (24, 16, 12), (32, 32, 16)]


def _lib():
    L = ctypes.CDLL(O.ORACLE_SO)
    dp = ctypes.POINTER(ctypes.c_double)
    L.fftw_plan_dft_3d.restype = ctypes.c_void_p
    L.fftw_plan_dft_3d.argtypes = [ctypes.c_int] * 3 + [dp, dp, ctypes.c_int, ctypes.c_uint]
    L.fftw_plan_dft_r2c_3d.restype = ctypes.c_void_p
    L.fftw_plan_dft_r2c_3d.argtypes = [ctypes.c_int] * 3 + [dp, dp, ctypes.c_uint]
    L.fftw_plan_dft_c2r_3d.restype = ctypes.c_void_p
    L.fftw_plan_dft_c2r_3d.argtypes = [ctypes.c_int] * 3 + [dp, dp, ctypes.c_uint]
    L.fftw_execute.argtypes = [ctypes.c_void_p]
    L.fftw_destroy_plan.argtypes = [ctypes.c_void_p]
    L.fftw_plan_with_nthreads.argtypes = [ctypes.c_int]
    L.gpe_shim_fft1d.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int]
    return L


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@pytest.mark.parametrize("shape", SIZES)
@pytest.mark.parametrize("sign", [-1, 1])
@pytest.mark.parametrize("threads", [1, 3])
def test_c2c_matches_numpy(shape, sign, threads):
    L = _lib()
    L.fftw_plan_with_nthreads(threads)
    rng = np.random.default_rng(sum(shape) + sign)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    xin = np.ascontiguousarray(x).view(np.float64).reshape(-1).copy()
    out = np.zeros_like(xin)
    plan = L.fftw_plan_dft_3d(*shape, _p(xin), _p(out), sign, 0)
    L.fftw_execute(plan)
    L.fftw_destroy_plan(plan)
    got = out.view(np.complex128).reshape(shape)
    want = np.fft.fftn(x) if sign < 0 else np.fft.ifftn(x) * x.size
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


@pytest.mark.parametrize("shape", SIZES)
def test_r2c_c2r_match_numpy(shape):
    L = _lib()
    L.fftw_plan_with_nthreads(2)
    rng = np.random.default_rng(7 + sum(shape))
    x = np.ascontiguousarray(rng.standard_normal(shape))
    h = shape[2] // 2 + 1
    spec = np.zeros(2 * shape[0] * shape[1] * h)
    plan = L.fftw_plan_dft_r2c_3d(*shape, _p(x), _p(spec), 0)
    L.fftw_execute(plan)
    L.fftw_destroy_plan(plan)
    want = np.fft.rfftn(x)
    got = spec.view(np.complex128).reshape(want.shape)
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    back = np.zeros(x.size)
    plan = L.fftw_plan_dft_c2r_3d(*shape, _p(spec), _p(back), 0)
    L.fftw_execute(plan)
    L.fftw_destroy_plan(plan)
    assert np.abs(back.reshape(shape) / x.size - x).max() <= 1e-13 * np.abs(x).max()


def test_known_answers():
    L = _lib()
    n = 48
    # delta -> constant
    d = np.zeros(2 * n)
    d[0] = 1.0
    out = np.zeros(2 * n)
    L.gpe_shim_fft1d(n, _p(d), _p(out), -1)
    assert np.allclose(out.view(np.complex128), 1.0, atol=1e-15)
    # plane wave -> single bin
    k0 = 5
    w = np.exp(2j * np.pi * k0 * np.arange(n) / n)
    wi = np.ascontiguousarray(w).view(np.float64).copy()
    L.gpe_shim_fft1d(n, _p(wi), _p(out), -1)
    spec = out.view(np.complex128)
    assert abs(spec[k0] - n) < 1e-12 and np.abs(np.delete(spec, k0)).max() < 1e-12
    # Parseval
    rng = np.random.default_rng(3)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    xi = np.ascontiguousarray(x).view(np.float64).copy()
    L.gpe_shim_fft1d(n, _p(xi), _p(out), -1)
    X = out.view(np.complex128)
    assert abs(np.sum(np.abs(X) ** 2) / n - np.sum(np.abs(x) ** 2)) < 1e-12 * np.sum(np.abs(x) ** 2)


def test_c2r_ignores_imaginary_part_of_self_conjugate_bins():
    # FFTW's c2r uses only the Hermitian part of the half spectrum.
    L = _lib()
    L.fftw_plan_with_nthreads(1)
    shape = (4, 4, 6)
    rng = np.random.default_rng(11)
    x = rng.standard_normal(shape)
    spec = np.fft.rfftn(x)
    spec2 = spec.copy()
    spec2[0, 0, 0] += 3j
    spec2[0, 0, -1] += 2j
    outs = []
    for s in (spec, spec2):
        si = np.ascontiguousarray(s).view(np.float64).reshape(-1).copy()
        back = np.zeros(x.size)
        plan = L.fftw_plan_dft_c2r_3d(*shape, _p(si), _p(back), 0)
        L.fftw_execute(plan)
        L.fftw_destroy_plan(plan)
        outs.append(back)
    assert np.allclose(outs[0], outs[1], atol=1e-12)
