"""The C ABI without a GPU: the library loads, exports every entry point that
include/gpe_b200.h declares, and its host-only functions agree with the oracle."""
import ctypes
import os
import re

import pytest

from gpesolver_b200 import capi
from oracle import oracle as O

from .helpers import as_json

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "gpe_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gpe_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # the binding table covers the whole header too
    assert sorted(n for n, _, _ in capi.SIGNATURES) == names


def test_abi_version():
    assert capi.lib().gpe_abi_version() == 1


def test_params_derive_matches_reference_formulas_bit_for_bit():
    import gpesolver_b200 as G

    cfg = O.default_config(edd=1.37, n_atoms=3.3e4, m=161.9)
    p = G.params_from_json(as_json(cfg))
    g = capi.gpe_params()
    g.nx, g.ny, g.nz = p.nx, p.ny, p.nz
    g.dx, g.dy, g.dz, g.m, g.n_atoms, g.edd = p.dx, p.dy, p.dz, p.m, p.n_atoms, p.edd
    assert capi.lib().gpe_params_derive(ctypes.byref(g)) == 0
    op = O.make_params(cfg)
    assert (g.cdd, g.ggp11, g.gamma, g.w_15, g.add) == (op.cdd, op.ggp11, op.gamma, op.w_15, op.add)
    assert (g.real_time_dt, g.imag_time_dt) == (1.0e10, 1.25e11)


def test_params_edd_at_matches_update_edd():
    cfg = O.default_config(edd=None, edd_start=1.40, edd_stop=1.60, iter_real=20000)
    op = O.make_params(cfg)
    g = capi.gpe_params()
    g.m, g.add, g.edd_start, g.edd_stop, g.iter_real = op.m, op.add, 1.40, 1.60, 20000
    out = (ctypes.c_double * 3)()
    for it in (0, 5, 12345, 20000):
        assert capi.lib().gpe_params_edd_at(ctypes.byref(g), it, out) == 0
        O.olib().gpeo_update_edd(ctypes.byref(op), it)
        assert tuple(out) == (op.edd, op.ggp11, op.gamma)


def test_argument_errors_are_reported():
    L = capi.lib()
    assert L.gpe_params_derive(None) == capi.GPE_ERR_ARG
    assert b"null" in L.gpe_last_error()
    h = ctypes.c_void_p()
    assert L.gpe_create(None, ctypes.byref(h)) == capi.GPE_ERR_ARG
    assert L.gpe_calc_fi3d(None) == capi.GPE_ERR_ARG
    g = capi.gpe_params()
    g.nx = g.ny = g.nz = 8
    g.precision = 7
    assert L.gpe_create(ctypes.byref(g), ctypes.byref(h)) == capi.GPE_ERR_ARG


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU failure path")
def test_create_fails_loudly_without_a_gpu():
    import gpesolver_b200 as G

    p = G.params_from_json(as_json(O.default_config(nx=8, ny=8, nz=8)))
    with pytest.raises(G.GpeError) as ei:
        G.B200GrossPitaevskiSolver(p)
    assert ei.value.code in (capi.GPE_ERR_CUDA, capi.GPE_ERR_NOMEM)
