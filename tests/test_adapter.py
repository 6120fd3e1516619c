"""Drop-in check: the reference's own AbstractGrossPitaevskiSolver code driving
the B200 backend through B200GrossPitaevskiSolver (gpesolver_b200/adapter).

oracle/_ref/libgpe_adapter.so links the reference's base class, parameters,
context and initializer sources with the adapter and libgpe_b200.so; the same
reference code linked with its CPU backend (oracle/_ref/libgpe_ref.so) is the
expected result.  Both libraries are built from the reference's sources where
they are present (``make -C oracle ref adapter``).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

from .helpers import WELL_CONDITIONED, rel_l2

HAVE_ADAPTER = os.path.exists(O.ADAPTER_SO) and os.path.exists(O.REF_SO)
needs_adapter = pytest.mark.skipif(not HAVE_ADAPTER, reason="adapter library not built")

EXPORTS = ["gpeadp_create", "gpeadp_destroy", "gpeadp_imag_steps", "gpeadp_real_steps",
           "gpeadp_solve", "gpeadp_export_psi", "gpeadp_energy", "gpeadp_checkpoints",
           "gpeadp_saved_energies", "gpeadp_last_error"]


@needs_adapter
@pytest.mark.parametrize("fused", [False, True])
def test_adapter_library_loads(fused):
    L = O.alib(fused)
    for name in EXPORTS:
        assert hasattr(L, name), name


def _ref_run(cfg, it, rt, first=0):
    r = O.RefSolver(cfg)
    try:
        r.imag_steps(it)
        r.real_steps(rt, first)
        return r.psi().view(np.complex128).copy(), r.energy()
    finally:
        r.close()


@pytest.mark.gpu
@needs_adapter
@pytest.mark.parametrize("prec,tol", [(1, 1e-10), (0, 2e-5)])
def test_reference_iterations_on_adapter(prec, tol):
    """imag_time_iter / real_time_iter of the reference's base class (each virtual
    one call into the C ABI), with the edd ramp applied by the base class's
    update_edd between iterations."""
    cfg = WELL_CONDITIONED(32, 32, 16)
    want, e_want = _ref_run(cfg, 12, 8, 3)
    a = O.AdapterSolver(cfg, precision=prec)
    try:
        a.imag_steps(12)
        a.real_steps(8, 3)
        got = a.psi().view(np.complex128)
        e = a.energy()
    finally:
        a.close()
    assert rel_l2(got, want) < tol
    np.testing.assert_allclose(e, e_want, rtol=tol, atol=tol * abs(e_want[5]))


@pytest.mark.gpu
@needs_adapter
@pytest.mark.parametrize("fused", [False, True])
@pytest.mark.parametrize("prec,tol", [(1, 1e-9), (0, 1e-4)])
def test_reference_solve_on_adapter(fused, prec, tol):
    """AbstractGrossPitaevskiSolver::solve() with calc_strategy FS: imaginary
    time, the potential switch to MEXICAN_FREE through the mediator, the real-time
    ramp, checkpoints every 100 / 1000 iterations and the energies handed to
    save_energies -- all reference code, the adapter underneath.  ``fused`` is the
    adapter build whose calc_initial_state / calc_evolution run the iterations
    between checkpoints as one device call."""
    cfg = dict(WELL_CONDITIONED(32, 32, 16), iter_imag=130, iter_real=40)
    r = O.RefSolver(cfg)
    try:
        r.solve("FS")
        want = r.psi().view(np.complex128).copy()
        e_want = r.saved_energies()
        n_ck = r.checkpoints()
    finally:
        r.close()
    a = O.AdapterSolver(cfg, precision=prec, fused=fused)
    try:
        a.solve("FS")
        got = a.psi().view(np.complex128)
        e = a.saved_energies()
        assert a.checkpoints() == n_ck == 3  # IT 0, 100; RT 0
    finally:
        a.close()
    assert rel_l2(got, want) < tol
    assert e.shape == e_want.shape == (3, 6)
    np.testing.assert_allclose(e, e_want, rtol=tol, atol=tol * np.abs(e_want[:, 5:]).max())
