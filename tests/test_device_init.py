"""Device-side potentials and initial states against the host functions.

The host functions (gpesolver_b200.params.potential / initial_psi) reproduce
the reference's PotentialRegistry and DataInitializer bit for bit (they are
pinned in test_params.py and against the golden fixtures); the device
versions must give the same potential bit for bit and the same initial state
to within an ulp-level tolerance (exp / cos are not correctly rounded).
"""
import numpy as np
import pytest

import gpesolver_b200 as G
from oracle import oracle as O

from .helpers import c128, golden, golden_cases, gparams

pytestmark = pytest.mark.gpu

POTS = ["HARMONIC", "MEXICAN", "MEXICAN_FREE", "CYLINDRICAL", "FREE", "MEXICAN_ASYMETRIC",
        "MEXICAN_ASYMETRIC_FREE"]


def _params(**over):
    cfg = O.default_config(**over)
    return gparams(cfg), cfg


@pytest.mark.parametrize("key", POTS)
@pytest.mark.parametrize("dims", [(32, 32, 16), (64, 48, 24)])
def test_potential_bit_identical(key, dims):
    p, _ = _params(nx=dims[0], ny=dims[1], nz=dims[2], pote_strategy="MEXICAN")
    want = G.potential(p, key)
    with G.B200GrossPitaevskiSolver(p, precision="c128") as s:
        s.init_pote(key)
        got = s.export_pote().reshape(-1)
    assert np.array_equal(got, want), np.max(np.abs(got - want))


@pytest.mark.parametrize("name", list(golden_cases().CASES))
def test_potential_matches_reference_fixture(name):
    over = golden_cases().CASES[name][0]
    cfg = O.default_config(**over)
    p = gparams(cfg)
    g = golden(name)
    with G.B200GrossPitaevskiSolver(p, precision="c128") as s:
        s.init_pote()
        got = s.export_pote().reshape(-1)
    assert np.array_equal(got, g["pote0"])


@pytest.mark.parametrize("strategy,extra", [
    ("GAUSS", {}), ("MULTIPLE_GAUSS", {"initial_maximas": 2}), ("MULTIPLE_GAUSS", {"initial_maximas": 5}),
    ("SETUP_GAUSS", {"bec_droplets_x": 3, "bec_droplets_y": 3, "bec_droplets_z": 2}), ("COS", {})])
def test_initial_state_matches_host(strategy, extra):
    p, _ = _params(nx=48, ny=32, nz=16, init_strategy=strategy, pote_strategy="MEXICAN", **extra)
    host = G.initial_psi(p)
    with G.B200GrossPitaevskiSolver(p, precision="c128") as a, \
            G.B200GrossPitaevskiSolver(p, precision="c128") as b:
        a.init_buffer()
        b.load_buffer(host)
        got, want = a.export_data().reshape(-1), b.export_data().reshape(-1)
    # load_buffer normalises both the same way; exp / cos agree to an ulp or two
    assert np.max(np.abs(got - want)) <= 8 * np.finfo(np.float64).eps * np.max(np.abs(want))


@pytest.mark.parametrize("name", list(golden_cases().CASES))
def test_initial_state_matches_reference_fixture(name):
    over = golden_cases().CASES[name][0]
    cfg = O.default_config(**over)
    p = gparams(cfg)
    if p.init_strategy not in G.capi.INIT_IDS:
        pytest.skip("file-based initial state")
    g = golden(name)
    with G.B200GrossPitaevskiSolver(p, precision="c128") as a, \
            G.B200GrossPitaevskiSolver(p, precision="c128") as b:
        a.init_buffer()
        b.load_buffer(g["psi0"])
        got, want = a.export_data().reshape(-1), b.export_data().reshape(-1)
    assert np.max(np.abs(got - want)) <= 8 * np.finfo(np.float64).eps * np.max(np.abs(want))


def test_complex64_potential_same_rounding():
    p, _ = _params(nx=32, ny=32, nz=16, pote_strategy="CYLINDRICAL")
    with G.B200GrossPitaevskiSolver(p, precision="c64") as a, \
            G.B200GrossPitaevskiSolver(p, precision="c64") as b:
        a.init_pote()
        b.load_pote(G.potential(p))
        assert np.array_equal(a.export_pote(), b.export_pote())


def test_bad_arguments():
    p, _ = _params(nx=32, ny=32, nz=16, init_strategy="MULTIPLE_GAUSS", initial_maximas=65)
    with G.B200GrossPitaevskiSolver(p, precision="c64") as s:
        with pytest.raises(G.GpeError):
            s.init_buffer()
