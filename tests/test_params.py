"""The host parameter layer against the reference's rules and the oracle.

The required-key cases mirror the reference's own FileManager tests
(tests/filemanager/file_manager_test.cpp); the derived coefficients, potentials
and initial states are compared with the FP64 oracle.
"""
import copy
import os

import numpy as np
import pytest

import gpesolver_b200 as G
from gpesolver_b200 import params as P
from oracle import oracle as O

from .helpers import as_json

VALID = {
    "n_atoms": 1000, "m": 4.0, "dx": 0.1, "dy": 0.1, "dz": 0.1, "nx": 64, "ny": 64, "nz": 64,
    "omega_x": 1.0e9, "omega_y": 1.0e9, "omega_z": 1.0e9, "calc_strategy": "IT",
    "init_strategy": "GAUSS", "pote_strategy": "HARMONIC", "iter_imag": 1000, "iter_real": 5000,
    "edd": 0.0, "fftw_n_threads": 4,
}


def _j(**kw):
    j = copy.deepcopy(VALID)
    for k, v in kw.items():
        if v is None:
            j.pop(k, None)
        else:
            j[k] = v
    return j


@pytest.mark.parametrize("key", ["dx", "dy", "dz", "nx", "ny", "nz"])
def test_load_box_missing_key_throws(key):
    with pytest.raises(P.ParamsError, match=key):
        P.load_box(P.PhysicalParameters(), _j(**{key: None}))


@pytest.mark.parametrize("key", ["calc_strategy", "iter_imag", "iter_real", "n_atoms", "m"])
def test_load_simulation_missing_key_throws(key):
    with pytest.raises(P.ParamsError):
        P.load_simulation(P.PhysicalParameters(), _j(**{key: None}))


def test_load_simulation_optional_fftw_threads_default():
    p = P.PhysicalParameters()
    P.load_simulation(p, _j(fftw_n_threads=None))
    assert p.fftw_n_threads == 4


def test_edd_rules():
    # IT requires edd; RT/FS accept edd_start/edd_stop instead
    with pytest.raises(P.ParamsError):
        P.load_simulation(P.PhysicalParameters(), _j(edd=None))
    p = P.PhysicalParameters()
    P.load_simulation(p, _j(edd=None, calc_strategy="RT", edd_start=1.4, edd_stop=1.6))
    assert not p.const_edd and p.edd_start == 1.4 and p.edd_stop == 1.6 and p.edd == 1.4
    with pytest.raises(P.ParamsError):
        P.load_simulation(P.PhysicalParameters(), _j(edd=None, calc_strategy="RT", edd_start=1.4))


def test_initialization_rules():
    with pytest.raises(P.ParamsError):
        P.load_initialization(P.PhysicalParameters(), _j(init_strategy="MULTIPLE_GAUSS"))
    p = P.PhysicalParameters()
    P.load_initialization(p, _j(init_strategy="MULTIPLE_GAUSS", initial_maximas=3))
    assert p.n_gauss_max == 3
    with pytest.raises(P.ParamsError):
        P.load_initialization(P.PhysicalParameters(), _j(init_strategy="MULTIPLE_GAUSS", initial_maximas=0))
    with pytest.raises(P.ParamsError):
        P.load_initialization(P.PhysicalParameters(), _j(init_strategy="SETUP_GAUSS", bec_droplets_x=1))
    with pytest.raises(P.ParamsError):
        P.load_initialization(P.PhysicalParameters(), _j(init_strategy="BINARY_FILE"))
    with pytest.raises(P.ParamsError):
        P.load_initialization(P.PhysicalParameters(), _j(init_strategy="NOPE"))
    p = P.PhysicalParameters()
    P.load_initialization(p, _j(init_strategy="TEXT_FILE", load_filename="x"))
    assert p.load_filename == "x"


@pytest.mark.parametrize("pote", ["MEXICAN", "MEXICAN_FREE", "MEXICAN_ASYMETRIC", "MEXICAN_ASYMETRIC_FREE"])
def test_mexican_potentials_require_dd(pote):
    with pytest.raises(P.ParamsError, match="dd"):
        P.load_potential(P.PhysicalParameters(), _j(pote_strategy=pote))
    p = P.PhysicalParameters()
    P.load_potential(p, _j(pote_strategy=pote, dd=1500.0))
    assert p.dd == P.len_nm_to_au(1500.0)


def test_potential_rules():
    for key in ("omega_x", "omega_y", "omega_z", "pote_strategy"):
        with pytest.raises(P.ParamsError):
            P.load_potential(P.PhysicalParameters(), _j(**{key: None}))
    with pytest.raises(P.ParamsError):
        P.load_potential(P.PhysicalParameters(), _j(pote_strategy="WRONG"))


def test_check_params():
    with pytest.raises(P.ParamsError):
        G.params_from_json(_j(nx=0))
    with pytest.raises(P.ParamsError):
        G.params_from_json(_j(n_atoms=-1))


def test_error_message_contains_key():
    with pytest.raises(P.ParamsError, match="omega_y"):
        P.load_potential(P.PhysicalParameters(), _j(omega_y=None))


CFGS = [
    dict(nx=16, ny=12, nz=8, init_strategy="GAUSS", pote_strategy="HARMONIC"),
    dict(nx=16, ny=16, nz=8, init_strategy="MULTIPLE_GAUSS", initial_maximas=3, pote_strategy="MEXICAN"),
    dict(nx=16, ny=16, nz=8, init_strategy="MULTIPLE_GAUSS", initial_maximas=2, pote_strategy="MEXICAN_FREE"),
    dict(nx=12, ny=10, nz=6, init_strategy="SETUP_GAUSS", bec_droplets_x=2, bec_droplets_y=2,
         bec_droplets_z=1, pote_strategy="CYLINDRICAL"),
    dict(nx=10, ny=12, nz=8, init_strategy="COS", pote_strategy="FREE"),
    dict(nx=10, ny=12, nz=8, init_strategy="GAUSS", pote_strategy="MEXICAN_ASYMETRIC"),
    dict(nx=10, ny=12, nz=8, init_strategy="GAUSS", pote_strategy="MEXICAN_ASYMETRIC_FREE"),
]


@pytest.mark.parametrize("over", CFGS)
def test_coefficients_potentials_and_initial_states_match_oracle(over):
    cfg = O.default_config(**over)
    p = G.params_from_json(as_json(cfg))
    op = O.make_params(cfg)
    for name in ("dx", "dy", "dz", "m", "omega_x", "omega_y", "omega_z", "dd", "cdd", "ggp11",
                 "gamma", "w_15", "aa", "b", "dxdydz"):
        assert getattr(p, name) == getattr(op, name), name
    np.testing.assert_array_equal(G.potential(p), O.potential(op, cfg["pote_strategy"]))
    # numpy's exp may differ from libm's by one ulp
    np.testing.assert_allclose(G.initial_psi(p), O.initial_psi(op, cfg), rtol=4e-16, atol=1e-300)


def test_update_edd_matches_oracle():
    cfg = O.default_config(edd=None, edd_start=1.4, edd_stop=1.6, iter_real=20000)
    p = G.params_from_json(as_json(cfg, "RT"))
    op = O.make_params(cfg)
    L = O.olib()
    import ctypes
    for it in (0, 1, 777, 19999, 20000):
        p.update_edd(it)
        L.gpeo_update_edd(ctypes.byref(op), it)
        assert (p.edd, p.ggp11, p.gamma) == (op.edd, op.ggp11, op.gamma)


@pytest.mark.parametrize("key", ["HARMONIC", "MEXICAN", "MEXICAN_FREE", "CYLINDRICAL", "FREE",
                                 "MEXICAN_ASYMETRIC", "MEXICAN_ASYMETRIC_FREE"])
@pytest.mark.parametrize("dims", [(64, 48, 24), (128, 128, 32)])
def test_potential_bit_identical_to_reference_at_full_size(key, dims):
    """At these grids x^4 exceeds 2^53: the host potential must round it as
    std::pow does (the reference's own code, compiled, is the comparison)."""
    if not os.path.exists(O.REF_SO):
        pytest.skip("reference harness not built")
    cfg = O.default_config(nx=dims[0], ny=dims[1], nz=dims[2], pote_strategy=key)
    p = G.params_from_json(as_json(cfg))
    r = O.RefSolver(cfg, load_initial=False)
    try:
        want = r.pote()
    finally:
        r.close()
    np.testing.assert_array_equal(G.potential(p), want)


def test_sweep_generator_is_seeded_splitmix64():
    from gpesolver_b200 import sweep

    r = sweep.SplitMix64(0)
    # published first outputs of SplitMix64 from seed 0
    assert r.next() == 0xE220A8397B1DCDAF
    assert r.next() == 0x6E789E6AA1B965F4
    a, b = sweep.sweep_json(count=64, seed=0), sweep.sweep_json(count=64, seed=0)
    assert a == b and len(a) == 64
    for j in a:
        assert (j["nx"], j["ny"], j["nz"]) in sweep.GRIDS
        assert 1.2 <= j["edd"] < 1.8 and 1e4 <= j["n_atoms"] < 5e4
        assert 40 <= j["omega_x"] == j["omega_y"] < 80 and 1 <= j["omega_z"] / j["omega_x"] < 4
    ps = sweep.sweep_params(count=3, seed=1)
    assert all(p.pote_key == "CYLINDRICAL" and p.init_strategy == "GAUSS" for p in ps)
