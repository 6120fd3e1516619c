"""Pins the oracle: the plain-C restatement (oracle/gpe_oracle.c) must reproduce
the reference's own CPU solver bit for bit.

Two anchors: the golden fixtures in tests/golden/ (outputs of the reference's
unmodified CPU sources, see tests/golden/gen_golden.py), and -- where the
compiled reference oracle/_ref/libgpe_ref.so is present -- live runs of it.
"""
import numpy as np
import pytest

from oracle import oracle as O

from .helpers import golden, golden_cases

CASES = list(golden_cases().CASES)


def _run_oracle(name):
    mod = golden_cases()
    over, n_it, switch, n_rt, first = mod.CASES[name]
    cfg = O.default_config(**over)
    out = {}
    s = O.OracleSolver(cfg)
    out["psi0"] = s.psi()
    out["pote0"] = s.pote()
    s.calc_fi3d()
    out["op_fi3d"] = s.fi3d()
    s.potential_half_step()
    out["op_pot_half"] = s.psi()
    s.kinetic_step()
    out["op_kinetic"] = s.psi()
    out["op_energy"] = s.energy()
    s.close()
    s = O.OracleSolver(cfg)
    if n_it:
        s.imag_steps(n_it)
        out["it_psi"] = s.psi()
        out["it_fi3d"] = s.fi3d()
        out["it_energy"] = s.energy()
    if switch:
        s.change_potential(switch)
        out["pote1"] = s.pote()
    s.real_steps(n_rt, first)
    out["rt_psi"] = s.psi()
    out["rt_fi3d"] = s.fi3d()
    out["rt_energy"] = s.energy()
    s.close()
    return out


@pytest.mark.parametrize("name", CASES)
def test_restatement_matches_reference_golden_bit_for_bit(name):
    g = golden(name)
    o = _run_oracle(name)
    for key, val in o.items():
        np.testing.assert_array_equal(val, g[key], err_msg=f"{name}:{key}")


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference not built")
def test_restatement_matches_live_reference_longer_run():
    cfg = O.default_config(nx=24, ny=20, nz=12, init_strategy="MULTIPLE_GAUSS", initial_maximas=2,
                           pote_strategy="MEXICAN", dd=1200.0, edd=None, edd_start=1.3, edd_stop=1.7,
                           iter_real=40)
    r = O.RefSolver(cfg)
    o = O.OracleSolver(cfg)
    r.imag_steps(25)
    o.imag_steps(25)
    np.testing.assert_array_equal(r.psi(), o.psi())
    r.change_potential("MEXICAN_FREE")
    o.change_potential("MEXICAN_FREE")
    r.real_steps(30, 5)
    o.real_steps(30, 5)
    np.testing.assert_array_equal(r.psi(), o.psi())
    np.testing.assert_array_equal(r.fi3d(), o.fi3d())
    np.testing.assert_array_equal(r.energy(), o.energy())
    r.close()
    o.close()


def test_golden_fixtures_are_physical():
    # sanity of the pinned data itself: normalised initial state, IT lowers the
    # energy, RT keeps the norm.
    g = golden("fs_mexican_multigauss")
    cfg = O.default_config(**golden_cases().CASES["fs_mexican_multigauss"][0])
    p = O.make_params(cfg)
    dV = p.dx * p.dy * p.dz
    for key in ("psi0", "it_psi", "rt_psi"):
        n = np.sum(np.abs(g[key].view(np.complex128)) ** 2) * dV
        assert abs(n - 1.0) < 1e-9, key


def test_imaginary_time_lowers_the_energy():
    # after the first iteration (the initial energy sees phi = 0), each IT
    # iteration lowers E_total on the README-scale trap
    s = O.OracleSolver(O.default_config(nx=64, ny=64, nz=16))
    s.imag_steps(1)
    e = [s.energy()[5]]
    for _ in range(4):
        s.imag_steps(10)
        e.append(s.energy()[5])
    s.close()
    assert all(b <= a for a, b in zip(e, e[1:])) and e[-1] < e[0], e
