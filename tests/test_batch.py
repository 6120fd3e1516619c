"""Batched imaginary time (gpe_batch): every member's result equals the same
solve run alone through gpe_imag_steps, bit for bit (same kernels, same
inputs, deterministic reductions), for a batch that mixes grids and
parameters."""
import numpy as np
import pytest

import gpesolver_b200 as G
from oracle import oracle as O

from .helpers import gparams

pytestmark = pytest.mark.gpu


def _members():
    out = []
    for dims, pote, edd, n_atoms, wr, wzr in [((32, 32, 16), "CYLINDRICAL", 1.3, 1.2e4, 50., 2.0),
                                             ((64, 64, 16), "CYLINDRICAL", 1.6, 3.0e4, 70., 3.5),
                                             ((32, 32, 16), "HARMONIC", 1.5, 2.0e4, 60., 2.0),
                                             ((64, 64, 32), "CYLINDRICAL", 1.7, 4.5e4, 45., 1.5)]:
        cfg = O.default_config(nx=dims[0], ny=dims[1], nz=dims[2], init_strategy="GAUSS",
                               pote_strategy=pote, edd=edd, n_atoms=n_atoms, omega_x=wr, omega_y=wr,
                               omega_z=wr * wzr, dx=120.0, dy=120.0, dz=600.0)
        out.append(gparams(cfg, "IT"))
    return out


def _alone(p, steps):
    with G.B200GrossPitaevskiSolver(p, precision="c64") as s:
        s.init_pote()
        s.init_buffer()
        for k in steps:
            s.imag_steps(k)
        return s.export_data().copy(), np.array(s.calc_energy())


@pytest.mark.parametrize("steps", [[70], [3, 64, 5]])
def test_batch_equals_single_solves(steps):
    ps = _members()
    with G.B200Batch(ps) as b:
        for m in b.members:
            m.init_pote()
            m.init_buffer()
        for k in steps:
            b.imag_steps(k)
        got = [(m.export_data().copy(), np.array(m.calc_energy())) for m in b.members]
    for p, (psi, e) in zip(ps, got):
        want_psi, want_e = _alone(p, steps)
        assert np.array_equal(psi, want_psi)
        assert np.array_equal(e, want_e)


def test_batch_rejects_grid_without_fused_pipeline():
    cfg = O.default_config(nx=30, ny=30, nz=16)
    with pytest.raises(G.GpeError):
        G.B200Batch([gparams(cfg, "IT")])
