"""The pencil-pass autotuner (GPU): the tile widths it chooses between (x
pencils, y lines) give the same bits, and a grid's choice is made once per
device and reused."""
import numpy as np
import pytest

import gpesolver_b200 as G

from .helpers import WELL_CONDITIONED, gparams

pytestmark = pytest.mark.gpu

CHOICES = {(8, 8), (8, 16), (16, 8), (16, 16)}


@pytest.mark.parametrize("dims", [(64, 64, 16), (32, 256, 16)])
def test_x_tile_choices_give_identical_results(dims, monkeypatch):
    # the plane-kernel schedule (64^2 x 16) and the four-kernel one (32 x 256 x 16)
    p = gparams(WELL_CONDITIONED(*dims))
    V, psi0 = G.potential(p), G.initial_psi(p)
    outs = []
    for tiles in ("16,16", "8,8", "8,16", "16,8"):
        monkeypatch.setenv("GPE_X_TILES", tiles)
        with G.B200GrossPitaevskiSolver(p) as s:
            assert s.x_tiles() == tuple(int(t) for t in tiles.split(","))
            s.load_pote(V)
            s.load_buffer(psi0)
            s.imag_steps(20)
            s.real_steps(20, 0)
            outs.append(s.export_data())
    for o in outs[1:]:
        np.testing.assert_array_equal(o, outs[0])


def test_autotuner_choice_is_reused_per_grid(monkeypatch):
    monkeypatch.delenv("GPE_X_TILES", raising=False)
    p = gparams(WELL_CONDITIONED(64, 64, 16))
    with G.B200GrossPitaevskiSolver(p) as a, G.B200GrossPitaevskiSolver(p) as b:
        assert a.x_tiles() in CHOICES
        assert b.x_tiles() == a.x_tiles()
    with G.B200GrossPitaevskiSolver(p, precision="c128") as c:
        assert c.x_tiles() == (16, 16)  # no fused x pass in FP64


def test_y_column_choices_give_identical_results(monkeypatch):
    # four-kernel schedule: z columns per CTA of the y lines
    p = gparams(WELL_CONDITIONED(32, 256, 16))
    V, psi0 = G.potential(p), G.initial_psi(p)
    outs = []
    for cols in ("16", "8"):
        monkeypatch.setenv("GPE_Y_LINES", cols)
        with G.B200GrossPitaevskiSolver(p) as s:
            s.load_pote(V)
            s.load_buffer(psi0)
            s.imag_steps(20)
            s.real_steps(20, 0)
            outs.append(s.export_data())
    np.testing.assert_array_equal(outs[1], outs[0])
