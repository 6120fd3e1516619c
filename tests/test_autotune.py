"""The pencil-pass autotuner (GPU): the tile widths it chooses between (x
pencils, y lines) give the same bits, and a grid's choice is made once per
device and reused."""
import numpy as np
import pytest

import gpesolver_b200 as G

from .helpers import WELL_CONDITIONED, gparams, rel_l2

pytestmark = pytest.mark.gpu

CHOICES = {(8, 8), (8, 16), (16, 8), (16, 16)}


@pytest.mark.parametrize("dims", [(64, 64, 16), (96, 96, 24), (32, 256, 16)])
def test_x_tile_choices_give_identical_results(dims, monkeypatch):
    # the plane-kernel schedule (64^2 x 16; 96^2 x 24, whose x lines take three
    # stages) and the four-kernel one (32 x 256 x 16)
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
        if dims[0] == 96:
            # lines of 3 x 8 x 8 points: the widths' instances agree to FP32
            # rounding, not to the bit (measured: 7e-15 absolute on |psi| ~1e-6)
            assert rel_l2(o, outs[0]) < 1e-6
        else:
            np.testing.assert_array_equal(o, outs[0])


def test_autotuner_choice_is_reused_per_grid(monkeypatch):
    monkeypatch.delenv("GPE_X_TILES", raising=False)
    p = gparams(WELL_CONDITIONED(64, 64, 16))
    with G.B200GrossPitaevskiSolver(p) as a, G.B200GrossPitaevskiSolver(p) as b:
        assert a.x_tiles() in CHOICES
        assert b.x_tiles() == a.x_tiles()
    with G.B200GrossPitaevskiSolver(p, precision="c128") as c:
        assert c.x_tiles() == (16, 16)  # no fused x pass in FP64


def test_plane_decomposition_is_shared_when_x_tiles_are_fixed(monkeypatch):
    """Solvers whose x widths are fixed (GPE_X_TILES) still share the plane
    decomposition measured once per grid, so every solver of a grid runs the
    same plane kernels (the one-CTA and two-CTA real-time kernels agree to
    rounding, not to the bit)."""
    monkeypatch.delenv("GPE_PLANE_PAIR", raising=False)
    p = gparams(WELL_CONDITIONED(64, 64, 32))
    picks = []
    for tiles in ("16,16", "8,8", "16,8", "8,16"):
        monkeypatch.setenv("GPE_X_TILES", tiles)
        with G.B200GrossPitaevskiSolver(p) as s:
            picks.append(s.plane_kernel())
    assert picks[0] in ("k4_yz", "k5_yz_pair") and len(set(picks)) == 1, picks


def test_imaginary_time_block_widths_agree(monkeypatch):
    """The one-CTA imaginary-time plane kernel at twice the real-time block and
    at the real-time block (the autotuner picks per grid; GPE_IT_WIDE fixes
    it): every butterfly and stencil point is computed alike, only the norm's
    partial sums are grouped differently."""
    p = gparams(WELL_CONDITIONED(64, 64, 32))
    monkeypatch.setenv("GPE_PLANE_PAIR", "0")
    monkeypatch.setenv("GPE_X_TILES", "16,16")
    out = {}
    for wide in ("1", "0"):
        monkeypatch.setenv("GPE_IT_WIDE", wide)
        with G.B200GrossPitaevskiSolver(p) as s:
            s.load_pote(G.potential(p))
            s.load_buffer(G.initial_psi(p))
            s.imag_steps(50)
            out[wide] = (s.export_data().copy(), s.calc_norm())
    assert rel_l2(out["0"][0], out["1"][0]) < 1e-9
    assert abs(out["0"][1] - out["1"][1]) < 1e-12 * abs(out["1"][1])


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


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(32, 32, 16), (64, 64, 16), (64, 64, 32), (96, 96, 24), (128, 128, 32)])
def test_plane_pair_kernel_matches_one_cta_plane_kernel(dims, monkeypatch):
    """The middle imaginary- and real-time iterations on the two-CTA plane
    kernels (k5_yz_pair_it, k5_yz_pair: one cluster per x plane) against the
    one-CTA plane kernel (k4_yz): each line goes through the same radices and
    twiddles, so psi and phi agree to FP32 rounding (1e-6) and the norm after
    the imaginary-time iterations to 1e-7 (the one-CTA kernel reads its
    twiddles from shared memory and feeds its first stages from the previous
    pass's output directly; measured 2e-8 at 32^2 x 16, 5e-11 at 128^2 x 32)."""
    p = gparams(WELL_CONDITIONED(*dims))
    out = {}
    monkeypatch.setenv("GPE_X_TILES", "16,16")  # the same x pass in both runs
    for pair in ("1", "0"):
        monkeypatch.setenv("GPE_PLANE_PAIR", pair)
        with G.B200GrossPitaevskiSolver(p, precision="c64") as s:
            assert s.plane_kernel() == ("k5_yz_pair" if pair == "1" else "k4_yz")
            s.load_pote(G.potential(p))
            s.load_buffer(G.initial_psi(p))
            s.imag_steps(20)
            it = (s.export_data().copy(), s.export_fi3d().copy(), s.calc_norm())
            s.real_steps(70, 0)
            out[pair] = it + (s.export_data().copy(), s.export_fi3d().copy())
    a, b = out["1"], out["0"]
    assert rel_l2(a[0], b[0]) < 1e-6 and rel_l2(a[1], b[1]) < 1e-6
    assert abs(a[2] - b[2]) < 1e-7 * abs(b[2])
    assert rel_l2(a[3], b[3]) < 1e-6 and rel_l2(a[4], b[4]) < 1e-6


@pytest.mark.gpu
def test_first_solver_of_a_grid_is_clean_after_tuning():
    """The first solver of a grid on a device runs the autotuner, whose
    imaginary-time candidates leave a zero norm (and NaN behind it) in the
    fields they wrote; the solver must come out as if just created: a finite
    energy before any iteration, and the same iterations as a solver that
    reused the tuner's choice.  Run in a fresh process so that no earlier test
    has tuned the grid."""
    import os
    import subprocess
    import sys

    code = """
import numpy as np, sys
sys.path.insert(0, %r)
import gpesolver_b200 as G
from tests.helpers import WELL_CONDITIONED, gparams
p = gparams(WELL_CONDITIONED(64, 64, 16))
out = []
for _ in range(2):  # the first solver tunes, the second reuses the choice
    with G.B200GrossPitaevskiSolver(p, precision="c64") as s:
        s.init_pote()
        s.init_buffer()
        e0 = s.calc_energy().e_total
        assert np.isfinite(e0), e0
        s.imag_steps(30)
        s.real_steps(30, 0)
        out.append(s.export_data().copy())
d = np.linalg.norm(out[0] - out[1]) / np.linalg.norm(out[1])
assert d == 0.0, d
print("ok")
""" % os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ("GPE_PLANE_PAIR", "GPE_X_TILES", "GPE_Y_LINES")}
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr
