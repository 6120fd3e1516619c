"""Wavefunction files and energy logs in the reference's formats: files written
here are byte-for-byte those the reference's own FileManager writes (its
compiled code, oracle/_ref), and files it writes load here; checkpoints of a
running solve (asynchronous copy, background write) and resuming from them."""
import os

import numpy as np
import pytest

import gpesolver_b200 as G
from gpesolver_b200 import checkpoint as CK
from oracle import oracle as O

from .helpers import WELL_CONDITIONED, as_json

needs_ref = pytest.mark.skipif(not os.path.exists(O.REF_SO), reason="reference harness not built")


def _ref_state(tmp_path, monkeypatch, **over):
    monkeypatch.chdir(tmp_path)
    cfg = O.default_config(nx=12, ny=10, nz=8, **over)
    r = O.RefSolver(cfg)
    r.imag_steps(5)
    return cfg, r


@needs_ref
def test_binary_file_bytes_match_reference(tmp_path, monkeypatch):
    cfg, r = _ref_state(tmp_path, monkeypatch)
    try:
        r.save_binary("ref")
        psi = r.psi().view(np.complex128)
    finally:
        r.close()
    p = G.params_from_json(as_json(cfg))
    CK.save_binary(psi, p, "ours")
    assert open("ours.gpe.bin", "rb").read() == open("ref.gpe.bin", "rb").read()
    np.testing.assert_array_equal(CK.load_binary(p, "ref"), psi)


@needs_ref
def test_reference_loads_our_binary(tmp_path, monkeypatch):
    cfg, r = _ref_state(tmp_path, monkeypatch)
    p = G.params_from_json(as_json(cfg))
    psi = (np.arange(p.n) * (1 + 2j) / p.n).astype(np.complex128)
    CK.save_binary(psi, p, "ours")
    try:
        back = r.load_binary("ours")
    finally:
        r.close()
    np.testing.assert_array_equal(back.view(np.complex128), psi)


@needs_ref
def test_text_and_potential_files_match_reference(tmp_path, monkeypatch):
    cfg, r = _ref_state(tmp_path, monkeypatch, pote_strategy="HARMONIC")
    try:
        r.save_text("ref")
        r.save_pote_text("refpote")
        psi = r.psi().view(np.complex128)
        V = r.pote()
    finally:
        r.close()
    p = G.params_from_json(as_json(cfg))
    CK.save_text(psi, p, "ours")
    CK.save_potential_text(V, p, "ourpote")
    assert open("ours.gpe.dat").read() == open("ref.gpe.dat").read()
    assert open("ourpote.gpe.dat").read() == open("refpote.gpe.dat").read()
    np.testing.assert_allclose(CK.load_text(p, "ref"), psi, rtol=1e-5, atol=1e-300)


@needs_ref
def test_energy_file_matches_reference(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    cfg = O.default_config(nx=12, ny=10, nz=8, iter_imag=230)
    r = O.RefSolver(cfg)
    try:
        r.solve("IT")
        rows = r.saved_energies()
        os.mkdir("ref")
        os.chdir("ref")
        r.save_energies()
        os.chdir("..")
    finally:
        r.close()
    CK.save_energies(rows, ".")
    assert open("energy.gpe.dat").read() == open("ref/energy.gpe.dat").read()


def test_load_checks_grid(tmp_path):
    p = G.params_from_json(as_json(O.default_config(nx=12, ny=10, nz=8)))
    CK.save_binary(np.zeros(p.n, complex), p, str(tmp_path / "a"))
    q = G.params_from_json(as_json(O.default_config(nx=12, ny=10, nz=6)))
    with pytest.raises(G.params.ParamsError, match="Grid dimensions"):
        CK.load_binary(q, str(tmp_path / "a"))
    q = G.params_from_json(as_json(O.default_config(nx=12, ny=10, nz=8, dx=130.0)))
    with pytest.raises(G.params.ParamsError, match="Grid size"):
        CK.load_binary(q, str(tmp_path / "a"))


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [("c128", 1e-9), ("c64", 2e-5)])
def test_checkpointed_solve_and_resume(tmp_path, prec, tol):
    cfg = dict(WELL_CONDITIONED(32, 32, 16), iter_imag=250, iter_real=2000)
    p = G.params_from_json(as_json(cfg, "FS"))
    prefix = str(tmp_path / "wavefunction")
    with G.B200GrossPitaevskiSolver(p, precision=prec) as s:
        s.init_pote()
        s.init_buffer()
        ck = CK.Checkpointer(s, prefix)
        s.solve(checkpointer=ck)
        final = s.export_data().copy()
        enes = list(s.enes)
    # IT checkpoints at 0, 100, 200; RT at 0, 1000, 2000 (each with its fi3d)
    names = sorted(f for f in os.listdir(tmp_path) if f.endswith(".gpe.bin"))
    assert len(names) == 6 and len(enes) == 6
    assert len([f for f in os.listdir(tmp_path) if f.endswith(".fi3d.f64")]) == 3
    rec = CK.resume_record(prefix + "_4")
    assert rec["phase"] == "real" and rec["iteration"] == 1000 and rec["fi3d_file"]
    # resume from the RT checkpoint at iteration 1000: psi from the file, the
    # field of the next half step from the record; the run repeats the
    # uninterrupted one (load_buffer renormalises psi: in complex64 that
    # rescales it by the ~1e-7 norm drift of the first 1000 iterations)
    with G.B200GrossPitaevskiSolver(p, precision=prec) as s:
        s.init_pote("MEXICAN_FREE")
        s.load_buffer(CK.load_binary(p, prefix + "_4"))
        s.solve(resume=rec)
        again = s.export_data()
    assert np.linalg.norm(again - final) / np.linalg.norm(final) < tol
    # the last file holds the final state
    np.testing.assert_allclose(CK.load_binary(p, prefix + "_5").reshape(final.shape), final, rtol=0, atol=1e-12)
