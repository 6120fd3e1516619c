"""Shared helpers of the test suite (fixtures, configs, error metrics)."""
from __future__ import annotations

import os

import numpy as np

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_cases():
    import importlib.util

    spec = importlib.util.spec_from_file_location("gen_golden", os.path.join(GOLDEN, "gen_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, name + ".npz")) as f:
        return {k: f[k] for k in f.files}


def as_json(cfg: dict, calc: str = "FS") -> dict:
    """An oracle config dict -> a gpe_params.json-style dict."""
    j = dict(cfg)
    j["calc_strategy"] = calc
    if j.get("edd") is None:
        j.pop("edd", None)
    else:
        j.pop("edd_start", None)
        j.pop("edd_stop", None)
    return j


def gparams(cfg: dict, calc: str = "FS"):
    import gpesolver_b200 as G

    return G.params_from_json(as_json(cfg, calc))


def rel_l2(a, b) -> float:
    a = np.asarray(a).reshape(-1)
    b = np.asarray(b).reshape(-1)
    if np.iscomplexobj(a) or np.iscomplexobj(b):
        a = a.astype(np.complex128)
        b = b.astype(np.complex128)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def c128(flat: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(flat).view(np.complex128)


def WELL_CONDITIONED(nx, ny, nz):
    """Single-well, contact-dominated configuration (edd ramp 0.70 -> 0.80)."""
    return O.default_config(nx=nx, ny=ny, nz=nz, init_strategy="GAUSS", pote_strategy="HARMONIC",
                            dx=200.0, dy=200.0, dz=800.0, edd=None, edd_start=0.70, edd_stop=0.80,
                            iter_real=500)
