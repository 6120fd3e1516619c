"""bench.py's reference arm (the reference's own CPU code, compiled into
oracle/_ref) prints one JSON line with the keys its consumers read; it needs
no GPU, so it runs here."""
import json
import os
import subprocess
import sys

import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not os.path.exists(O.REF_SO) and not os.path.exists(O.ORACLE_SO),
                    reason="oracle libraries not built")
def test_reference_arm_prints_one_json_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1",
                          "--ref-it-setup", "2"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600, check=True).stdout
    lines = [x for x in out.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "split-step RT iterations/s at 128x128x32"
    assert d["unit"] == "iterations/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"]
    fc = cb["fft_backend_check"]
    assert fc["shape"] == [256, 256, 64] and fc["shim_r2c_c2r_s"] > 0
    assert fc["numpy_pocketfft_r2c_c2r_s_1_thread"] > 0
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["grid"] == [128, 128, 32]
