"""Build recipe of the gpe_b200 shared library (in-tree, for sm_100a).

``python -m gpesolver_b200.build`` compiles gpesolver_b200/csrc/*.cu into
gpesolver_b200/libgpe_b200.so with nvcc.  No JIT cache is used: the library is
built next to the package so that it travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgpe_b200.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
]
# per-source objects (not committed), so that a change rebuilds only what it touches
OBJDIR = os.path.join(HERE, "_build")


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers() -> list[str]:
    out = [os.path.join(ROOT, "include", "gpe_b200.h")]
    out += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    return out


def _obj(src: str) -> str:
    return os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(f) > t for f in deps)


def up_to_date() -> bool:
    hdrs = headers()
    return not any(_stale(_obj(s), [s] + hdrs) for s in sources()) and not _stale(
        LIB, [_obj(s) for s in sources()])


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles each csrc/*.cu into an object (in parallel, only those older than
    their source or a header), then links libgpe_b200.so."""
    os.makedirs(OBJDIR, exist_ok=True)
    hdrs = headers()
    todo = [s for s in sources() if force or _stale(_obj(s), [s] + hdrs)]
    procs = []
    for src in todo:
        cmd = [nvcc()] + NVCC_FLAGS + ["-c", "-o", _obj(src) + ".tmp", src]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, cwd=CSRC)))
    failed = [src for src, pr in procs if pr.wait() != 0]
    if failed:
        raise RuntimeError("nvcc failed on " + ", ".join(os.path.basename(f) for f in failed))
    for src in todo:
        os.replace(_obj(src) + ".tmp", _obj(src))
    objs = [_obj(s) for s in sources()]
    if force or todo or _stale(LIB, objs):
        cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB + ".tmp"] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd, cwd=CSRC)
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
