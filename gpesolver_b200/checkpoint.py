"""Wavefunction files, energy logs and checkpoints in the reference's formats.

FileManager (src/filemanager/file_manager.cpp) writes
  <name>.gpe.bin   int32 nx, ny, nz; float64 dx, dy, dz [nm]; then nx*ny*nz
                   (re, im) float64 pairs, row-major (x slowest, z fastest),
                   native byte order (file_manager.cpp:251-290)
  <name>.gpe.dat   nx, ny, nz, dx, dy, dz one per line, then one "re<TAB>im"
                   line per point (file_manager.cpp:81-112)
  energy.gpe.dat   "<index>\\t e_kin \\t e_pot \\t e_int \\t e_ext \\t e_bmf \\t
                   e_total" per energy evaluation (file_manager.cpp:387-401)
  potentials       "# nx = ..." header lines, then one value per line
                   (file_manager.cpp:404-434)
with C++ stream formatting (6 significant digits, %g style) for the text
files.  Loading checks the grid and spacings as the reference does and raises
with its messages.

``Checkpointer`` adds what the reference lacks: a resume record (iteration,
phase, edd) beside each .gpe.bin, and the device-to-host copy of psi issued
asynchronously so that it overlaps the next iterations, with the file written
from a background thread.
"""
from __future__ import annotations

import json
import os
import threading
from typing import Optional, Sequence

import numpy as np

from .params import PhysicalParameters, ParamsError, len_au_to_nm, len_nm_to_au

BINARY_EXT = ".gpe.bin"
TEXT_EXT = ".gpe.dat"
ENERGIES_FILENAME = "energy.gpe.dat"


def _g(x: float) -> str:
    """std::ostream << double with the default precision (6, %g style)."""
    return format(float(x), "g")


def save_binary(psi: np.ndarray, p: PhysicalParameters, name: str) -> str:
    """FileManager::save_to_binary_file."""
    path = name + BINARY_EXT
    a = np.ascontiguousarray(np.asarray(psi).reshape(-1), dtype=np.complex128)
    with open(path, "wb") as f:
        f.write(np.array([p.nx, p.ny, p.nz], dtype=np.int32).tobytes())
        f.write(np.array([len_au_to_nm(p.dx), len_au_to_nm(p.dy), len_au_to_nm(p.dz)], dtype=np.float64).tobytes())
        f.write(a.view(np.float64).tobytes())
    return path


def load_binary(p: PhysicalParameters, name: str) -> np.ndarray:
    """FileManager::load_from_binary_file: psi (complex128, flat) after the
    reference's grid checks."""
    path = name + BINARY_EXT
    try:
        f = open(path, "rb")
    except OSError as e:
        raise ParamsError("Could not open last state file for reading.") from e
    with f:
        dims = np.frombuffer(f.read(12), dtype=np.int32)
        if tuple(dims) != (p.nx, p.ny, p.nz):
            raise ParamsError("Grid dimensions in the file do not match current parameters.")
        d = np.frombuffer(f.read(24), dtype=np.float64)
        d_au = [len_nm_to_au(v) for v in d]
        if any(abs(a - b) > 1e-3 for a, b in zip(d_au, (p.dx, p.dy, p.dz))):
            raise ParamsError("Grid size in the file do not match current parameters.")
        data = np.frombuffer(f.read(16 * p.n), dtype=np.float64)
        if data.size != 2 * p.n:
            raise ParamsError("Truncated wavefunction file.")
    return data.view(np.complex128).copy()


def save_text(psi: np.ndarray, p: PhysicalParameters, name: str) -> str:
    """FileManager::save_to_text_file."""
    path = name + TEXT_EXT
    a = np.asarray(psi).reshape(-1)
    with open(path, "w") as f:
        f.write(f"{p.nx}\n{p.ny}\n{p.nz}\n")
        f.write(f"{_g(len_au_to_nm(p.dx))}\n{_g(len_au_to_nm(p.dy))}\n{_g(len_au_to_nm(p.dz))}\n")
        f.writelines(f"{_g(v.real)}\t{_g(v.imag)}\n" for v in a)
    return path


def load_text(p: PhysicalParameters, name: str) -> np.ndarray:
    """FileManager::load_from_text_file."""
    path = name + TEXT_EXT
    try:
        tok = open(path).read().split()
    except OSError as e:
        raise ParamsError("Could not open initial state file for reading.") from e
    if tuple(int(v) for v in tok[:3]) != (p.nx, p.ny, p.nz):
        raise ParamsError("Grid dimensions in the file do not match current parameters.")
    d_au = [len_nm_to_au(float(v)) for v in tok[3:6]]
    if any(abs(a - b) > 1e-3 for a, b in zip(d_au, (p.dx, p.dy, p.dz))):
        raise ParamsError("Grid size in the file do not match current parameters.")
    v = np.array(tok[6:6 + 2 * p.n], dtype=np.float64)
    return v.view(np.complex128).copy()


def save_potential_text(V: np.ndarray, p: PhysicalParameters, name: str) -> str:
    """FileManager::save_pote_to_text_file."""
    path = name + TEXT_EXT
    with open(path, "w") as f:
        f.write(f"# nx = {p.nx}\n# ny = {p.ny}\n# nz = {p.nz}\n")
        f.write(f"# dx = {_g(len_au_to_nm(p.dx))}\n# dy = {_g(len_au_to_nm(p.dy))}\n"
                f"# dz = {_g(len_au_to_nm(p.dz))}\n")
        f.writelines(f"{_g(v)}\n" for v in np.asarray(V).reshape(-1))
    return path


def save_energies(enes: Sequence, directory: str = ".") -> str:
    """FileManager::save_energies: one line per energy evaluation."""
    path = os.path.join(directory, ENERGIES_FILENAME)
    with open(path, "w") as f:
        for it, e in enumerate(enes):
            f.write("\t".join([str(it)] + [_g(v) for v in tuple(e)[:6]]) + "\n")
    return path


class Checkpointer:
    """Checkpoints of a running solver: psi copied to pinned host memory by an
    asynchronous device-to-host copy (issued before the next iterations, so it
    overlaps them), then written as <prefix>_<counter>.gpe.bin by a background
    thread, with <prefix>_<counter>.resume.json recording the iteration, the
    phase and edd for resume()."""

    def __init__(self, solver, prefix: str = "wavefunction"):
        import torch

        self.solver = solver
        self.prefix = prefix
        self.counter = 0
        self._bufs = [torch.empty(2 * solver.n, dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]
        self._which = 0
        self._pending: Optional[tuple] = None
        self._thread: Optional[threading.Thread] = None

    def _flush(self):
        if self._pending is None:
            return
        buf, name, meta, fi3d = self._pending
        self.solver.export_wait()
        psi = buf.view(np.complex128)

        def write():
            save_binary(psi, self.solver.params, name)
            if fi3d is not None:
                fi3d.tofile(meta["fi3d_file"])
            with open(name + ".resume.json", "w") as f:
                json.dump(meta, f)

        if self._thread is not None:
            self._thread.join()
        self._thread = threading.Thread(target=write)
        self._thread.start()
        self._pending = None

    def checkpoint(self, phase: str, iteration: int) -> None:
        """Queue a checkpoint of the solver's current psi (returns at once)."""
        self._flush()
        buf = self._bufs[self._which]
        self._which ^= 1
        self.solver.export_async(buf)
        name = f"{self.prefix}_{self.counter}"
        self.counter += 1
        meta = {"phase": phase, "iteration": int(iteration), "edd": float(self.solver.params.edd),
                "file": name + BINARY_EXT}
        fi3d = None
        if phase == "real":
            # the field the next real-time iteration's first half step uses
            # (raw FP64, nx*ny*nz values), for an exact resume
            fi3d = self.solver.export_fi3d().reshape(-1)
            meta["fi3d_file"] = name + ".fi3d.f64"
        self._pending = (buf, name, meta, fi3d)

    def close(self) -> None:
        self._flush()
        if self._thread is not None:
            self._thread.join()
            self._thread = None


def resume_record(name: str) -> dict:
    with open(name + ".resume.json") as f:
        return json.load(f)
