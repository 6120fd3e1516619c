"""Batched imaginary time: many independent solves on one GPU.

A parameter sweep (trap, atom number, dipolar strength, grid) is a set of
independent imaginary-time solves.  ``B200Batch`` creates them as one
``gpe_batch`` (include/gpe_b200.h): every member's fused iteration chain is a
branch of the same CUDA graph, so one graph launch (per call of up to 1024
iterations) runs all members side by side and small grids fill the GPU
together.  Each member
is a ``B200GrossPitaevskiSolver`` view for loading, device-side initialisation,
export and energies; the reference runs each member as a separate process.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

from . import capi
from .params import PhysicalParameters
from .solver import B200GrossPitaevskiSolver, make_gpe_params


class B200Batch:
    def __init__(self, params: Sequence[PhysicalParameters], device: int = 0):
        if not params:
            raise capi.GpeError(capi.GPE_ERR_ARG, "empty batch")
        self._L = capi.lib()
        arr = (capi.gpe_params * len(params))(*[make_gpe_params(p, "c64", device) for p in params])
        b = ctypes.c_void_p()
        capi.check(self._L.gpe_batch_create(arr, len(params), ctypes.byref(b)))
        self._b = b
        self.members: list[B200GrossPitaevskiSolver] = []
        for m, p in enumerate(params):
            h = ctypes.c_void_p()
            capi.check(self._L.gpe_batch_member(self._b, m, ctypes.byref(h)))
            self.members.append(B200GrossPitaevskiSolver._borrow(h, p, "c64"))

    def __len__(self) -> int:
        return len(self.members)

    def __getitem__(self, m: int) -> B200GrossPitaevskiSolver:
        return self.members[m]

    def set_stream(self, stream_ptr: int) -> None:
        capi.check(self._L.gpe_batch_set_stream(self._b, ctypes.c_void_p(stream_ptr)))

    def imag_steps(self, k: int) -> None:
        """k imaginary-time iterations of every member (imag_time_iter, k times)."""
        capi.check(self._L.gpe_batch_imag_steps(self._b, int(k)))

    def close(self) -> None:
        if getattr(self, "_b", None):
            for m in self.members:
                m.close()
            self._L.gpe_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
