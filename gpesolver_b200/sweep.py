"""Parameter sweeps of imaginary-time ground states.

A sweep is a list of independent solves whose parameters are drawn from a
seeded generator (SplitMix64, so that the members are reproducible from the
seed alone): grid, dipolar strength edd, atom number, radial and axial trap
frequencies, in a CYLINDRICAL trap from a GAUSS initial state.  The members run
together as one ``B200Batch``; the reference would run each as its own
process with its own gpe_params.json.
"""
from __future__ import annotations

from .params import PhysicalParameters, params_from_json

MASK = (1 << 64) - 1

# the sweep's default ranges
GRIDS = ((64, 64, 16), (96, 96, 24), (128, 128, 32))


class SplitMix64:
    """SplitMix64 (Steele, Lea and Flood, 2014): 64-bit state, golden-ratio
    increment, two xor-shift-multiply mixing rounds."""

    def __init__(self, seed: int):
        self.state = seed & MASK

    def next(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
        return z ^ (z >> 31)

    def uniform(self) -> float:
        """U[0, 1) from the top 53 bits."""
        return (self.next() >> 11) * (1.0 / (1 << 53))


def sweep_json(count: int = 64, seed: int = 0, iter_imag: int = 1000, grids=GRIDS,
               edd=(1.2, 1.8), n_atoms=(1e4, 5e4), omega_r=(40.0, 80.0), wz_over_wr=(1.0, 4.0),
               spacing=(120.0, 120.0, 600.0)) -> list[dict]:
    """gpe_params.json dicts of the sweep members (file units: nm, Da, Hz)."""
    rng = SplitMix64(seed)
    out = []
    for _ in range(count):
        g = grids[min(int(rng.uniform() * len(grids)), len(grids) - 1)]
        e = edd[0] + (edd[1] - edd[0]) * rng.uniform()
        n = n_atoms[0] + (n_atoms[1] - n_atoms[0]) * rng.uniform()
        wr = omega_r[0] + (omega_r[1] - omega_r[0]) * rng.uniform()
        wz = wr * (wz_over_wr[0] + (wz_over_wr[1] - wz_over_wr[0]) * rng.uniform())
        out.append({
            "nx": g[0], "ny": g[1], "nz": g[2], "dx": spacing[0], "dy": spacing[1], "dz": spacing[2],
            "m": 163.929, "n_atoms": n, "edd": e, "omega_x": wr, "omega_y": wr, "omega_z": wz,
            "calc_strategy": "IT", "init_strategy": "GAUSS", "pote_strategy": "CYLINDRICAL",
            "iter_imag": iter_imag, "iter_real": 1,
        })
    return out


def sweep_params(**kw) -> list[PhysicalParameters]:
    return [params_from_json(j) for j in sweep_json(**kw)]
