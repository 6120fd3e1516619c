"""Host-side mirror of GPESolver's parameter layer for the B200 backend.

* ``PhysicalParameters`` holds what the reference's singleton of the same name
  holds (src/parameters/parameters.hpp:10-123), in atomic units, and derives the
  coefficients with the same formulas (init_parameters / update_edd,
  src/parameters/parameters.cpp:37-59).
* ``load_params`` reads a gpe_params.json (v1 format) with the reference's
  required-key rules and unit conversions (src/filemanager/file_manager.cpp:436-548)
  and its validation (check_params, :216-235).
* ``potential`` and ``initial_psi`` build V_ext and psi_0 on the host in FP64
  exactly as DataInitializer does (src/initializer/initializer.cpp:46-248),
  including its int-truncated potential coordinates.
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass, field

import numpy as np

# UnitConverter (src/utils/units/units.cpp:3-41)
def len_nm_to_au(nm: float) -> float:
    return nm * 18.897261260649092


def len_au_to_nm(au: float) -> float:
    return au * 0.05291772105


def mass_da_to_au(da: float) -> float:
    return da / 0.000548579909


def mass_au_to_da(au: float) -> float:
    return au * 0.000548579909


def freq_hz_to_au(hz: float) -> float:
    return hz * (4.1356e-12 / 27211.6)


def freq_au_to_hz(au: float) -> float:
    return au / (4.1356e-12 / 27211.6)


def ene_au_to_mev(au: float) -> float:
    return au * 27211.407953


POTENTIALS = ("HARMONIC", "MEXICAN", "MEXICAN_FREE", "CYLINDRICAL", "FREE",
              "MEXICAN_ASYMETRIC", "MEXICAN_ASYMETRIC_FREE")
INIT_STRATEGIES = ("COS", "GAUSS", "MULTIPLE_GAUSS", "SETUP_GAUSS", "BINARY_FILE", "TEXT_FILE")
CALC_STRATEGIES = ("IT", "RT", "FS")


@dataclass
class PhysicalParameters:
    nx: int = 64
    ny: int = 64
    nz: int = 16
    dx: float = 0.0
    dy: float = 0.0
    dz: float = 0.0
    m: float = 0.0
    n_atoms: float = 0.0
    omega_x: float = 0.0
    omega_y: float = 0.0
    omega_z: float = 0.0
    dd: float = 0.0
    const_edd: bool = True
    edd: float = 1.5
    edd_start: float = 0.0
    edd_stop: float = 0.0
    iter_imag: int = 0
    iter_real: int = 0
    fftw_n_threads: int = 4
    calc_strategy: str = "FS"
    init_strategy: str = "MULTIPLE_GAUSS"
    pote_key: str = "HARMONIC"
    n_gauss_max: int = 2
    bec_droplets_x: int = 1
    bec_droplets_y: int = 1
    bec_droplets_z: int = 1
    load_filename: str = ""
    # compile-time constants of the reference (parameters.hpp:69-72)
    real_time_dt: float = 1.00e10
    imag_time_dt: float = 1.25e11
    # derived
    aa: float = field(default=0.0)
    b: float = field(default=0.0)
    dxdydz: float = field(default=0.0)
    add: float = field(default=131.0)
    cdd: float = field(default=0.0)
    ggp11: float = field(default=0.0)
    gamma: float = field(default=0.0)
    w_15: float = field(default=0.0)

    def init_parameters(self) -> None:
        """PhysicalParameters::init_parameters (parameters.cpp:37-51)."""
        num = self.m * math.pow(self.omega_x, 2) / 4.
        self.aa = num / math.pow(self.dd, 2) if self.dd else (math.inf if num else math.nan)
        self.b = 0.5 * self.m * math.pow(self.omega_x, 2)
        self.dxdydz = self.dx * self.dy * self.dz
        self.add = 131.
        self.cdd = 12. * math.pi * self.add / self.m
        a = self.add / self.edd if self.edd != 0 else math.inf
        self.ggp11 = 4. * math.pi * a / self.m
        self.gamma = 128. * math.sqrt(math.pi) * math.pow(a, 2.5) / 3. / self.m * (
            1. + 1.5 * math.pow(self.edd, 2))
        self.w_15 = math.pow(self.n_atoms, 1.5)

    def update_edd(self, it: int) -> None:
        """PhysicalParameters::update_edd (parameters.cpp:53-59)."""
        self.edd = self.edd_start + (self.edd_stop - self.edd_start) * it / float(self.iter_real)
        a = self.add / self.edd if self.edd != 0 else math.inf
        self.ggp11 = 4 * math.pi * a / self.m
        self.gamma = 128. * math.sqrt(math.pi) * math.pow(a, 2.5) / 3. / self.m * (
            1. + 1.5 * math.pow(self.edd, 2))

    @property
    def shape(self) -> tuple[int, int, int]:
        return (self.nx, self.ny, self.nz)

    @property
    def n(self) -> int:
        return self.nx * self.ny * self.nz

    def coords(self):
        """SimulationContext::initialize (src/context/context.cpp:17-34)."""
        x = (np.arange(self.nx) - self.nx // 2) * self.dx
        y = (np.arange(self.ny) - self.ny // 2) * self.dy
        z = (np.arange(self.nz) - self.nz // 2) * self.dz
        return x, y, z


class ParamsError(RuntimeError):
    """Raised where FileManager throws std::runtime_error."""


def _req(j: dict, key: str):
    if key not in j:
        raise ParamsError(f"Missing required key: {key}")
    return j[key]


def load_initialization(p: PhysicalParameters, j: dict) -> None:
    """FileManager::load_initialization (file_manager.cpp:436-466)."""
    init = _req(j, "init_strategy")
    if init not in INIT_STRATEGIES:
        raise ParamsError("Unknown initialization strategy: " + str(init))
    p.init_strategy = init
    if init == "MULTIPLE_GAUSS":
        p.n_gauss_max = int(_req(j, "initial_maximas"))
        if p.n_gauss_max <= 0:
            raise ParamsError("Number of Gaussian maxima must be positive.")
    if init == "SETUP_GAUSS":
        p.bec_droplets_x = int(_req(j, "bec_droplets_x"))
        p.bec_droplets_y = int(_req(j, "bec_droplets_y"))
        p.bec_droplets_z = int(_req(j, "bec_droplets_z"))
    if init in ("BINARY_FILE", "TEXT_FILE"):
        p.load_filename = str(_req(j, "load_filename"))


def load_simulation(p: PhysicalParameters, j: dict) -> None:
    """FileManager::load_simulation (file_manager.cpp:507-541)."""
    calc = _req(j, "calc_strategy")
    _req(j, "iter_imag")
    _req(j, "iter_real")
    _req(j, "n_atoms")
    _req(j, "m")
    if calc in CALC_STRATEGIES:
        p.calc_strategy = calc
    p.iter_imag = int(j["iter_imag"])
    p.iter_real = int(j["iter_real"])
    p.n_atoms = float(j["n_atoms"])
    p.m = mass_da_to_au(float(j["m"]))
    if p.calc_strategy == "IT":
        _req(j, "edd")
    if "edd" in j:
        p.const_edd = True
        p.edd = float(j["edd"])
    else:
        p.edd_start = float(_req(j, "edd_start"))
        p.edd_stop = float(_req(j, "edd_stop"))
        p.const_edd = False
        # The reference leaves edd undefined here (parameters.hpp:120); this
        # build defines it as edd_start.
        p.edd = p.edd_start
    p.fftw_n_threads = int(j.get("fftw_n_threads", 4))
    if p.fftw_n_threads <= 0:
        raise ParamsError("FFTW number of threads must be positive.")


def load_box(p: PhysicalParameters, j: dict) -> None:
    """FileManager::load_box (file_manager.cpp:491-505)."""
    for key in ("dx", "dy", "dz", "nx", "ny", "nz"):
        _req(j, key)
    p.dx, p.dy, p.dz = (len_nm_to_au(float(j[k])) for k in ("dx", "dy", "dz"))
    p.nx, p.ny, p.nz = (int(j[k]) for k in ("nx", "ny", "nz"))


def load_potential(p: PhysicalParameters, j: dict) -> None:
    """FileManager::load_potential (file_manager.cpp:468-489)."""
    p.pote_key = _req(j, "pote_strategy")
    if p.pote_key not in POTENTIALS:
        raise ParamsError("Not know potential option")
    if p.pote_key in ("MEXICAN", "MEXICAN_FREE", "MEXICAN_ASYMETRIC", "MEXICAN_ASYMETRIC_FREE"):
        p.dd = len_nm_to_au(float(_req(j, "dd")))
    elif "dd" in j:
        # not read by the reference for these potentials; kept for the FS switch
        p.dd = len_nm_to_au(float(j["dd"]))
    p.omega_x = freq_hz_to_au(float(_req(j, "omega_x")))
    p.omega_y = freq_hz_to_au(float(_req(j, "omega_y")))
    p.omega_z = freq_hz_to_au(float(_req(j, "omega_z")))


def check_params(p: PhysicalParameters) -> None:
    """FileManager::check_params (file_manager.cpp:216-235)."""
    if p.nx <= 0 or p.ny <= 0 or p.nz <= 0:
        raise ParamsError("Grid dimensions must be positive.")
    if p.dx <= 0 or p.dy <= 0 or p.dz <= 0:
        raise ParamsError("Grid spacings must be positive.")
    if p.n_atoms <= 0:
        raise ParamsError("Number of atoms must be positive.")
    if p.m <= 0:
        raise ParamsError("Mass must be positive.")


def load_all_v1(p: PhysicalParameters, j: dict) -> None:
    """FileManager::load_all_v1 (file_manager.cpp:543-548)."""
    load_initialization(p, j)
    load_simulation(p, j)
    load_box(p, j)
    load_potential(p, j)


def params_from_json(j: dict) -> PhysicalParameters:
    """load_all_v1 + check_params + init_parameters, as FileManager::load_params
    and SimulationManager::on_params_loaded do (file_manager.cpp:56-79,
    sim_manager.cpp:50-52)."""
    p = PhysicalParameters()
    load_all_v1(p, j)
    check_params(p)
    p.init_parameters()
    return p


def load_params(path: str = "gpe_params.json") -> PhysicalParameters:
    try:
        with open(path) as f:
            j = json.load(f)
    except OSError as e:
        raise ParamsError("Could not open params file.") from e
    return params_from_json(j)


# ---------------------------------------------------------------------------
# Potentials and initial states (DataInitializer, host FP64)
# ---------------------------------------------------------------------------
def _pote_eval(p: PhysicalParameters, key: str, x, y, z):
    """PotentialRegistry lambdas (src/parameters/potentials.hpp:76-157).

    std::pow(x, 4) of an integer x is the correctly rounded x^4, which is
    (x*x)*(x*x) (x*x is exact); numpy's power is off by an ulp on some x."""
    m = p.m
    x4 = (x * x) * (x * x)
    if key == "HARMONIC":
        return (0.5 * m * x ** 2 * p.omega_x ** 2 + 0.5 * m * y ** 2 * p.omega_y ** 2) + \
            0.5 * m * z ** 2 * p.omega_z ** 2
    if key == "MEXICAN":
        vx = -p.b * x ** 2 + p.aa * x4
        return (vx + 0.5 * m * y ** 2 * p.omega_y ** 2) + 0.5 * m * z ** 2 * p.omega_z ** 2
    if key == "MEXICAN_FREE":
        vx = p.aa * x4
        return (vx + 0.5 * m * y ** 2 * p.omega_y ** 2) + 0.5 * m * z ** 2 * p.omega_z ** 2
    if key == "CYLINDRICAL":
        r = np.sqrt(x * x + y * y)
        return 0.5 * m * r ** 2 * ((p.omega_y + p.omega_x) / 2.) ** 2 + \
            0.5 * m * z ** 2 * p.omega_z ** 2
    if key == "FREE":
        return 0.5 * m * z ** 2 * p.omega_z ** 2 + 0.0 * x * y
    if key in ("MEXICAN_ASYMETRIC", "MEXICAN_ASYMETRIC_FREE"):
        conv = 27211.4 * 11.6 * 1e9
        slope = (0.25 / conv) / p.dd
        if key == "MEXICAN_ASYMETRIC":
            vx = -p.b * x ** 2 + p.aa * x4 - slope * x
        else:
            vx = p.aa * x4 - slope * x
        return (vx + 0.5 * m * y ** 2 * p.omega_y ** 2) + 0.5 * m * z ** 2 * p.omega_z ** 2
    raise ParamsError("Not know potential option: " + key)


def potential(p: PhysicalParameters, key: str | None = None) -> np.ndarray:
    """DataInitializer::init_pote (initializer.cpp:229-248): V on the full grid,
    with each coordinate truncated toward zero to an int (the initializer keeps
    the potential as std::function<double(int,int,int)>, initializer.hpp:37)."""
    key = key or p.pote_key
    x, y, z = p.coords()
    xi, yi, zi = (np.trunc(v).astype(np.int64).astype(np.float64) for v in (x, y, z))
    X, Y, Z = np.meshgrid(xi, yi, zi, indexing="ij")
    return np.ascontiguousarray(_pote_eval(p, key, X, Y, Z), dtype=np.float64).reshape(-1)


def initial_psi(p: PhysicalParameters) -> np.ndarray:
    """DataInitializer::init_with_* (initializer.cpp:46-219): psi_0 on the
    interior 1..n-2 (boundary zero), as interleaved complex128 (flat float64)."""
    x, y, z = p.coords()
    X, Y, Z = np.meshgrid(x[1:-1], y[1:-1], z[1:-1], indexing="ij")
    s = p.init_strategy
    if s == "COS":
        rrr = int(p.nx / 2) * p.dx
        val = np.cos(2 * math.pi * (X - p.dd) / rrr) * np.cos(2 * math.pi * Y / rrr) * \
            np.cos(1 * math.pi * Z / rrr)
    elif s == "GAUSS":
        sx, sy, sz = p.nx * p.dx / 10., p.ny * p.dy / 10., p.nz * p.dz / 10.
        val = np.exp(-0.5 * (X * X) / (sx * sx)) * np.exp(-0.5 * (Y * Y) / (sy * sy)) * \
            np.exp(-0.5 * (Z * Z) / (sz * sz))
    elif s in ("MULTIPLE_GAUSS", "SETUP_GAUSS"):
        sx, sy, sz = p.nx * p.dx / 20., p.ny * p.dy / 20., p.nz * p.dz / 20.
        centers = []
        if s == "MULTIPLE_GAUSS":
            n = p.n_gauss_max
            for idx in range(n):
                cx = p.dd if idx % 2 else -p.dd
                if n % 2 == 1:
                    cy = (idx - n // 2) * (p.ny * p.dy) / 2. / (n + 1.)
                else:
                    cy = y[0] + (idx // 2 + 1) * (p.ny * p.dy) / (n // 2 + 1)
                centers.append((cx, cy, None))
        else:
            xt, yt, zt = p.nx * p.dx, p.ny * p.dy, p.nz * p.dz
            bx, by, bz = p.bec_droplets_x, p.bec_droplets_y, p.bec_droplets_z
            for i in range(bx):
                for j in range(by):
                    for k in range(bz):
                        centers.append((-xt / 2 + xt / float(bx + 1) * (i + 1),
                                        -yt / 2 + yt / float(by + 1) * (j + 1),
                                        -zt / 2 + zt / float(bz + 1) * (k + 1)))
        val = np.zeros_like(X)
        for cx, cy, cz in centers:
            xc, yc = X - cx, Y - cy
            zc = Z if cz is None else Z - cz
            val = val + np.exp(-0.5 * (xc * xc) / (sx * sx)) * np.exp(-0.5 * (yc * yc) / (sy * sy)) * \
                np.exp(-0.5 * (zc * zc) / (sz * sz))
    else:
        raise ParamsError("initial_psi: strategy " + s + " is loaded from a file")
    psi = np.zeros(p.shape, dtype=np.complex128)
    psi[1:-1, 1:-1, 1:-1] = val
    return psi.reshape(-1).view(np.float64).copy()
