"""TEST INFRASTRUCTURE ONLY: Python side of the CPU oracle.

Two things live here, both used only by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline leg:

* ``load_input``: restates how the reference turns ``input.json`` into
  atomic-unit parameters -- schema defaults overlaid per laser object
  (src/InputVariables/simulation_parameters.cpp:17-90, input_schema.json),
  ``unit()`` with its silent zero ``NullUnit`` for unknown strings
  (src/ConvertUnits.cpp:22-37) and ``Convert`` = value / out * in
  (src/ConvertUnits.hpp:68-73), as applied in Simulation.cpp:18-41,121-144.
* ``Oracle``: a ctypes wrapper around ``oracle/liboracle.so`` built from
  ``oracle/edus_oracle.cpp``.
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

# src/Constants.hpp:12-22
BOHR = 5.2917721090380e-11
EV = 1.602176634e-19
RYDBERG = 2.1798723611035e-18
AUTIME = 2.4188843265857e-17
EPS0 = 8.8541878188e-12
E0_AU = 5.14220674763e11
FINE = 7.2973525693e-03
C_SI = 299792458.0
C_AU = 1.0 / FINE
AUINTENSITY = 0.5 * C_SI * EPS0 * E0_AU * E0_AU

# unit() table, src/ConvertUnits.cpp:9-37 (anything else -> NullUnit, value 0)
_UNITS = {
    "angstrom": 1.0e-10,
    "nanometers": 1.0e-09,
    "nm": 1.0e-09,
    "electronvolt": EV,
    "joule": 1.0,
    "wcm2": 1.0e04,
    "femtoseconds": 1.0e-15,
    "fs": 1.0e-15,
    "auintensity": AUINTENSITY,
    "autime": AUTIME,
    "aulength": BOHR,
    "auenergy": 2.0 * RYDBERG,
}
AU = {"time": AUTIME, "length": BOHR, "energy": 2.0 * RYDBERG, "intensity": AUINTENSITY}


def unit(name: str) -> float:
    return _UNITS.get(name, 0.0)


def convert(x: float, in_unit: float, out_unit: float) -> float:
    return x / out_unit * in_unit


# input_schema.json defaults (top level and per laser object)
_DEFAULTS = {
    "tb_file": "", "fermienergy": 0.0, "fermienergy_units": "electronvolt", "coulomb": False,
    "opengap": 0, "opengap_units": "electronvolt", "epsilon": 1.0, "r0": [10.0],
    "r0_units": "angstrom", "grid": [10, 10, 1], "filledbands": 0, "dt": 0.01,
    "gradient_space": "R", "dt_units": "autime", "printresolution": 1,
    "printresolution_pulse": 0, "initialtime": 0.0, "initialtime_units": "autime",
    "finaltime": 0.0, "finaltime_units": "autime", "solver": "RK", "order": 4,
    "peierls": False, "kpath": [], "lasers": [],
}
_LASER_DEFAULTS = {
    "intensity": 0.0, "intensity_units": "Wcm2", "frequency": 0.0, "frequency_units": "eV",
    "wavelength": 0.0, "wavelength_units": "nm", "polarization": None, "t0": 0.0,
    "t0_units": "fs", "cycles": 0.0, "phase": 0.0,
    # extension (not in the reference schema): Gaussian envelope with cos carrier
    "envelope": "sin2", "fwhm": 0.0, "fwhm_units": "fs",
}


@dataclass
class LaserAU:
    intensity: float
    omega: float
    pol: tuple
    cycles: float
    t0: float
    phase: float
    envelope: int = 0
    fwhm: float = 0.0


@dataclass
class SimConfig:
    tb_path: str
    grid: tuple
    filledbands: int
    dt: float
    initialtime: float
    finaltime: float
    solver: int  # 0 AB, 1 RK
    order: int
    coulomb: bool
    epsilon: float
    r0: tuple
    gradient_space: str
    lasers: list = field(default_factory=list)
    coulomb_fix_centres: bool = False
    hermitian_nyquist: bool = False  # test switch: the packed forms' Hermitian generator
    printresolution: int = 1
    printresolution_pulse: int = 1
    peierls: bool = False

    @property
    def nsteps(self) -> int:
        # Simulation::Propagate: int((tf - ti)/dt) + 2  (Simulation.cpp:355)
        return int((self.finaltime - self.initialtime) / self.dt) + 2


def load_input(src, base_dir: str | None = None) -> SimConfig:
    """Parse an EDUS ``input.json`` (path, JSON text or dict) to atomic units."""
    if isinstance(src, dict):
        user = src
    elif isinstance(src, str) and os.path.exists(src):
        with open(src) as f:
            user = json.load(f)
        base_dir = base_dir or os.path.dirname(os.path.abspath(src))
    else:
        user = json.loads(src)
    d = dict(_DEFAULTS)
    for k, v in user.items():
        if k != "lasers":
            d[k] = v
    lasers = []
    for L in user.get("lasers", []):
        ld = dict(_LASER_DEFAULTS)
        ld.update(L)
        lasers.append(ld)
    ti = convert(float(d["initialtime"]), unit(d["initialtime_units"]), AU["time"])
    tf = convert(float(d["finaltime"]), unit(d["finaltime_units"]), AU["time"])
    dt = convert(float(d["dt"]), unit(d["dt_units"]), AU["time"])
    # DESolver::set_ResolutionTime re-converts from "autime" (Simulation.cpp:172-174)
    dt = convert(dt, unit("autime"), AU["time"])
    # the schema declares r0 an array; the reference's accessor
    # (config.hpp:100-103, get<std::vector<double>>) rejects a bare number,
    # which the ci-test inputs still use -- read it as a one-element list
    r0_in = d["r0"] if isinstance(d["r0"], (list, tuple)) else [d["r0"]]
    r0 = [convert(float(x), unit(d["r0_units"]), AU["length"]) for x in r0_in]
    las = []
    for ld in lasers:
        t0 = convert(float(ld["t0"]), unit(ld["t0_units"]), AU["time"])
        inten = convert(float(ld["intensity"]), unit(ld["intensity_units"]), AU["intensity"])
        if abs(float(ld["frequency"])) > 1e-7:
            omega = convert(float(ld["frequency"]), unit(ld["frequency_units"]), AU["energy"])
        else:
            if not ld["wavelength"]:
                raise ValueError("You must specify (nonzero) frequency *xor* wavelength!")
            lam = convert(float(ld["wavelength"]), unit(ld["wavelength_units"]), AU["length"])
            omega = 2 * math.pi * C_AU / lam
        env = 1 if ld.get("envelope", "sin2") == "gaussian" else 0
        fwhm = convert(float(ld.get("fwhm", 0.0)), unit(ld.get("fwhm_units", "fs")), AU["time"])
        pol = tuple(float(x) for x in ld["polarization"])
        las.append(LaserAU(inten, omega, pol, float(ld["cycles"]), t0, float(ld["phase"]), env, fwhm))
    tb = d["tb_file"]
    if base_dir and not os.path.isabs(tb):
        tb = os.path.join(base_dir, tb)
    pr = int(d["printresolution"])
    prp = int(d["printresolution_pulse"]) or pr
    return SimConfig(
        tb_path=tb + "_tb.dat", grid=tuple(int(x) for x in d["grid"]),
        filledbands=int(d["filledbands"]), dt=dt, initialtime=ti, finaltime=tf,
        solver=0 if d["solver"] == "AB" else 1, order=int(d["order"]),
        coulomb=bool(d["coulomb"]), epsilon=float(d["epsilon"]), r0=tuple(r0),
        gradient_space=str(d["gradient_space"]), lasers=las,
        coulomb_fix_centres=bool(d.get("coulomb_fix_centres", False)),
        printresolution=pr, printresolution_pulse=prp, peierls=bool(d["peierls"]),
    )


class _Laser(ctypes.Structure):
    _fields_ = [("intensity_au", ctypes.c_double), ("omega_au", ctypes.c_double),
                ("pol", ctypes.c_double * 3), ("cycles", ctypes.c_double),
                ("t0_au", ctypes.c_double), ("phase", ctypes.c_double),
                ("fwhm_au", ctypes.c_double), ("envelope", ctypes.c_int)]


class _Cfg(ctypes.Structure):
    _fields_ = [("tb_path", ctypes.c_char_p), ("grid", ctypes.c_int * 3),
                ("filledbands", ctypes.c_int), ("dt_au", ctypes.c_double),
                ("solver", ctypes.c_int), ("order", ctypes.c_int), ("coulomb", ctypes.c_int),
                ("epsilon", ctypes.c_double), ("r0_au", ctypes.c_double * 3),
                ("nr0", ctypes.c_int), ("coulomb_fix_centres", ctypes.c_int),
                ("hermitian_nyquist", ctypes.c_int), ("gradient_k", ctypes.c_int),
                ("peierls", ctypes.c_int),
                ("nlasers", ctypes.c_int), ("lasers", _Laser * 8)]


def build_lib(force: bool = False) -> str:
    src = os.path.join(HERE, "edus_oracle.cpp")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build_lib()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        dp = P(ctypes.c_double)
        L.oracle_create.restype = ctypes.c_void_p
        L.oracle_create.argtypes = [P(_Cfg)]
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_dims.argtypes = [ctypes.c_void_p, P(ctypes.c_int)]
        L.oracle_time.restype = ctypes.c_double
        L.oracle_time.argtypes = [ctypes.c_void_p]
        L.oracle_set_time.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.oracle_get_array.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.oracle_get_hartree.argtypes = [ctypes.c_void_p, dp]
        L.oracle_get_rcart.argtypes = [ctypes.c_void_p, dp]
        L.oracle_get_eval.argtypes = [ctypes.c_void_p, dp]
        L.oracle_get_lattice.argtypes = [ctypes.c_void_p, dp]
        L.oracle_set_state.argtypes = [ctypes.c_void_p, dp]
        L.oracle_efield.argtypes = [ctypes.c_void_p, ctypes.c_double, dp]
        L.oracle_rhs.argtypes = [ctypes.c_void_p, ctypes.c_double, dp, dp]
        L.oracle_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_observables.argtypes = [ctypes.c_void_p, dp, dp, dp]
        L.oracle_vector_potential.argtypes = [ctypes.c_void_p, ctypes.c_double, dp]
        L.oracle_struve0.restype = ctypes.c_double
        L.oracle_struve0.argtypes = [ctypes.c_double]
        L.oracle_fft.argtypes = [P(ctypes.c_int), ctypes.c_int, dp, dp, ctypes.c_int]
        L.oracle_eigh.argtypes = [ctypes.c_int, dp, dp, dp]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_cfg(cfg: SimConfig) -> _Cfg:
    c = _Cfg()
    c.tb_path = cfg.tb_path.encode()
    for i in range(3):
        c.grid[i] = cfg.grid[i]
    c.filledbands = cfg.filledbands
    c.dt_au = cfg.dt
    c.solver = cfg.solver
    c.order = cfg.order
    c.coulomb = int(cfg.coulomb)
    c.epsilon = cfg.epsilon
    for i, x in enumerate(cfg.r0[:3]):
        c.r0_au[i] = x
    c.nr0 = len(cfg.r0)
    c.coulomb_fix_centres = int(cfg.coulomb_fix_centres)
    c.hermitian_nyquist = int(cfg.hermitian_nyquist)
    c.gradient_k = 1 if cfg.gradient_space == "k" else 0
    c.peierls = int(cfg.peierls)
    if len(cfg.lasers) > 8:
        raise ValueError("at most 8 lasers")
    c.nlasers = len(cfg.lasers)
    for i, L in enumerate(cfg.lasers):
        c.lasers[i].intensity_au = L.intensity
        c.lasers[i].omega_au = L.omega
        for j in range(3):
            c.lasers[i].pol[j] = L.pol[j]
        c.lasers[i].cycles = L.cycles
        c.lasers[i].t0_au = L.t0
        c.lasers[i].phase = L.phase
        c.lasers[i].fwhm_au = L.fwhm
        c.lasers[i].envelope = L.envelope
    return c


class Oracle:
    """FP64 CPU restatement of the reference propagation for one input."""

    ARRAYS = {"H0k": 0, "xk": 1, "yk": 2, "zk": 3, "W": 4, "DM0R": 5, "rho": 6, "U": 7,
              "vx": 8, "vy": 9, "vz": 10, "H0R": 11, "V": 12}

    def __init__(self, cfg: SimConfig):
        self.cfg = cfg
        self._c = make_cfg(cfg)
        L = lib()
        self.h = L.oracle_create(ctypes.byref(self._c))
        if not self.h:
            raise RuntimeError("oracle: " + L.oracle_last_error().decode())
        dims = (ctypes.c_int * 6)()
        L.oracle_dims(self.h, dims)
        self.N = (dims[0], dims[1], dims[2])
        self.nb = dims[3]
        self.Nk = dims[4]
        self.dims = dims[5]

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().oracle_destroy(h)
            self.h = None

    @property
    def shape(self):
        return (self.Nk, self.nb, self.nb)

    def get(self, name: str) -> np.ndarray | None:
        a = np.zeros(self.shape, dtype=np.complex128)
        rc = lib().oracle_get_array(self.h, self.ARRAYS[name], _dp(a))
        return a if rc == 0 else None

    def hartree(self) -> np.ndarray:
        a = np.zeros((self.nb, self.nb), dtype=np.complex128)
        lib().oracle_get_hartree(self.h, _dp(a))
        return a

    def rcart(self) -> np.ndarray:
        a = np.zeros((self.Nk, 3))
        lib().oracle_get_rcart(self.h, _dp(a))
        return a

    def eigenvalues(self) -> np.ndarray:
        a = np.zeros((self.Nk, self.nb))
        lib().oracle_get_eval(self.h, _dp(a))
        return a

    def lattice(self) -> np.ndarray:
        a = np.zeros((3, 3))
        lib().oracle_get_lattice(self.h, _dp(a))
        return a

    @property
    def time(self) -> float:
        return lib().oracle_time(self.h)

    @time.setter
    def time(self, t: float):
        lib().oracle_set_time(self.h, float(t))

    def set_state(self, rho: np.ndarray):
        a = np.ascontiguousarray(rho, dtype=np.complex128)
        assert a.shape == self.shape
        lib().oracle_set_state(self.h, _dp(a))

    def efield(self, t: float) -> np.ndarray:
        e = np.zeros(3)
        lib().oracle_efield(self.h, float(t), _dp(e))
        return e

    def rhs(self, t: float, rho: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(rho, dtype=np.complex128)
        out = np.zeros(self.shape, dtype=np.complex128)
        lib().oracle_rhs(self.h, float(t), _dp(a), _dp(out))
        return out

    def step(self, n: int = 1):
        lib().oracle_step(self.h, int(n))

    def vector_potential(self, t: float) -> np.ndarray:
        """A(t), advancing the integrator to t (Laser::VectorPotential)."""
        A = np.zeros(3)
        lib().oracle_vector_potential(self.h, float(t), _dp(A))
        return A

    def observables(self):
        """Population (Bloch, Wannier) and velocity rows as the reference prints them."""
        pb = np.zeros(self.nb)
        pw = np.zeros(self.nb)
        v = np.zeros(6)
        rc = lib().oracle_observables(self.h, _dp(pb), _dp(pw), _dp(v))
        fb = self.cfg.filledbands
        pb[:fb] = 1.0 - pb[:fb]
        return pb, pw, (v if rc == 0 else None)


def struve0(x: float) -> float:
    return lib().oracle_struve0(float(x))


def fft(a: np.ndarray, dims, sign: int) -> np.ndarray:
    """FFT of interleaved planes: a has shape (N0*N1*N2, howmany)."""
    a = np.ascontiguousarray(a, dtype=np.complex128)
    out = np.zeros_like(a)
    d = (ctypes.c_int * 3)(*dims)
    lib().oracle_fft(d, a.shape[1], _dp(a), _dp(out), int(sign))
    return out


def eigh(A: np.ndarray):
    A = np.ascontiguousarray(A, dtype=np.complex128)
    n = A.shape[0]
    w = np.zeros(n)
    V = np.zeros((n, n), dtype=np.complex128)
    lib().oracle_eigh(n, _dp(A), _dp(w), _dp(V))
    return w, V
