"""ctypes host layer over the C ABI of include/edus_gpu.h.

``Solver`` mirrors the reference's ``DESolver<Operator<complex<double>>>``
call surface (src/DESolver/DESolver.hpp:26-82): ``Propagate``,
``get_CurrentTime``, ``get_ResolutionTime``, ``get_Function``, plus
``rhs`` = one ``SourceTerm`` evaluation (Functional_SourceTerm.hpp:10-56).
Arrays are numpy complex128 in the reference layout [k][n][m].

There is no CPU path: if the CUDA library is missing or fails to load, every
entry raises ``EdusError``.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libedus_gpu.so")

EDUS_OK = 0
ERRORS = {1: "EDUS_ERR_ARG", 2: "EDUS_ERR_CUDA", 3: "EDUS_ERR_TIMEOUT", 4: "EDUS_ERR_DIVERGED",
          5: "EDUS_ERR_UNSUPPORTED", 6: "EDUS_ERR_NOMEM"}
SOLVER_AB, SOLVER_RK = 0, 1
PREC_FP64, PREC_HERM64, PREC_MIXED, PREC_SPLIT32, PREC_HPLANES = 0, 1, 2, 3, 4
ENVELOPE_SIN2, ENVELOPE_GAUSS = 0, 1

# every entry point of include/edus_gpu.h
EXPORTS = [
    "edus_create", "edus_destroy", "edus_last_error", "edus_upload_model", "edus_set_lasers",
    "edus_set_state", "edus_get_state", "edus_set_time", "edus_get_time", "edus_rhs", "edus_step",
    "edus_synchronize", "edus_population_wannier", "edus_device_bytes", "edus_kernel_launches",
    "edus_get_stream", "edus_set_profiling", "edus_get_profile", "edus_rhs_noalloc",
    "edus_set_anchor_interval", "edus_state_rspace", "edus_set_fock_override",
    "edus_mlp_create", "edus_mlp_destroy", "edus_mlp_last_error", "edus_mlp_param_count", "edus_mlp_set_params",
    "edus_mlp_get_params", "edus_mlp_forward", "edus_mlp_gradients", "edus_mlp_train_step",    "edus_upload_model_solve", "edus_sweep_step", "edus_autotune",
    "edus_upload_observables", "edus_observables", "edus_efield", "edus_set_kgradient",
    "edus_set_peierls", "edus_vector_potential", "edus_set_wait_limit",
]


class EdusError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class _Desc(ctypes.Structure):
    _fields_ = [("grid", ctypes.c_int * 3), ("nbands", ctypes.c_int), ("solver", ctypes.c_int),
                ("order", ctypes.c_int), ("dt", ctypes.c_double), ("coulomb", ctypes.c_int),
                ("precision", ctypes.c_int), ("batch", ctypes.c_int), ("device", ctypes.c_int)]


class _Laser(ctypes.Structure):
    _fields_ = [("intensity", ctypes.c_double), ("omega", ctypes.c_double), ("pol", ctypes.c_double * 3),
                ("cycles", ctypes.c_double), ("t0", ctypes.c_double), ("phase", ctypes.c_double),
                ("fwhm", ctypes.c_double), ("envelope", ctypes.c_int)]


@dataclass
class Laser:
    """One pulse in atomic units (see edus_laser in include/edus_gpu.h)."""
    intensity: float
    omega: float
    pol: tuple
    cycles: float = 0.0
    t0: float = 0.0
    phase: float = 0.0
    fwhm: float = 0.0
    envelope: int = ENVELOPE_SIN2


_lib = None


def load_library(path: str | None = None):
    """Load libedus_gpu.so (raises EdusError when absent: no fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise EdusError(2, f"CUDA library not built: {p} (run edus_2.0_b200/build.py)")
    try:
        L = ctypes.CDLL(p)
    except OSError as e:  # pragma: no cover - depends on the box
        raise EdusError(2, f"cannot load {p}: {e}") from e
    P = ctypes.POINTER
    dp = P(ctypes.c_double)
    h = ctypes.c_void_p
    L.edus_create.argtypes = [P(_Desc), P(h)]
    L.edus_destroy.argtypes = [h]
    L.edus_last_error.argtypes = [h]
    L.edus_last_error.restype = ctypes.c_char_p
    L.edus_upload_model.argtypes = [h, dp, dp, dp, dp, dp, dp]
    L.edus_set_lasers.argtypes = [h, ctypes.c_int, ctypes.c_int, P(_Laser)]
    L.edus_set_state.argtypes = [h, ctypes.c_int, dp]
    L.edus_get_state.argtypes = [h, ctypes.c_int, dp]
    L.edus_set_time.argtypes = [h, ctypes.c_double]
    L.edus_get_time.argtypes = [h, dp]
    L.edus_rhs.argtypes = [h, ctypes.c_double, dp, dp]
    L.edus_step.argtypes = [h, ctypes.c_int]
    L.edus_synchronize.argtypes = [h]
    L.edus_population_wannier.argtypes = [h, ctypes.c_int, dp]
    L.edus_device_bytes.argtypes = [h, P(ctypes.c_ulonglong)]
    L.edus_kernel_launches.argtypes = [h, P(ctypes.c_ulonglong)]
    L.edus_get_stream.argtypes = [h, P(ctypes.c_void_p)]
    L.edus_set_profiling.argtypes = [h, ctypes.c_int]
    L.edus_get_profile.argtypes = [h, ctypes.c_int, dp, P(ctypes.c_ulonglong)]
    vp = ctypes.c_void_p
    L.edus_set_anchor_interval.argtypes = [h, ctypes.c_int]
    L.edus_upload_model_solve.argtypes = [h, ctypes.c_int, dp, dp]
    L.edus_upload_observables.argtypes = [h, dp, dp]
    L.edus_set_kgradient.argtypes = [h, ctypes.c_int, P(ctypes.c_int), dp, dp]
    L.edus_observables.argtypes = [h, ctypes.c_int, ctypes.c_int, dp, dp, dp]
    L.edus_efield.argtypes = [h, ctypes.c_int, ctypes.c_double, dp]
    L.edus_set_peierls.argtypes = [h, ctypes.c_int]
    L.edus_set_wait_limit.argtypes = [h, ctypes.c_int]
    L.edus_vector_potential.argtypes = [h, ctypes.c_int, ctypes.c_double, dp]
    L.edus_sweep_step.argtypes = [P(h), ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.edus_autotune.argtypes = [h, P(ctypes.c_int), P(ctypes.c_int)]
    ip = P(ctypes.c_int)
    L.edus_state_rspace.argtypes = [h, ctypes.c_int, ctypes.c_int, ip, dp]
    L.edus_set_fock_override.argtypes = [h, ctypes.c_int, ip, dp]
    mp = ctypes.c_void_p
    fp = P(ctypes.c_float)
    L.edus_mlp_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong, ctypes.c_int, P(mp)]
    L.edus_mlp_destroy.argtypes = [mp]
    L.edus_mlp_last_error.argtypes = [mp]
    L.edus_mlp_last_error.restype = ctypes.c_char_p
    L.edus_mlp_param_count.argtypes = [mp]
    L.edus_mlp_param_count.restype = ctypes.c_longlong
    L.edus_mlp_set_params.argtypes = [mp, fp]
    L.edus_mlp_get_params.argtypes = [mp, fp]
    L.edus_mlp_forward.argtypes = [mp, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    L.edus_mlp_gradients.argtypes = [mp, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, fp, fp]
    L.edus_mlp_train_step.argtypes = [mp, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, fp]
    L.edus_rhs_noalloc.argtypes = [P(ctypes.c_int), ctypes.c_int, ctypes.c_int, dp, dp, vp, vp, vp, vp, vp, vp, vp,
                                   vp, ctypes.c_char_p, ctypes.c_int]
    for name in EXPORTS:
        if name not in ("edus_last_error", "edus_mlp_last_error", "edus_mlp_param_count"):
            getattr(L, name).restype = ctypes.c_int
    if path is None:
        _lib = L
    return L


def _dp(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _c128(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    if shape is not None and a.shape != tuple(shape):
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


class Solver:
    """GPU counterpart of DESolver<Operator<complex<double>>> for one model.

    grid      : (N0, N1, N2) k grid
    nbands    : nb
    solver    : SOLVER_RK or SOLVER_AB ; order 4 (RK) or 4/5 (AB)
    dt        : ResolutionTime in a.u.
    coulomb   : include the HSEX self-energy
    batch     : number of independent solves sharing the model
    """

    def __init__(self, grid, nbands, dt, solver=SOLVER_RK, order=4, coulomb=False, batch=1, device=0,
                 precision=PREC_FP64):
        self._L = load_library()
        d = _Desc()
        for i in range(3):
            d.grid[i] = int(grid[i])
        d.nbands = int(nbands)
        d.solver = int(solver)
        d.order = int(order)
        d.dt = float(dt)
        d.coulomb = int(bool(coulomb))
        d.precision = int(precision)
        d.batch = int(batch)
        d.device = int(device)
        self._h = ctypes.c_void_p()
        rc = self._L.edus_create(ctypes.byref(d), ctypes.byref(self._h))
        if rc != EDUS_OK:
            raise EdusError(rc, self._L.edus_last_error(None).decode())
        self.grid = tuple(int(x) for x in grid)
        self.nb = int(nbands)
        self.Nk = self.grid[0] * self.grid[1] * self.grid[2]
        self.batch = int(batch)
        self.dt = float(dt)
        self.coulomb = bool(coulomb)

    # -- plumbing -----------------------------------------------------------
    def _check(self, rc):
        if rc != EDUS_OK:
            raise EdusError(rc, self._L.edus_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._L.edus_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        return (self.Nk, self.nb, self.nb)

    # -- model / lasers / state ---------------------------------------------
    def upload_model(self, H0k, xik, lattice, W=None, rho0R=None, hartree=None):
        H0k = _c128(H0k, self.shape)
        xik = _c128(xik, (3,) + self.shape)
        lat = np.ascontiguousarray(lattice, dtype=np.float64).reshape(3, 3)
        Wc = _c128(W, self.shape) if W is not None else None
        r0 = _c128(rho0R, self.shape) if rho0R is not None else None
        hc = _c128(hartree, (self.nb, self.nb)) if hartree is not None else None
        self._check(self._L.edus_upload_model(self._h, _dp(H0k), _dp(xik), _dp(lat), _dp(Wc), _dp(r0), _dp(hc)))

    def set_lasers(self, lasers, b=0):
        arr = (_Laser * max(1, len(lasers)))()
        for i, L in enumerate(lasers):
            arr[i].intensity = L.intensity
            arr[i].omega = L.omega
            for j in range(3):
                arr[i].pol[j] = L.pol[j]
            arr[i].cycles = L.cycles
            arr[i].t0 = L.t0
            arr[i].phase = L.phase
            arr[i].fwhm = L.fwhm
            arr[i].envelope = L.envelope
        self._check(self._L.edus_set_lasers(self._h, int(b), len(lasers), arr))

    def set_state(self, rho, b=0):
        a = _c128(rho, self.shape)
        self._check(self._L.edus_set_state(self._h, int(b), _dp(a)))

    def get_state(self, b=0, out=None):
        a = out if out is not None else np.empty(self.shape, dtype=np.complex128)
        self._check(self._L.edus_get_state(self._h, int(b), _dp(a)))
        return a

    # DESolver names
    def get_Function(self, b=0):
        return self.get_state(b)

    @property
    def time(self) -> float:
        t = ctypes.c_double()
        self._check(self._L.edus_get_time(self._h, ctypes.byref(t)))
        return t.value

    @time.setter
    def time(self, t):
        self._check(self._L.edus_set_time(self._h, float(t)))

    def get_CurrentTime(self):
        return self.time

    def get_ResolutionTime(self):
        return self.dt

    # -- compute ------------------------------------------------------------
    def rhs(self, t, rho):
        a = _c128(rho, self.shape)
        out = np.empty(self.shape, dtype=np.complex128)
        self._check(self._L.edus_rhs(self._h, float(t), _dp(a), _dp(out)))
        return out

    def step(self, n=1):
        self._check(self._L.edus_step(self._h, int(n)))

    def Propagate(self, n=1):
        self.step(n)

    def synchronize(self):
        self._check(self._L.edus_synchronize(self._h))

    def set_kgradient(self, shift=None, b=None, w=None):
        """gradient_space "k": the finite-difference stencil (model.kgradient_stencil);
        no arguments restores the R-space gradient."""
        if shift is None:
            self._check(self._L.edus_set_kgradient(self._h, 0, None, None, None))
            return
        sh = np.ascontiguousarray(shift, dtype=np.int32)
        bb = np.ascontiguousarray(b, dtype=np.float64)
        ww = np.ascontiguousarray(w, dtype=np.float64)
        self._check(self._L.edus_set_kgradient(self._h, len(ww), sh.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                               _dp(bb), _dp(ww)))

    def upload_observables(self, U=None, vel=None):
        """Eigenvectors U [Nk][nb][nb] and/or velocity operator [3][Nk][nb][nb]."""
        Uc = _c128(U, self.shape) if U is not None else None
        Vc = _c128(vel, (3,) + self.shape) if vel is not None else None
        self._check(self._L.edus_upload_observables(self._h, _dp(Uc), _dp(Vc)))
        self._has_U = getattr(self, "_has_U", False) or U is not None
        self._has_vel = getattr(self, "_has_vel", False) or vel is not None

    def observables(self, b=0, filled=0):
        """(Bloch populations, Wannier populations, velocity as 3 complex)."""
        pb = np.empty(self.nb) if getattr(self, "_has_U", False) else None
        pw = np.empty(self.nb)
        v = np.empty(6) if getattr(self, "_has_vel", False) else None
        self._check(self._L.edus_observables(self._h, int(b), int(filled), _dp(pb), _dp(pw), _dp(v)))
        return pb, pw, (v[0::2] + 1j * v[1::2]) if v is not None else None

    def efield(self, t, b=0):
        E = np.empty(3)
        self._check(self._L.edus_efield(self._h, int(b), float(t), _dp(E)))
        return E

    def set_peierls(self, on=True):
        """Propagate in the Peierls gauge (input key "peierls"); resets the
        vector-potential integrators."""
        self._check(self._L.edus_set_peierls(self._h, int(bool(on))))

    def vector_potential(self, t, b=0):
        """A(t) of solve b, advancing its integrator to t (Laser::VectorPotential)."""
        A = np.empty(3)
        self._check(self._L.edus_vector_potential(self._h, int(b), float(t), _dp(A)))
        return A

    def upload_model_solve(self, b, H0k, xik):
        """A model of its own for solve b (FP64 form without HSEX)."""
        H = _c128(H0k, self.shape)
        X = _c128(xik, (3,) + self.shape)
        self._check(self._L.edus_upload_model_solve(self._h, int(b), _dp(H), _dp(X)))

    def set_wait_limit(self, polls: int):
        """Poll limit of the plane kernel's bulk-load wait (< 0: the default; 0 gives up at once)."""
        self._check(self._L.edus_set_wait_limit(self._h, int(polls)))

    def autotune(self):
        """Time the launch variants on this handle's data and keep the fastest;
        returns (plane-kernel threads, tensor-core commutator)."""
        t, c = ctypes.c_int(0), ctypes.c_int(0)
        self._check(self._L.edus_autotune(self._h, ctypes.byref(t), ctypes.byref(c)))
        return t.value, bool(c.value)

    def set_anchor_interval(self, steps):
        """Split-precision form: steps between moves of the anchor rho_ref."""
        self._check(self._L.edus_set_anchor_interval(self._h, int(steps)))

    def population_wannier(self, b=0):
        out = np.empty(self.nb)
        self._check(self._L.edus_population_wannier(self._h, int(b), _dp(out)))
        return out

    @property
    def stream(self) -> int:
        """cudaStream_t of the handle, as an integer."""
        v = ctypes.c_void_p()
        self._check(self._L.edus_get_stream(self._h, ctypes.byref(v)))
        return v.value or 0

    def set_profiling(self, on: bool):
        self._check(self._L.edus_set_profiling(self._h, int(bool(on))))

    def profile(self, kind: int):
        """(total ms, launches) of kernel kind 0 (plane) or 1 (commutator)."""
        ms = ctypes.c_double()
        n = ctypes.c_ulonglong()
        self._check(self._L.edus_get_profile(self._h, int(kind), ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    @property
    def device_bytes(self) -> int:
        v = ctypes.c_ulonglong()
        self._check(self._L.edus_device_bytes(self._h, ctypes.byref(v)))
        return v.value

    @property
    def kernel_launches(self) -> int:
        v = ctypes.c_ulonglong()
        self._check(self._L.edus_kernel_launches(self._h, ctypes.byref(v)))
        return v.value


def sweep_step(solvers, steps, graph=True, fused=False):
    """Advance several Solvers (one device, FP64 form) by `steps` steps
    together (edus_sweep_step): each on its own stream, chunks of RK4 steps
    captured into one CUDA graph when `graph`; with `fused`, one persistent
    launch per RK stage for the planes and one for the commutators of every
    solve (independent-particle RK4 handles), captured the same way."""
    if not solvers:
        return
    L = solvers[0]._L
    arr = (ctypes.c_void_p * len(solvers))(*[s._h.value if hasattr(s._h, "value") else s._h for s in solvers])
    rc = L.edus_sweep_step(ctypes.cast(arr, ctypes.POINTER(ctypes.c_void_p)), len(solvers), int(steps),
                           2 if fused else (1 if graph else 0))
    if rc:
        msgs = "; ".join(L.edus_last_error(s._h).decode() for s in solvers if L.edus_last_error(s._h))
        raise EdusError(rc, msgs)
