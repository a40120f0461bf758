"""Host-side model setup for the GPU propagator (one-off, numpy, FP64).

Builds, from an EDUS ``input.json`` and its ``_tb.dat`` model, every array the
C ABI's ``edus_upload_model`` takes, plus the initial density matrix and the
lasers.  It follows the reference's set-up sequence (Simulation.cpp:10-233):

  units            Convert = value / out * in, unknown unit strings -> 0
                   (src/ConvertUnits.cpp:22-37, ConvertUnits.hpp:68-73)
  lattice          A = UC^T in bohr, lattice vectors in columns (Model.hpp:41-44)
  H0(k), r(k)      sum_R exp(+2 pi i k.R) X(R) on k = i/N (fftPair.cpp:110-142),
                   r(k) made Hermitian (BlockMatrix_definitions.hpp:258-277)
  eigensystem      per-k Hermitian eigensolve, ascending (Simulation.cpp:263-286)
  rho(t0)          U diag(f) U^H (Functional_InitialCondition.hpp:15-31)
  HSEX             W, V on the Gamma-centred R grid with the reference's
                   cumulative r_nm (ModelCoulomb.cpp:62-83), Struve H0 of
                   ModelCoulomb.cpp:7-44, Hartree = sum_R V symmetrised
                   (Coulomb.cpp:41-58), rho0(R) = FFT_{-1}(rho(t0))/Nk
The eigensolve here is LAPACK's (numpy); the initial density matrix is a
projector, so it does not depend on the eigenvector gauge.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass

import numpy as np

from . import edus

# src/Constants.hpp:8-22
PI = 3.14159265358979323846
BOHR = 5.2917721090380e-11
EV = 1.602176634e-19
RYD = 2.1798723611035e-18
AUTIME = 2.4188843265857e-17
EPS0 = 8.8541878188e-12
E0_AU = 5.14220674763e11
FINE = 7.2973525693e-03
C_SI = 299792458.0
AUINT = 0.5 * C_SI * EPS0 * E0_AU * E0_AU
THRESHOLD = 1e-8

UNITS = {"angstrom": 1e-10, "nanometers": 1e-9, "nm": 1e-9, "electronvolt": EV, "joule": 1.0,
         "wcm2": 1e4, "femtoseconds": 1e-15, "fs": 1e-15, "auintensity": AUINT, "autime": AUTIME,
         "aulength": BOHR, "auenergy": 2 * RYD}
AU_TIME, AU_LENGTH, AU_ENERGY, AU_INTENSITY = AUTIME, BOHR, 2 * RYD, AUINT

SCHEMA_DEFAULTS = {
    "tb_file": "", "coulomb": False, "epsilon": 1.0, "r0": [10.0], "r0_units": "angstrom",
    "grid": [10, 10, 1], "filledbands": 0, "dt": 0.01, "gradient_space": "R", "dt_units": "autime",
    "printresolution": 1, "printresolution_pulse": 0, "initialtime": 0.0, "initialtime_units": "autime",
    "finaltime": 0.0, "finaltime_units": "autime", "solver": "RK", "order": 4, "peierls": False,
}
LASER_DEFAULTS = {
    "intensity": 0.0, "intensity_units": "Wcm2", "frequency": 0.0, "frequency_units": "eV",
    "wavelength": 0.0, "wavelength_units": "nm", "polarization": None, "t0": 0.0, "t0_units": "fs",
    "cycles": 0.0, "phase": 0.0, "envelope": "sin2", "fwhm": 0.0, "fwhm_units": "fs",
}


def unit(s: str) -> float:
    return UNITS.get(s, 0.0)


def convert(x, u_in, u_out):
    return x / u_out * u_in


def struve0(x):
    """Struve H0 with the series / asymptotic split of ModelCoulomb.cpp:7-44
    (vectorised; each element stops its series where the scalar loop breaks)."""
    X = np.asarray(x, dtype=np.float64)
    out = np.zeros_like(X)
    lo = X <= 20.0
    if lo.any():
        x = X[lo]
        S = np.ones_like(x)
        R = np.ones_like(x)
        act = np.ones(x.shape, dtype=bool)
        for K in range(1, 61):
            Rn = -R * x / (2.0 * K + 1.0) * x / (2.0 * K + 1.0)
            R = np.where(act, Rn, R)
            S = np.where(act, S + Rn, S)
            act &= ~(np.abs(Rn) < np.abs(S) * 1.0e-12)
            if not act.any():
                break
        out[lo] = 2.0 * x / PI * S
    hi = ~lo
    if hi.any():
        x = X[hi]
        KM = np.where(x >= 50.0, 25, (0.5 * (x + 1.0)).astype(np.int64))
        S = np.ones_like(x)
        R = np.ones_like(x)
        act = np.ones(x.shape, dtype=bool)
        for K in range(1, int(KM.max()) + 1):
            act &= K <= KM
            Rn = -R * ((2.0 * K - 1.0) / x) ** 2
            R = np.where(act, Rn, R)
            S = np.where(act, S + Rn, S)
            act &= ~(np.abs(Rn) < np.abs(S) * 1.0e-12)
            if not act.any():
                break
        T = 4.0 / x
        T2 = T * T
        P0 = ((((-.37043e-5 * T2 + .173565e-4) * T2 - .487613e-4) * T2 + .17343e-3) * T2 - 0.1753062e-2) * T2 + .3989422793
        Q0 = T * (((((.32312e-5 * T2 - 0.142078e-4) * T2 + 0.342468e-4) * T2 - 0.869791e-4) * T2 + 0.4564324e-3) * T2 - 0.0124669441)
        TA0 = x - 0.25 * PI
        BY0 = 2.0 / np.sqrt(x) * (P0 * np.sin(TA0) + Q0 * np.cos(TA0))
        out[hi] = 2.0 / (PI * x) * S + BY0
    return out


def read_tb(path: str):
    """Wannier90 _tb.dat (src/Wannier/ReadWannier.cpp:5-153)."""
    with open(path) as f:
        lines = [l.split() for l in f.read().splitlines()]
    uc = np.array([[float(v) for v in lines[i]] for i in (1, 2, 3)])
    nb = int(lines[4][0])
    nR = int(lines[5][0])
    li = 6
    ndeg = 0
    while li < len(lines) and lines[li]:
        ndeg += len(lines[li])
        li += 1
    if ndeg != nR:
        raise ValueError("degeneracy count mismatch")
    while li < len(lines) and not lines[li]:
        li += 1
    Rs = np.zeros((nR, 3), dtype=np.int64)
    H = np.zeros((nR, nb, nb), dtype=np.complex128)
    r = np.zeros((3, nR, nb, nb), dtype=np.complex128)
    idx = 0
    while li + 1 < len(lines) and len(lines[li + 1]) == 4:
        Rs[idx] = [int(round(float(v))) for v in lines[li][:3]]
        li += 1
        while li < len(lines) and lines[li]:
            t = lines[li]
            H[idx, int(t[0]) - 1, int(t[1]) - 1] = float(t[2]) + 1j * float(t[3])
            li += 1
        li += 1
        idx += 1
    if idx != nR:
        raise ValueError("H block count mismatch")
    idx = 0
    while li + 1 < len(lines) and len(lines[li + 1]) == 8:
        li += 1
        while li < len(lines) and len(lines[li]) == 8:
            t = lines[li]
            a, b = int(t[0]) - 1, int(t[1]) - 1
            for d in range(3):
                r[d, idx, a, b] = float(t[2 + 2 * d]) + 1j * float(t[3 + 2 * d])
            li += 1
        li += 1
        idx += 1
    if idx != nR:
        raise ValueError("r block count mismatch")
    return uc, Rs, H, r


def fft_k_to_R(xk, grid):
    """Operator::go_to_R: FFT sign -1 over the k grid, divided by Nk."""
    Nk = xk.shape[0]
    a = xk.reshape(*grid, -1)
    return (np.fft.fftn(a, axes=(0, 1, 2)) / Nk).reshape(xk.shape)


def fft_R_to_k(xR, grid):
    """Operator::go_to_k: FFT sign +1 over the R grid, unnormalised."""
    Nk = xR.shape[0]
    a = xR.reshape(*grid, -1)
    return (np.fft.ifftn(a, axes=(0, 1, 2)) * Nk).reshape(xR.shape)


@dataclass
class Config:
    tb_path: str
    grid: tuple
    filledbands: int
    dt: float
    ti: float
    tf: float
    solver: int
    order: int
    coulomb: bool
    epsilon: float
    r0: tuple
    lasers: list
    coulomb_fix_centres: bool = False
    printresolution: int = 1
    printresolution_pulse: int = 1  # 0 in the input means printresolution
    gradient_space: str = "R"  # "k": finite-difference gradient over k shells
    peierls: bool = False  # propagation in the Peierls gauge (Functional_SourceTerm.hpp:15-50)

    @property
    def nsteps(self):
        return int((self.tf - self.ti) / self.dt) + 2


def parse_input(src, base_dir=None) -> Config:
    """input.json (path, JSON text or dict) -> Config in atomic units
    (simulation_parameters.cpp:17-90, Simulation.cpp:18-41,121-144)."""
    if isinstance(src, dict):
        user = src
    elif os.path.exists(src):
        with open(src) as f:
            user = json.load(f)
        base_dir = base_dir or os.path.dirname(os.path.abspath(src))
    else:
        user = json.loads(src)
    d = dict(SCHEMA_DEFAULTS)
    d.update({k: v for k, v in user.items() if k != "lasers"})
    ti = convert(float(d["initialtime"]), unit(d["initialtime_units"]), AU_TIME)
    tf = convert(float(d["finaltime"]), unit(d["finaltime_units"]), AU_TIME)
    dt = convert(float(d["dt"]), unit(d["dt_units"]), AU_TIME)
    dt = convert(dt, unit("autime"), AU_TIME)
    r0 = d["r0"] if isinstance(d["r0"], (list, tuple)) else [d["r0"]]
    r0 = tuple(convert(float(x), unit(d["r0_units"]), AU_LENGTH) for x in r0)
    lasers = []
    for L in user.get("lasers", []):
        ld = dict(LASER_DEFAULTS)
        ld.update(L)
        t0 = convert(float(ld["t0"]), unit(ld["t0_units"]), AU_TIME)
        inten = convert(float(ld["intensity"]), unit(ld["intensity_units"]), AU_INTENSITY)
        if abs(float(ld["frequency"])) > 1e-7:
            omega = convert(float(ld["frequency"]), unit(ld["frequency_units"]), AU_ENERGY)
        else:
            lam = convert(float(ld["wavelength"]), unit(ld["wavelength_units"]), AU_LENGTH)
            if lam == 0:
                raise ValueError("You must specify (nonzero) frequency *xor* wavelength!")
            omega = 2 * PI * (1.0 / FINE) / lam
        env = edus.ENVELOPE_GAUSS if ld.get("envelope") == "gaussian" else edus.ENVELOPE_SIN2
        fwhm = convert(float(ld.get("fwhm", 0.0)), unit(ld.get("fwhm_units", "fs")), AU_TIME)
        lasers.append(edus.Laser(inten, omega, tuple(float(x) for x in ld["polarization"]),
                                 float(ld["cycles"]), t0, float(ld["phase"]), fwhm, env))
    tb = d["tb_file"]
    if base_dir and not os.path.isabs(tb):
        tb = os.path.join(base_dir, tb)
    return Config(tb + "_tb.dat", tuple(int(x) for x in d["grid"]), int(d["filledbands"]), dt, ti, tf,
                  edus.SOLVER_AB if d["solver"] == "AB" else edus.SOLVER_RK, int(d["order"]),
                  bool(d["coulomb"]), float(d["epsilon"]), r0, lasers,
                  bool(user.get("coulomb_fix_centres", False)), int(d["printresolution"]),
                  int(d["printresolution_pulse"]) or int(d["printresolution"]), str(d["gradient_space"]),
                  bool(d["peierls"]))


class Model:
    """All one-off arrays of a simulation, in the reference's [k][n][m] layout."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        uc, Rs, H, r = read_tb(cfg.tb_path)
        N = cfg.grid
        self.grid = N
        self.Nk = N[0] * N[1] * N[2]
        self.nb = H.shape[1]
        self.A = np.array([[convert(uc[j][i], 1e-10, BOHR) for j in range(3)] for i in range(3)])
        H = convert(H.real, EV, AU_ENERGY) + 1j * convert(H.imag, EV, AU_ENERGY)
        r = convert(r.real, 1e-10, BOHR) + 1j * convert(r.imag, 1e-10, BOHR)
        for d in range(3):
            lo, up = -N[d] / 2.0, N[d] / 2.0
            x = Rs[:, d]
            if np.any(((x < lo) & (np.abs(x - lo) > THRESHOLD)) | (x > up) | (np.abs(x - up) < THRESHOLD)):
                raise ValueError("model R point outside the Gamma-centred grid range")
        i0, i1, i2 = np.meshgrid(np.arange(N[0]), np.arange(N[1]), np.arange(N[2]), indexing="ij")
        kc = np.stack([i0 / N[0], i1 / N[1], i2 / N[2]], -1).reshape(-1, 3)
        ph = np.exp(2j * PI * (kc @ Rs.T.astype(np.float64)))
        self.H0k = np.einsum("kr,rnm->knm", ph, H)
        self.xik = np.stack([np.einsum("kr,rnm->knm", ph, r[d]) for d in range(3)])
        self.xik = 0.5 * (self.xik + np.conj(np.swapaxes(self.xik, -1, -2)))
        # Gamma-centred R of each FFT index
        jc = np.stack([np.where(2 * g >= n, g - n, g) for g, n in zip((i0, i1, i2), N)], -1).reshape(-1, 3)
        self.Rcrys = jc.astype(np.float64)
        self.Rcart = self.Rcrys @ self.A.T
        # eigensystem with the upper triangle ('U' of zheevd)
        Hu = np.triu(self.H0k) + np.conj(np.swapaxes(np.triu(self.H0k, 1), -1, -2))
        self.eval, self.U = np.linalg.eigh(Hu, UPLO="U")
        f = np.zeros(self.nb)
        f[: cfg.filledbands] = 1.0
        self.rho0k = np.einsum("knm,m,klm->knl", self.U, f, np.conj(self.U))
        self.W = self.DM0R = self.hartree = None
        if cfg.coulomb:
            self._coulomb(Rs, r)

    def kgradient_stencil(self):
        """Finite-difference k gradient of gradient_space "k" (kGradient.cpp:26-211,
        Mostofi et al., CPC 178 (2008) 685): (shift [n][3] FFT index of b,
        b [n][3] Cartesian 1/bohr, w [n]) with E.grad f(k) = sum w (b.E) f(k + b)
        over the fewest shells of equal |b| whose A w = q has an exact solution."""
        N = self.grid
        B = 2.0 * PI * np.linalg.inv(self.A).T  # columns: reciprocal vectors
        i0, i1, i2 = np.meshgrid(np.arange(N[0]), np.arange(N[1]), np.arange(N[2]), indexing="ij")
        j = np.stack([i0, i1, i2], -1).reshape(-1, 3)
        x = j / np.array(N, dtype=np.float64)
        for d in range(3):  # Gamma-centred crystal coordinates in [-1/2, 1/2)
            c = x[:, d]
            c = np.where((c < -0.5) & (np.abs(c + 0.5) > THRESHOLD), c + 1.0, c)
            c = np.where((c > 0.5) | (np.abs(c - 0.5) < THRESHOLD), c - 1.0, c)
            x[:, d] = c
        kc = x @ B.T
        norm = np.linalg.norm(kc, axis=1)
        knorms = []
        for v in norm:
            if not any(abs(v - kn) < THRESHOLD for kn in knorms):
                knorms.append(v)
        knorms.sort()
        shells = [[] for _ in knorms]
        for ik, v in enumerate(norm):
            for sh, kn in enumerate(knorms):
                if abs(kn - v) < 1e-7:
                    shells[sh].append(ik)
                    break
        if abs(knorms[0]) > THRESHOLD:
            raise ValueError("k mesh without k = 0")
        shells = shells[1:]
        q = np.array([N[0] > 1, N[1] > 1, N[2] > 1, 0, 0, 0], dtype=np.float64)
        al, be = [0, 1, 2, 0, 0, 1], [0, 1, 2, 1, 2, 2]
        for ns in range(1, len(shells) + 1):
            A = np.array([[sum(kc[ik, al[jj]] * kc[ik, be[jj]] for ik in shells[sh]) for sh in range(ns)]
                          for jj in range(6)])
            w = np.linalg.pinv(A) @ q
            if np.linalg.norm(A @ w - q) < THRESHOLD:
                break
        else:
            raise ValueError("k gradient: no set of shells solves A w = q")
        idx = [ik for sh in range(ns) for ik in shells[sh]]
        ww = [w[sh] for sh in range(ns) for _ in shells[sh]]
        return j[idx].astype(np.int32), kc[idx], np.array(ww)

    def velocity(self):
        """Velocity operator v_d(k), [3][Nk][nb][nb] (Simulation.cpp:523-576):
        -i [r_d(k), H0(k)], plus the gradient of H0 along axis d taken in the
        space of the propagation's gradient (:554-556): i R_d H0(R) added in R
        for gradient_space "R", the finite-difference stencil sum_b w b_d
        H0(k + b) for "k" (kGradient_definitions.hpp:18-30); over the cell area
        (2-D) or volume (3-D); zero for 1-D grids, which the reference leaves
        unset."""
        N = self.grid
        dims = sum(1 for n in N if n > 1)
        v = np.zeros((3,) + self.H0k.shape, dtype=np.complex128)
        if dims < 2:
            return v
        A = self.A
        if dims == 3:
            det = abs(np.linalg.det(A))
        else:
            if N[2] > 1:
                raise ValueError("perpendicular != 2 -> implement me!")
            det = abs(A[0, 0] * A[1, 1] - A[1, 0] * A[0, 1])
        if self.cfg.gradient_space == "k":
            shift, b, w = self.kgradient_stencil()
            j = np.stack(np.meshgrid(np.arange(N[0]), np.arange(N[1]), np.arange(N[2]), indexing="ij"),
                         -1).reshape(-1, 3)
            for d in range(3):
                c = -1j * (self.xik[d] @ self.H0k - self.H0k @ self.xik[d])
                for s in range(len(w)):
                    if w[s] * b[s, d] == 0.0:
                        continue
                    jn = (j + shift[s]) % np.array(N)
                    kn = (jn[:, 0] * N[1] + jn[:, 1]) * N[2] + jn[:, 2]
                    c = c + (w[s] * b[s, d]) * self.H0k[kn]
                v[d] = c / det
            return v
        H0R = fft_k_to_R(self.H0k, N)
        for d in range(3):
            c = -1j * (self.xik[d] @ self.H0k - self.H0k @ self.xik[d])
            cR = fft_k_to_R(c, N) + 1j * self.Rcart[:, d][:, None, None] * H0R
            v[d] = fft_R_to_k(cR, N) / det
        return v

    def _coulomb(self, Rs, r):
        cfg = self.cfg
        nb = self.nb
        r0 = list(cfg.r0)
        if len(r0) == 1:
            r0 = [r0[0]] * 3
        elif len(r0) == 2:
            r0 = [r0[0], r0[1], (r0[0] + r0[1]) / 2.0]
        r0_avg = (r0[0] + r0[1] + r0[2]) / 3.0
        iorg = [i for i in range(len(Rs)) if not Rs[i].any()]
        if not iorg:
            raise ValueError("model has no R=0 block")
        wc = np.array([[r[d, iorg[0], n, n].real for d in range(3)] for n in range(nb)])
        self.centres = wc  # [nb][3] Wannier centres (bohr)
        md, mdn = np.array([100.0, 0.0, 0.0]), 100.0
        for n in range(nb):
            for m in range(n + 1, nb):
                dd = wc[n] - wc[m]
                dn = math.sqrt(dd @ dd)
                if dn < mdn and dn > 1e-5:
                    md, mdn = dd, dn
        # r_nm(R): cumulative subtraction of ModelCoulomb.cpp:76-79 unless fixed
        Rc = self.Rcart
        rr = np.empty((self.Nk, nb, nb, 3))
        for n in range(nb):
            cur = wc[n][None, :] - Rc
            for m in range(nb):
                if cfg.coulomb_fix_centres:
                    rr[:, n, m] = wc[n][None, :] - Rc - wc[m][None, :]
                else:
                    cur = cur - wc[m][None, :]
                    rr[:, n, m] = cur

        def W_of(v):
            red = v / np.array(r0)
            rn = np.sqrt(np.sum(red * red, axis=-1))
            from scipy.special import y0

            safe = np.where(rn < THRESHOLD, 1.0, rn)
            w = PI / (2.0 * r0_avg * cfg.epsilon) * (struve0(safe) - y0(safe))
            return w, rn

        w, rn = W_of(rr)
        if np.any(rn < THRESHOLD):
            wmin, _ = W_of(md[None, :])
            w = np.where(rn < THRESHOLD, wmin[0], w)
        vn = np.sqrt(np.sum(rr * rr, axis=-1))
        vmin = 2.0 / mdn
        V = np.where(vn < mdn, vmin, 2.0 / np.where(vn < mdn, 1.0, vn))
        self.W = w.astype(np.complex128)
        self.V = V
        hart = V.sum(axis=0).astype(np.complex128)
        iu = np.triu_indices(nb, 1)
        sym = (hart[iu] + hart.T[iu]) / 2.0
        hart[iu] = sym
        hart.T[iu] = sym
        self.hartree = hart
        self.DM0R = fft_k_to_R(self.rho0k, self.grid)

    def solver(self, batch=1, device=0, precision=edus.PREC_FP64) -> "edus.Solver":
        cfg = self.cfg
        s = edus.Solver(self.grid, self.nb, cfg.dt, solver=cfg.solver, order=cfg.order, coulomb=cfg.coulomb,
                        batch=batch, device=device, precision=precision)
        if cfg.coulomb:
            s.upload_model(self.H0k, self.xik, self.A, self.W, self.DM0R, self.hartree)
        else:
            s.upload_model(self.H0k, self.xik, self.A)
        if cfg.gradient_space == "k":
            s.set_kgradient(*self.kgradient_stencil())
        for b in range(batch):
            s.set_lasers(cfg.lasers, b)
            s.set_state(self.rho0k, b)
        if cfg.peierls:
            s.set_peierls(True)
        return s
