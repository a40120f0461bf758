"""Synthetic tight-binding workloads (seeded) in the reference's input format.

Each workload is an EDUS ``input.json`` dictionary plus a Wannier90
``_tb.dat`` model file written next to it.  There is no public dataset for
this path: the models are generated here from their physical description.

  chain2     1-D two-band chain, 64x1x1, Gaussian pulse, RK4 (cpu-runnable case)
  hbn2       2-D hexagonal two-band (hBN-like) model, 120x120, Gaussian pulse, RK4
  tmd22      22-orbital spin-orbit TMD-like model, 72x72, HSEX, AB4 (RK4 variant for
             the throughput metric); gap 1.8 eV
  hbn_golden the reference's own hBN IPA test (ci-test/inputs/hBN.json.in)

File format written by ``write_tb`` follows what the reference parser reads
(src/Wannier/ReadWannier.cpp:5-153): header line, three unit-cell rows (A),
number of bands, number of R points, degeneracies, blank line, H blocks
("R" line then "m n re im" lines, eV), then r blocks ("m n x_re x_im y_re y_im
z_re z_im", Angstrom).
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

HBAR_EV_FS = 0.6582119569  # hbar in eV*fs (for fs <-> a.u. checks only)


def write_tb(path: str, uc_rows, Rs, H, r, title="synthetic model"):
    """Write a _tb.dat file.  uc_rows: 3x3 (rows = lattice vectors, A);
    Rs: list of integer 3-tuples; H: [nR][nb][nb] complex (eV); r: [3][nR][nb][nb] (A)."""
    H = np.asarray(H, dtype=np.complex128)
    r = np.asarray(r, dtype=np.complex128)
    nR, nb = H.shape[0], H.shape[1]
    lines = [title]
    for row in uc_rows:
        lines.append("  ".join(f"{x:.16f}" for x in row))
    lines.append(f"{nb}")
    lines.append(f"{nR}")
    deg = ["1"] * nR
    for i in range(0, nR, 15):
        lines.append(" ".join(deg[i:i + 15]))
    lines.append("")
    for iR, R in enumerate(Rs):
        lines.append(f"{R[0]} {R[1]} {R[2]}")
        for n in range(nb):
            for m in range(nb):
                v = H[iR, m, n]
                lines.append(f"{m + 1} {n + 1} {v.real:.17g} {v.imag:.17g}")
        lines.append("")
    for iR, R in enumerate(Rs):
        lines.append(f"{R[0]} {R[1]} {R[2]}")
        for n in range(nb):
            for m in range(nb):
                x, y, z = r[0, iR, m, n], r[1, iR, m, n], r[2, iR, m, n]
                lines.append(f"{m + 1} {n + 1} {x.real:.17g} {x.imag:.17g} {y.real:.17g} {y.imag:.17g} "
                             f"{z.real:.17g} {z.imag:.17g}")
        lines.append("")
    lines.append("")
    with open(path, "w") as f:
        f.write("\n".join(lines))


# ---------------------------------------------------------------------------
def hexagonal_two_band(a=2.5, onsite=3.625, t=-2.3, centre=None):
    """hBN-like two-band model: orbital 1 at the origin, orbital 2 at (a/sqrt3,0,0),
    nearest-neighbour hopping t (the layout of tb_models/hBN_gap7.25eV_a2.5A_tb.dat)."""
    uc = [[a * math.sqrt(3) / 2, a / 2, 0.0], [a * math.sqrt(3) / 2, -a / 2, 0.0], [0.0, 0.0, 10000.0]]
    Rs = [(-1, 0, 0), (0, -1, 0), (0, 0, 0), (0, 1, 0), (1, 0, 0)]
    nb = 2
    H = np.zeros((5, nb, nb), dtype=np.complex128)
    H[0, 0, 1] = t
    H[1, 0, 1] = t
    H[2, 0, 0] = -onsite
    H[2, 1, 1] = onsite
    H[2, 1, 0] = t
    H[2, 0, 1] = t
    H[3, 1, 0] = t
    H[4, 1, 0] = t
    r = np.zeros((3, 5, nb, nb), dtype=np.complex128)
    r[0, 2, 1, 1] = a / math.sqrt(3) if centre is None else centre
    return uc, Rs, H, r


def chain_two_band(a=2.0, onsite=1.0, t_intra=-1.0, t_inter=0.2, dipole_bohr=1.0):
    """1-D two-band chain along x; on-site inter-orbital dipole along x."""
    bohr_A = 0.52917721090380
    uc = [[a, 0.0, 0.0], [0.0, 1000.0, 0.0], [0.0, 0.0, 1000.0]]
    Rs = [(-1, 0, 0), (0, 0, 0), (1, 0, 0)]
    nb = 2
    H = np.zeros((3, nb, nb), dtype=np.complex128)
    for iR in (0, 2):
        H[iR, 0, 0] = H[iR, 1, 1] = t_intra
        H[iR, 0, 1] = H[iR, 1, 0] = t_inter
    H[1, 0, 0] = -onsite
    H[1, 1, 1] = onsite
    r = np.zeros((3, 3, nb, nb), dtype=np.complex128)
    r[0, 1, 0, 1] = r[0, 1, 1, 0] = dipole_bohr * bohr_A
    return uc, Rs, H, r


def _hex_shells():
    """Crystal vectors of the first three neighbour shells of a 60-degree lattice."""
    s1 = [(1, 0), (0, 1), (1, -1)]
    s2 = [(1, 1), (2, -1), (1, -2)]
    s3 = [(2, 0), (0, 2), (2, -2)]
    return [s1, s2, s3]


def _bands_on_grid(uc_A, Rs, H, grid):
    """Eigenvalues of H(k) = sum_R exp(+2 pi i k.R) H(R) on the k grid (k = i/N)."""
    N0, N1, N2 = grid
    k = np.stack(np.meshgrid(np.arange(N0) / N0, np.arange(N1) / N1, np.arange(N2) / N2, indexing="ij"), -1).reshape(-1, 3)
    R = np.asarray(Rs, dtype=np.float64)
    ph = np.exp(2j * np.pi * (k @ R.T))
    Hk = np.einsum("kr,rnm->knm", ph, H)
    Hk = 0.5 * (Hk + np.conj(np.transpose(Hk, (0, 2, 1))))
    return np.linalg.eigvalsh(Hk)


def tmd_like(nb=22, a=3.19, tmax=1.5, gap=1.8, grid=(72, 72, 1), seed=1234, dipole_A=0.3):
    """22-orbital spin-orbit TMD-like model with random Hermitian hoppings out to
    third neighbours (|t| <= tmax eV, complex: spin-orbit), seeded.

    The first nb/2 orbitals are valence-like, the rest conduction-like; a rigid
    on-site offset between the two manifolds is tuned by bisection so that the
    band gap (band nb/2 minus band nb/2-1, over the k grid) equals `gap` eV.
    This plays the role of the scissor: the gap lives in H0 itself, as the
    reference's OpenGap never reaches the propagated H0 (Simulation.cpp:106-118
    vs 148).  Wannier centres: all at the origin except the last orbital, which
    keeps the reference's cumulative r_nm of ModelCoulomb.cpp:76-79 equal to
    c_n - R - c_m.
    """
    rng = np.random.default_rng(seed)
    nv = nb // 2
    uc = [[a * math.sqrt(3) / 2, a / 2, 0.0], [a * math.sqrt(3) / 2, -a / 2, 0.0], [0.0, 0.0, 20.0]]
    shells = _hex_shells()
    Rs = [(0, 0, 0)]
    blocks = [None]
    decay = [1.0, 0.45, 0.2]
    for s, shell in enumerate(shells):
        for (i, j) in shell:
            T = (rng.uniform(-1, 1, (nb, nb)) + 1j * rng.uniform(-1, 1, (nb, nb))) * tmax * decay[s] / math.sqrt(2)
            # weak valence-conduction mixing keeps the gap tunable
            T[:nv, nv:] *= 0.15
            T[nv:, :nv] *= 0.15
            T = np.clip(T.real, -tmax, tmax) + 1j * np.clip(T.imag, -tmax, tmax)
            Rs.append((i, j, 0))
            blocks.append(T)
            Rs.append((-i, -j, 0))
            blocks.append(T.conj().T)
    nR = len(Rs)
    H = np.zeros((nR, nb, nb), dtype=np.complex128)
    for iR in range(1, nR):
        H[iR] = blocks[iR]
    # on-site: random Hermitian with a spread of orbital energies
    A0 = (rng.uniform(-1, 1, (nb, nb)) + 1j * rng.uniform(-1, 1, (nb, nb))) * 0.3
    A0 = 0.5 * (A0 + A0.conj().T)
    A0[:nv, nv:] *= 0.15
    A0[nv:, :nv] *= 0.15
    base = A0 + np.diag(rng.uniform(-0.5, 0.5, nb))

    def gap_for(offset):
        H[0] = base + np.diag(np.r_[-np.full(nv, offset / 2), np.full(nb - nv, offset / 2)])
        ev = _bands_on_grid(uc, Rs, H, grid)
        return ev[:, nv].min() - ev[:, nv - 1].max()

    from scipy.optimize import brentq

    if gap_for(60.0) < gap:
        raise RuntimeError("cannot open the requested gap")
    off = brentq(lambda o: gap_for(o) - gap, 0.0, 60.0, xtol=1e-12, rtol=1e-14)
    gap_for(off)
    r = np.zeros((3, nR, nb, nb), dtype=np.complex128)
    # on-site dipoles (Hermitian), in-plane
    for d in (0, 1):
        D = (rng.uniform(-1, 1, (nb, nb)) + 1j * rng.uniform(-1, 1, (nb, nb))) * dipole_A
        D = 0.5 * (D + D.conj().T)
        np.fill_diagonal(D, 0.0)
        r[d, 0] = D
    r[0, 0, nb - 1, nb - 1] = a / math.sqrt(3)  # the one off-origin Wannier centre
    return uc, Rs, H, r


def random_model(nb, seed, shells=1, tmax=1.0, a=3.0, dims=2):
    """Small random Hermitian model for parity tests (nb bands, `shells`
    neighbour shells); centres at the origin except the last orbital."""
    rng = np.random.default_rng(seed)
    if dims == 3:
        uc = [[a, 0.1, 0.0], [0.2, a * 1.1, 0.0], [0.0, 0.3, a * 0.9]]
        base = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0)]
    elif dims == 1:
        uc = [[a, 0.0, 0.0], [0.0, 1000.0, 0.0], [0.0, 0.0, 1000.0]]
        base = [(1, 0, 0), (2, 0, 0)]
    else:
        uc = [[a * math.sqrt(3) / 2, a / 2, 0.0], [a * math.sqrt(3) / 2, -a / 2, 0.0], [0.0, 0.0, 20.0]]
        base = [(i, j, 0) for sh in _hex_shells()[:shells] for (i, j) in sh]
    Rs = [(0, 0, 0)]
    mats = [None]
    for v in base[: max(1, len(base) if dims != 2 else len(base))]:
        T = (rng.uniform(-1, 1, (nb, nb)) + 1j * rng.uniform(-1, 1, (nb, nb))) * tmax
        Rs.append(v)
        mats.append(T)
        Rs.append(tuple(-x for x in v))
        mats.append(T.conj().T)
    nR = len(Rs)
    H = np.zeros((nR, nb, nb), dtype=np.complex128)
    A0 = (rng.uniform(-1, 1, (nb, nb)) + 1j * rng.uniform(-1, 1, (nb, nb)))
    H[0] = 0.5 * (A0 + A0.conj().T) + np.diag(np.linspace(-4, 4, nb))
    for iR in range(1, nR):
        H[iR] = mats[iR]
    r = np.zeros((3, nR, nb, nb), dtype=np.complex128)
    for d in range(3):
        D = (rng.uniform(-1, 1, (nb, nb)) + 1j * rng.uniform(-1, 1, (nb, nb))) * 0.4
        D = 0.5 * (D + D.conj().T)
        np.fill_diagonal(D, 0.0)
        r[d, 0] = D
    r[0, 0, nb - 1, nb - 1] = 0.7
    return uc, Rs, H, r


# ---------------------------------------------------------------------------
def gaussian_laser(photon_eV, fwhm_fs, E0_au, centre_fs, pol=(1, 0, 0), phase=0.0):
    """Gaussian-envelope cos pulse: peak field E0 (a.u.) -> intensity E0^2 in a.u."""
    return {"intensity": E0_au ** 2, "intensity_units": "auintensity",
            "frequency": photon_eV, "frequency_units": "electronvolt",
            "polarization": list(pol), "t0": centre_fs, "t0_units": "fs", "phase": phase,
            "envelope": "gaussian", "fwhm": fwhm_fs, "fwhm_units": "fs", "cycles": 0}


def sin2_laser(photon_eV, intensity_wcm2, cycles, t0_fs=0.0, pol=(1, 0, 0)):
    return {"intensity": intensity_wcm2, "intensity_units": "wcm2", "frequency": photon_eV,
            "frequency_units": "electronvolt", "polarization": list(pol), "cycles": cycles,
            "t0": t0_fs, "t0_units": "fs"}


def _input(tb, grid, filled, dt_fs, nsteps, solver, lasers, coulomb=False, epsilon=1.0, r0_A=10.0):
    return {
        "tb_file": tb, "grid": list(grid), "filledbands": filled,
        "dt": dt_fs, "dt_units": "femtoseconds", "initialtime": 0, "initialtime_units": "femtoseconds",
        # Simulation::Propagate runs int((tf-ti)/dt)+2 steps; choose tf for `nsteps`
        "finaltime": dt_fs * (nsteps - 2) + dt_fs * 0.5, "finaltime_units": "femtoseconds",
        "solver": solver, "order": 4, "coulomb": coulomb, "epsilon": epsilon, "r0": [r0_A],
        "r0_units": "angstrom", "printresolution": 1, "printresolution_pulse": 1, "lasers": lasers,
    }


WORKLOADS = ("chain2", "hbn2", "tmd22", "tmd22_rk4")


def make(name: str, outdir: str, grid=None, nsteps=None):
    """Write the model of workload `name` in outdir; return the input dict."""
    os.makedirs(outdir, exist_ok=True)
    if name == "chain2":
        uc, Rs, H, r = chain_two_band()
        seed = os.path.join(outdir, "chain2")
        write_tb(seed + "_tb.dat", uc, Rs, H, r, "two-band linear chain")
        las = [gaussian_laser(1.5, 10.0, 0.01, 10.0)]
        return _input(seed, grid or (64, 1, 1), 1, 0.01, nsteps or 2000, "RK", las)
    if name == "hbn2":
        uc, Rs, H, r = hexagonal_two_band(t=-2.7)
        seed = os.path.join(outdir, "hbn2")
        write_tb(seed + "_tb.dat", uc, Rs, H, r, "hBN-like two-band model t=-2.7 eV")
        las = [gaussian_laser(2.0, 10.0, 0.01, 10.0)]
        return _input(seed, grid or (120, 120, 1), 1, 0.01, nsteps or 2000, "RK", las)
    if name in ("tmd22", "tmd22_rk4"):
        g = tuple(grid or (72, 72, 1))
        uc, Rs, H, r = tmd_like(grid=g)
        seed = os.path.join(outdir, f"tmd22_{g[0]}x{g[1]}")
        write_tb(seed + "_tb.dat", uc, Rs, H, r, "22-orbital TMD-like model, seed 1234, gap 1.8 eV")
        las = [gaussian_laser(1.5, 10.0, 0.005, 10.0)]
        solver = "AB" if name == "tmd22" else "RK"
        return _input(seed, g, 11, 0.005, nsteps or 4000, solver, las, coulomb=True, epsilon=1.0, r0_A=40.0)
    raise KeyError(name)


def hbn_golden_input(tb_seed: str) -> dict:
    """The reference's ci-test/inputs/hBN.json.in with the model path filled in."""
    return {
        "tb_file": tb_seed, "fermienergy": 0, "fermienergy_units": "electronvolt", "coulomb": False,
        "epsilon": 2.0, "r0": 10, "grid": [50, 50, 1], "filledbands": 1, "dt": 0.01,
        "dt_units": "femtoseconds", "printresolution": 1, "printresolution_pulse": 1,
        "initialtime": 0, "initialtime_units": "femtoseconds", "finaltime": 1,
        "finaltime_units": "femtoseconds", "solver": "RK", "order": 4,
        "lasers": [{"intensity": 1e10, "intensity_units": "wcm2", "frequency": 10,
                    "frequency_units": "electronvolt", "polarization": [1, 1, 0], "cycles": 1,
                    "t0": 0.0, "t0_units": "fs"}],
    }


def save_input(d: dict, path: str):
    with open(path, "w") as f:
        json.dump(d, f, indent=2)


# ---------------------------------------------------------------------------
# Batched laser sweep: solves of uneven band count and k grid, each a seeded
# random tight-binding model (IPA, RK4) under its own Gaussian pulse.
SWEEP_BANDS = (2, 4, 8, 14, 22)
SWEEP_SIDES = (24, 36, 48, 72, 96)


def sweep_specs(n: int = 256, seed: int = 2024):
    """n solves: band count and square grid side drawn from SWEEP_BANDS and
    SWEEP_SIDES, photon energy uniform in [1, 3] eV, peak field log-uniform in
    [1e-4, 2e-2] a.u., a model seed each."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        out.append(dict(nb=int(rng.choice(SWEEP_BANDS)), N=int(rng.choice(SWEEP_SIDES)),
                        model_seed=int(rng.integers(1 << 30)), photon_eV=float(rng.uniform(1.0, 3.0)),
                        E0_au=float(10.0 ** rng.uniform(-4.0, math.log10(2e-2)))))
    return out


def sweep_input(spec: dict, outdir: str, dt_fs: float = 0.005, nsteps: int = 1000):
    """input.json dict of one sweep solve (its model file written in outdir)."""
    os.makedirs(outdir, exist_ok=True)
    nb, N = spec["nb"], spec["N"]
    uc, Rs, H, r = random_model(nb, spec["model_seed"])
    seed = os.path.join(outdir, f"sweep_{nb}_{spec['model_seed']}")
    write_tb(seed + "_tb.dat", uc, Rs, H, r, f"random {nb}-band model, seed {spec['model_seed']}")
    las = [gaussian_laser(spec["photon_eV"], 2.0, spec["E0_au"], 2.5, pol=(1.0, 0.3, 0.0))]
    return _input(seed, (N, N, 1), max(1, nb // 2), dt_fs, nsteps, "RK", las)
