"""Inputs of the reference runs whose outputs are committed under tests/golden/ref/.

Each case is a seeded model (written with the package's `_tb.dat` writer) and
an input.json for it, in the reference's own schema.  The reference binary
(oracle/_ref/EDUS, built by oracle/build_ref.py from the reference's unchanged
sources) ran each one; tests/golden/make_ref_outputs.py stored its text
outputs.  The tests regenerate the same model and input, check the model
file's SHA-256 against the one the reference read, and compare the oracle (on
the CPU) and the GPU product (through its command line) with those outputs.

The reference has only the sin^2 pulse, so every case uses it.  The cases
cover what the headline workload runs and the benchmark-free paths beside it:
HSEX (the Hartree and Fock terms with the Rytova-Keldysh W, including the
cumulative-centre quirk of ModelCoulomb.cpp:76-79: orbitals off the origin),
RK4, AB4 and AB5, even and odd grids, 2 to 13 bands, the k-space gradient and
the Peierls gauge.
"""
from __future__ import annotations

import hashlib
import math
import os

# name -> (model, grid, filledbands, dt_fs, nsteps, solver, order, laser, extra)
#   model: ("hbn",) the reference's hBN model (tb_models/hBN_gap7.25eV_a2.5A),
#          ("random", nb, seed, shells)  workloads.random_model
#   laser: (photon_eV, intensity_wcm2, cycles, t0_fs, polarization)
CASES = {
    # the reference's own HSEX test input (ci-test/inputs/hBN_coulomb.json.in)
    # with r0 given as a list, which the current schema requires
    "hbn_coulomb": dict(model=("hbn",), grid=(40, 40, 1), filled=1, dt=0.01, nsteps=102, solver="RK", order=4,
                        laser=(10.0, 1e10, 1, 0.0, (1, 1, 0)), coulomb=True, epsilon=2.0, r0=10.0),
    # strong resonant pulse: excitation large enough that HSEX moves the populations
    "hbn_coulomb_strong": dict(model=("hbn",), grid=(24, 24, 1), filled=1, dt=0.01, nsteps=160, solver="RK",
                               order=4, laser=(8.0, 5e12, 3, 0.0, (1, 0.5, 0)), coulomb=True, epsilon=1.0,
                               r0=20.0),
    "rand4_rk4": dict(model=("random", 4, 11, 2), grid=(12, 12, 1), filled=2, dt=0.01, nsteps=80, solver="RK",
                      order=4, laser=(3.0, 2e12, 2, 0.0, (1, 0.3, 0)), coulomb=True, epsilon=1.0, r0=15.0),
    "rand5_ab4_odd": dict(model=("random", 5, 12, 2), grid=(9, 11, 1), filled=2, dt=0.005, nsteps=120,
                          solver="AB", order=4, laser=(2.5, 3e12, 2, 0.0, (0.4, 1, 0)), coulomb=True,
                          epsilon=1.5, r0=30.0),
    "rand13_ab5": dict(model=("random", 13, 13, 1), grid=(8, 6, 1), filled=6, dt=0.005, nsteps=60, solver="AB",
                       order=5, laser=(2.0, 1e12, 2, 0.0, (1, 0, 0)), coulomb=True, epsilon=1.0, r0=40.0),
    "rand3_ipa_rk4": dict(model=("random", 3, 14, 2), grid=(10, 7, 1), filled=1, dt=0.01, nsteps=60, solver="RK",
                          order=4, laser=(2.0, 2e12, 2, 0.0, (1, 1, 0)), coulomb=False, epsilon=1.0, r0=10.0),
    "hbn_kgrad": dict(model=("hbn",), grid=(12, 12, 1), filled=1, dt=0.01, nsteps=80, solver="RK", order=4,
                      laser=(8.0, 5e12, 2, 0.0, (1, 0.5, 0)), coulomb=False, epsilon=1.0, r0=10.0,
                      gradient_space="k"),
    "rand4_peierls_hsex": dict(model=("random", 4, 15, 1), grid=(10, 10, 1), filled=2, dt=0.01, nsteps=60,
                               solver="RK", order=4, laser=(3.0, 2e12, 2, 0.0, (1, 0.3, 0)), coulomb=True,
                               epsilon=1.0, r0=15.0, peierls=True),
    # the benchmark's own model at full size (22 orbitals, 72 x 72, HSEX with the
    # Rytova-Keldysh W at r0 = 40 A, RK4 at 0.005 fs), 40 steps from the middle of
    # a strong one-cycle 2.5 eV sin^2 pulse (above the 1.8 eV gap; t0 = -T/2, so
    # the envelope peaks at t = 0); too large for the CPU oracle in the CPU
    # suite, so checked on the GPU only
    "tmd22_72_rk4": dict(model=("tmd22",), grid=(72, 72, 1), filled=11, dt=0.005, nsteps=40, solver="RK",
                         order=4, laser=(2.5, 5e13, 1, -0.827, (1, 0.5, 0)), coulomb=True, epsilon=1.0,
                         r0=40.0, gpu_only=True),
    # the same model with the stepper of that configuration, Adams-Bashforth 4
    # (cold history), 80 steps, at 2e12 W/cm2: the gradient term's largest rate,
    # E R_max ~ E 216 bohr, times dt must stay inside AB4's stability interval
    # on the imaginary axis (the 5e13 W/cm2 pulse above makes the reference's
    # own AB4 run diverge after 40 steps)
    "tmd22_72_ab4": dict(model=("tmd22",), grid=(72, 72, 1), filled=11, dt=0.005, nsteps=80, solver="AB",
                         order=4, laser=(2.5, 2e12, 1, -0.827, (1, 0.5, 0)), coulomb=True, epsilon=1.0,
                         r0=40.0, gpu_only=True),
}

OUTPUTS = ("Population.txt", "Population_wannier.txt", "Velocity.txt", "Laser.txt", "Time.txt")


def write_model(workloads, case: dict, outdir: str) -> str:
    """Write the case's model file in outdir; return its seed path (no `_tb.dat`)."""
    m = case["model"]
    if m[0] == "tmd22":
        uc, Rs, H, r = workloads.tmd_like(grid=tuple(case["grid"]))
        title = "22-orbital TMD-like model, seed 1234, gap 1.8 eV"
    elif m[0] == "hbn":
        uc, Rs, H, r = workloads.hexagonal_two_band(a=2.5, onsite=3.625, t=-2.3, centre=1.44337567297406441)
        title = "hBN two-band model, a = 2.5 A, gap 7.25 eV"
    else:
        _, nb, seed, shells = m
        uc, Rs, H, r = workloads.random_model(nb, seed, shells=shells)
        title = f"random {nb}-band model, seed {seed}"
    seed_path = os.path.join(outdir, "model")
    workloads.write_tb(seed_path + "_tb.dat", uc, Rs, H, r, title)
    return seed_path


def make_input(case: dict, tb_seed: str) -> dict:
    """The reference's input.json for the case (every step printed)."""
    ph, inten, cyc, t0, pol = case["laser"]
    n = case["nsteps"]
    d = {
        "tb_file": tb_seed, "grid": list(case["grid"]), "filledbands": case["filled"],
        "dt": case["dt"], "dt_units": "femtoseconds", "initialtime": 0, "initialtime_units": "femtoseconds",
        # Simulation::Propagate runs int((tf - ti)/dt) + 2 steps
        "finaltime": case["dt"] * (n - 2) + case["dt"] * 0.5, "finaltime_units": "femtoseconds",
        "solver": case["solver"], "order": case["order"], "coulomb": case["coulomb"],
        "epsilon": case["epsilon"], "r0": [case["r0"]], "r0_units": "angstrom",
        "printresolution": 1, "printresolution_pulse": 1,
        "lasers": [{"intensity": inten, "intensity_units": "wcm2", "frequency": ph,
                    "frequency_units": "electronvolt", "polarization": list(pol), "cycles": cyc,
                    "t0": t0, "t0_units": "fs"}],
    }
    if "gradient_space" in case:
        d["gradient_space"] = case["gradient_space"]
    if case.get("peierls"):
        d["peierls"] = True
    return d


def sha256(path: str) -> str:
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()
