"""Command-line propagation of a reference input.json on the GPU.

    python edus_2.0_b200/cli.py input.json [--outdir DIR] [--device N]

Reads the reference's input schema (model.parse_input), sets the simulation up
as Simulation's constructor does (model.Model: H0(k), r(k), eigensystem,
initial condition, HSEX arrays), propagates `int((tf - ti)/dt) + 2` steps
(Simulation::Propagate, Simulation.cpp:352-375) with the FP64 form, and writes
the text outputs of Simulation::do_onestep (Simulation.cpp:381-432) before
each step whose time t has int(round(t/dt)) % printresolution_pulse == 0
(PrintObservables with use_sparse = false, Simulation.cpp:240-257):

    Time.txt                t (a.u.)
    Laser.txt               E(t), Cartesian (a.u.)
    Laser_A.txt             the vector potential, integrated by Simpson's rule
                            from one printed time to the next (Laser.cpp:136-151);
                            in the Peierls gauge every stage time is a step of the
                            same integrator, as there the source term requests A too
    Population.txt          Bloch populations, holes of the filled bands
    Population_wannier.txt  Wannier populations
    Velocity.txt            re, im of the x, y, z velocity

The observables are computed on the GPU (edus_observables; in the Peierls gauge
of the state rho(R) e^{-iA.R}, Simulation.cpp:447-449, 593-595).

output.h5 (Simulation.cpp:202-233, 384-416; GlobalFunctions.cpp:22-66) is written
by the package's own HDF5 writer (h5.py) in the reference's layout:

    json/...                         the input (tb_file, coulomb, grid, filledbands,
                                     dt, printresolution, initialtime, finaltime,
                                     num_bands, num_kpoints, solver, laser<i>/...,
                                     kpoints, A, B) as dump_json_in_h5 writes it
    fullH, DensityMatrix_k,          per printed step <it> (0, 1, ...):
    DensityMatrix_k_bloch,           <node>/<it>/0/local, the [k][n][m] complex
    SelfEnergy                       matrix as 2 Nk nb^2 doubles, for the
                                     quantities that "toprint" selects
    time_au/<it>                     CurrentTime of print <it>

A step is printed there when int(round(t/dt)) % r == 0 with r = the pulse print
resolution inside any laser's window and printresolution outside it
(PrintObservables(t, true), Simulation.cpp:236-257).  The Gaussian-envelope
lasers (an extension) count t0 +- 3 fwhm as their window.

Differences from the reference: the vector potential integrates the total field
of all lasers (the reference's accumulator is a function-static shared by every
laser, which only agrees for a single laser).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys

import numpy as np


def _package():
    if "edus_b200" in sys.modules:
        return sys.modules["edus_b200"]
    here = os.path.dirname(os.path.abspath(__file__))
    spec = importlib.util.spec_from_file_location("edus_b200", os.path.join(here, "__init__.py"),
                                                  submodule_search_locations=[here])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["edus_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


TOPRINT = {"DMk_wannier": "DensityMatrix_k", "DMk_bloch": "DensityMatrix_k_bloch", "fullH": "fullH",
           "SelfEnergy": "SelfEnergy"}


def _raw_input(input_path: str, pkg) -> dict:
    with open(input_path) as f:
        user = json.load(f)
    d = dict(pkg.model.SCHEMA_DEFAULTS)
    d.update({k: v for k, v in user.items() if k != "lasers"})
    d["lasers"] = [dict(pkg.model.LASER_DEFAULTS, **L) for L in user.get("lasers", [])]
    d["toprint"] = dict({k: "false" for k in TOPRINT}, **user.get("toprint", {}))
    return d


def _h5_json(h5, raw: dict, m) -> None:
    """dump_json_in_h5 (GlobalFunctions.cpp:22-66); "polarization" of each laser
    receives its "cycles", as the reference writes it."""
    j = h5.group("json")
    j.write("tb_file", str(raw["tb_file"]))
    j.write("coulomb", int(bool(raw["coulomb"])))
    j.write("grid", np.array([int(x) for x in raw["grid"]], dtype=np.int32))
    j.write("filledbands", int(raw["filledbands"]))
    j.write("dt", float(raw["dt"]))
    j.write("printresolution", int(raw["printresolution"]))
    j.write("initialtime", float(raw["initialtime"]))
    j.write("finaltime", float(raw["finaltime"]))
    j.write("num_bands", int(m.nb))
    j.write("num_kpoints", int(m.Nk))
    j.write("solver", str(raw["solver"]))
    for i, L in enumerate(raw["lasers"]):
        g = j.group(f"laser{i}")
        g.write("intensity", float(L["intensity"]))
        g.write("frequency", float(L["frequency"]))
        g.write("wavelength", float(L["wavelength"]))
        g.write("cycles", int(L["cycles"]))
        g.write("polarization", int(L["cycles"]))
    # bare k (crystal coordinates, ix / N) and the bases (Simulation.cpp:207-216)
    N = m.grid
    idx = np.indices(N).reshape(3, -1).T
    j.write("kpoints", (idx / np.array(N, dtype=float)).reshape(-1))
    j.write("A", m.A.reshape(-1))
    j.write("B", (2.0 * np.pi * np.linalg.inv(m.A).T).reshape(-1))


def _in_pulse(t: float, lasers) -> bool:
    pkg = _package()
    for L in lasers:
        if L.envelope == pkg.edus.ENVELOPE_SIN2:
            t1 = L.t0 + L.cycles * 2.0 * np.pi / L.omega
            if L.t0 + 1e-7 < t < t1 + 1e-7:
                return True
        elif abs(t - L.t0) < 3.0 * L.fwhm:
            return True
    return False


def _self_energy_k(m, rho_k):
    """Coulomb::EffectiveHamiltonian with H erased (Coulomb.cpp:134-180), to k."""
    pkg = _package()
    rR = pkg.model.fft_k_to_R(rho_k, m.grid)
    sig = -m.W * (rR - m.DM0R)
    d = np.diagonal(rR[0]) - np.diagonal(m.DM0R[0])
    sig[0][np.diag_indices(m.nb)] += m.hartree @ d
    return pkg.model.fft_R_to_k(sig, m.grid)


def run(input_path: str, outdir: str, device: int = 0) -> int:
    """Propagate and write the text outputs and output.h5; returns the number of steps."""
    pkg = _package()
    cfg = pkg.model.parse_input(input_path)
    raw = _raw_input(input_path, pkg)
    m = pkg.model.Model(cfg)
    s = m.solver(device=device)
    s.upload_observables(U=m.U, vel=m.velocity())
    os.makedirs(outdir, exist_ok=True)
    names = ("Time", "Laser", "Laser_A", "Population", "Population_wannier", "Velocity")
    files = {n: open(os.path.join(outdir, n + ".txt"), "w") for n in names}
    h5 = pkg.h5.H5Tree()
    _h5_json(h5, raw, m)
    for node in ("fullH", "DensityMatrix_k", "DensityMatrix_k_bloch", "SelfEnergy", "time_au"):
        h5.group(node)
    wanted = [k for k in TOPRINT if str(raw["toprint"].get(k, "false")).lower() == "true"]
    if "SelfEnergy" in wanted and not cfg.coulomb:
        wanted.remove("SelfEnergy")  # no self-energy without HSEX: nothing to write
    dt = cfg.dt
    pr = max(1, int(cfg.printresolution_pulse))
    pr_out = max(1, int(cfg.printresolution))
    nsteps = cfg.nsteps
    A = [0.0, 0.0, 0.0]
    t_prev = 0.0
    it_h5 = 0

    def h5_due(t):
        r = pr if _in_pulse(t, cfg.lasers) else pr_out
        return int(round(t / dt)) % r == 0

    try:
        t = s.time  # the library's CurrentTime: accumulated by += dt, as DESolver does
        it = 0
        while it < nsteps:
            if h5_due(t):
                # Simulation::do_onestep (Simulation.cpp:384-416)
                node = str(it_h5)
                rho = s.get_state() if wanted else None
                for key in wanted:
                    if key == "DMk_wannier":
                        mat = rho
                    elif key == "DMk_bloch":
                        mat = np.einsum("kji,kjl,klm->kim", m.U.conj(), rho, m.U)
                    elif key == "fullH":
                        E = s.efield(t)
                        mat = m.H0k + E[0] * m.xik[0] + E[1] * m.xik[1] + E[2] * m.xik[2]
                    else:
                        mat = _self_energy_k(m, rho)
                    h5[TOPRINT[key]].group(node).group("0").write("local", np.ascontiguousarray(mat))
                h5["time_au"].write(node, float(t))
                it_h5 += 1
            if int(round(t / dt)) % pr == 0:
                E = s.efield(t)
                if cfg.peierls:
                    A = list(s.vector_potential(t))
                else:
                    dT = t - t_prev
                    if dT >= 1e-7:
                        E1, E2 = s.efield(t_prev), s.efield(t_prev + dT / 2.0)
                        A = [A[d] - dT / 6.0 * (E1[d] + 4.0 * E2[d] + E[d]) for d in range(3)]
                        t_prev = t
                pb, pw, v = s.observables(0, cfg.filledbands)
                files["Time"].write(f"{t:g}\n")
                files["Laser"].write("".join(f"{x:24.15g}" for x in E) + "\n")
                files["Laser_A"].write("".join(f"{x:24.15g}" for x in A) + "\n")
                files["Population"].write("".join(f"{x:30.14g} " for x in pb) + "\n")
                files["Population_wannier"].write("".join(f"{x:30.14g} " for x in pw) + "\n")
                files["Velocity"].write("".join(f"{x:20.8g}" for c in v for x in (c.real, c.imag)) + "\n")
            # step to the next printed time (or the end) in one call
            n = 1
            tn = t + dt
            while it + n < nsteps and int(round(tn / dt)) % pr != 0 and not h5_due(tn):
                n += 1
                tn += dt
            s.step(n)
            it += n
            t = tn
            if abs(s.time - t) > 0.0:
                raise RuntimeError("host and device CurrentTime diverged")
    finally:
        for f in files.values():
            f.close()
    s.synchronize()
    h5.save(os.path.join(outdir, "output.h5"))
    return nsteps


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("input", help="input.json in the reference's schema")
    ap.add_argument("--outdir", default=None, help="output directory (default: Output/ beside the input)")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    out = a.outdir or os.path.join(os.path.dirname(os.path.abspath(a.input)), "Output")
    n = run(a.input, out, a.device)
    print(f"{n} steps, outputs in {out}")


if __name__ == "__main__":
    main()
