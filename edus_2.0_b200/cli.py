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
of the state rho(R) e^{-iA.R}, Simulation.cpp:447-449, 593-595).  Differences from
the reference: the vector potential integrates the total field of all lasers
(the reference's accumulator is a function-static shared by every laser, which
only agrees for a single laser); output.h5 is not written.
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import sys


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


def run(input_path: str, outdir: str, device: int = 0) -> int:
    """Propagate and write the text outputs; returns the number of steps."""
    pkg = _package()
    cfg = pkg.model.parse_input(input_path)
    m = pkg.model.Model(cfg)
    s = m.solver(device=device)
    s.upload_observables(U=m.U, vel=m.velocity())
    os.makedirs(outdir, exist_ok=True)
    names = ("Time", "Laser", "Laser_A", "Population", "Population_wannier", "Velocity")
    files = {n: open(os.path.join(outdir, n + ".txt"), "w") for n in names}
    dt = cfg.dt
    pr = max(1, int(cfg.printresolution_pulse))
    nsteps = cfg.nsteps
    A = [0.0, 0.0, 0.0]
    t_prev = 0.0
    try:
        t = s.time  # the library's CurrentTime: accumulated by += dt, as DESolver does
        it = 0
        while it < nsteps:
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
            while it + n < nsteps and int(round(tn / dt)) % pr != 0:
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
