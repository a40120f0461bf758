"""Build the reference's own propagator into oracle/_ref/EDUS (test infrastructure).

    python oracle/build_ref.py            # needs the reference sources
    EDUS_REFERENCE_DIR=/path/to/EDUS_2.0 python oracle/build_ref.py

The reference (gcistaro/EDUS_2.0) is compiled unchanged, from its sources where
they lie, with g++ -- not with its CMake project.  It needs MKL, FFTW3(-mpi)
and MPI, none of which exist on this image, so the build puts the project's
own stand-ins first on the include path (oracle/refshim/: one MPI rank, the
FFTW interface over the oracle's mixed-radix FFT, and the CBLAS/LAPACKE subset
the reference calls) and links their implementation (oracle/refshim/shims.cpp).
The three headers that CMake generates (core/githash.hpp, core/projectdir.hpp,
InputVariables/input_schema.hpp) are generated here into oracle/_ref/gen/.
Flags follow the reference's defaults for a one-process run: EDUS_MPI and
EDUS_PROFILE on, EDUS_HDF5 off (no HDF5 library), OpenMP on.

The binary reads the reference's input.json and writes its text outputs
(Population.txt, Velocity.txt, ...) into the working directory; tests compare
them with the oracle restatement.  Nothing in the product uses it.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
GEN = os.path.join(OUT, "gen")
OBJ = os.path.join(OUT, "obj")
SHIM = os.path.join(HERE, "refshim")
EXE = os.path.join(OUT, "EDUS")

# the library sources of the reference's CMakeLists.txt (_SOURCES) plus its main
SOURCES = [
    "initialize.cpp", "GlobalFunctions.cpp", "core/print_header.cpp", "ConvertUnits.cpp", "ostream.cpp",
    "StreamFile.cpp", "InputVariables/simulation_parameters.cpp", "Geometry/Matrix.cpp",
    "Geometry/Coordinate.cpp", "MeshGrid/MeshGrid.cpp", "Wannier/Wannier.cpp", "Wannier/ReadWannier.cpp",
    "Wannier/PrintWannier.cpp", "Laser/Laser.cpp", "fftPair/fftPair.cpp", "kGradient/kGradient.cpp",
    "DESolver/DESolver.cpp", "Simulation/Simulation.cpp", "core/profiler.cpp", "core/print_timing.cpp",
    "core/cmd_args/cmd_args.cpp", "core/rt_graph.cpp", "core/mpi/Communicator.cpp", "Coulomb/Coulomb.cpp",
    "Screened_potential/Screened_potential.cpp", "GreenFunction/GreenFunction.cpp",
    "ModelCoulomb/ModelCoulomb.cpp", "EDUS.cpp",
]
CXXFLAGS = ["-O3", "-DNDEBUG", "-fopenmp", "-std=c++17", "-DEDUS_MPI", "-DEDUS_PROFILE", "-w"]


def _candidate() -> str:
    return os.environ.get("EDUS_REFERENCE_DIR", "/root/reference")


def reference_available() -> bool:
    return os.path.isdir(os.path.join(_candidate(), "src"))


def reference_dir() -> str:
    ref = _candidate()
    if not reference_available():
        raise SystemExit(f"reference sources not found under {ref!r} (set EDUS_REFERENCE_DIR)")
    return ref


def write_if_changed(path: str, text: str) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    if os.path.exists(path) and open(path).read() == text:
        return
    with open(path, "w") as f:
        f.write(text)


def generate_headers(ref: str) -> None:
    write_if_changed(os.path.join(GEN, "core", "githash.hpp"),
                     '#ifndef GIT_HASH\n#define GIT_HASH\n'
                     'const char* const git_hash = "reference sources, project shims";\n'
                     'const char* const git_branchname = "";\n'
                     'const char* const build_date = "";\n#endif\n')
    write_if_changed(os.path.join(GEN, "core", "projectdir.hpp"),
                     f'#ifndef PROJECT_DIR\n#define PROJECT_DIR\nconst char* const ProjectDirectory = "{ref}";\n'
                     '#endif\n')
    schema = open(os.path.join(ref, "src", "InputVariables", "input_schema.json")).read()
    write_if_changed(os.path.join(GEN, "input_schema.hpp"),
                     'namespace EDUS {\n\n#pragma once\nconst nlohmann::json input_schema = R"schema(\n'
                     + schema + '\n)schema"_json;\n\n};\n')


def compile_one(cxx: str, src: str, obj: str, includes: list[str]) -> tuple[str, int, str]:
    os.makedirs(os.path.dirname(obj), exist_ok=True)
    deps = [src] + [os.path.join(SHIM, h) for h in os.listdir(SHIM)]
    deps += [os.path.join(HERE, "oracle_fft.hpp"), os.path.join(HERE, "oracle_linalg.hpp")]
    if os.path.exists(obj) and all(os.path.getmtime(d) <= os.path.getmtime(obj) for d in deps):
        return src, 0, ""
    cmd = [cxx, *CXXFLAGS, *[f"-I{i}" for i in includes], "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r.returncode, r.stderr


def build() -> str:
    ref = reference_dir()
    generate_headers(ref)
    cxx = "g++"
    includes = [SHIM, GEN, os.path.join(ref, "src")]
    jobs = [(os.path.join(ref, "src", s), os.path.join(OBJ, s.replace("/", "_") + ".o")) for s in SOURCES]
    jobs.append((os.path.join(SHIM, "shims.cpp"), os.path.join(OBJ, "refshim_shims.o")))
    failed = []
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for src, rc, err in ex.map(lambda j: compile_one(cxx, j[0], j[1], includes), jobs):
            if rc:
                failed.append(src)
                sys.stderr.write(f"--- {src}\n{err}\n")
    if failed:
        raise SystemExit(f"reference build failed in {len(failed)} file(s)")
    objs = [o for _, o in jobs]
    if not os.path.exists(EXE) or any(os.path.getmtime(o) > os.path.getmtime(EXE) for o in objs):
        subprocess.run([cxx, "-fopenmp", "-o", EXE, *objs], check=True)
    return EXE


if __name__ == "__main__":
    print(build())
