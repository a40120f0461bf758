"""Run the reference's own propagator on the cases of ref_cases.py and store its outputs.

    EDUS_REFERENCE_DIR=/path/to/EDUS_2.0 python tests/golden/make_ref_outputs.py [case ...]

Builds oracle/_ref/EDUS (oracle/build_ref.py: the reference's unchanged sources
compiled with g++ against the project's MPI / FFTW / MKL stand-ins), runs it
once per case in a scratch directory, and copies the text outputs it writes
(Output/Population.txt, Population_wannier.txt, Velocity.txt, Laser.txt,
Time.txt) into tests/golden/ref/<case>/, with meta.json recording the input
and the SHA-256 of the model file the reference read.  Run it where the
reference sources are available; the tests only read the stored files.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import ref_cases  # noqa: E402


def main(names: list[str]) -> None:
    import build_ref  # oracle/build_ref.py

    import __graft_entry__ as ge

    workloads = ge.load_package().workloads
    exe = build_ref.build()
    names = names or list(ref_cases.CASES)
    for name in names:
        case = ref_cases.CASES[name]
        out = os.path.join(HERE, "ref", name)
        with tempfile.TemporaryDirectory() as d:
            seed = ref_cases.write_model(workloads, case, d)
            inp = ref_cases.make_input(case, seed)
            with open(os.path.join(d, "input.json"), "w") as f:
                json.dump(inp, f, indent=2)
            env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))
            r = subprocess.run([exe, "input.json"], cwd=d, capture_output=True, text=True, env=env)
            if r.returncode != 0:
                sys.stderr.write(r.stdout[-4000:] + r.stderr[-4000:])
                raise SystemExit(f"{name}: the reference exited with {r.returncode}")
            os.makedirs(out, exist_ok=True)
            for fn in ref_cases.OUTPUTS:
                shutil.copyfile(os.path.join(d, "Output", fn), os.path.join(out, fn))
            inp["tb_file"] = "model"
            meta = {"case": name, "input": inp, "model_sha256": ref_cases.sha256(seed + "_tb.dat"),
                    "built_by": "oracle/build_ref.py (reference sources, project MPI/FFTW/MKL stand-ins)"}
            with open(os.path.join(out, "meta.json"), "w") as f:
                json.dump(meta, f, indent=2)
        print(f"{name}: {out}")


if __name__ == "__main__":
    main(sys.argv[1:])
