"""Pin the CPU oracle to outputs of the reference's own propagator (CPU).

The reference (gcistaro/EDUS_2.0) was compiled from its unchanged sources
against the project's MPI / FFTW / MKL stand-ins (oracle/build_ref.py) and run
on the cases of tests/golden/ref_cases.py; tests/golden/make_ref_outputs.py
stored its Population.txt, Population_wannier.txt, Velocity.txt, Laser.txt and
Time.txt under tests/golden/ref/<case>/.  These cover the HSEX path of the
benchmark workload (Hartree + Fock with the Rytova-Keldysh W, the cumulative
centre quirk), RK4 / AB4 / AB5, even and odd grids, 2 to 13 bands, the k-space
gradient and the Peierls gauge.

The oracle must reproduce every printed column at ci-test/compare.py's 1e-10;
populations are printed with 14 significant digits, velocities with 8.  The
stand-ins are checked first: the same build reproduces the reference's own
checked-in hBN outputs (ci-test/outputs/hBN), see test_reference_build_*.
"""
import json
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN

sys.path.insert(0, GOLDEN)
import ref_cases  # noqa: E402

REF = os.path.join(GOLDEN, "ref")


def _oracle_outputs(po, pkg, case, tmp_path, **override):
    seed = ref_cases.write_model(pkg.workloads, case, str(tmp_path))
    inp = ref_cases.make_input(case, seed)
    inp.update(override)
    cfg = po.load_input(inp)
    o = po.Oracle(cfg)
    rows = {"Population.txt": [], "Population_wannier.txt": [], "Velocity.txt": [], "Laser.txt": [], "Time.txt": []}
    for _ in range(cfg.nsteps):
        pb, pw, v = o.observables()
        rows["Population.txt"].append(pb)
        rows["Population_wannier.txt"].append(pw)
        rows["Velocity.txt"].append(v)
        rows["Laser.txt"].append(o.efield(o.time))
        rows["Time.txt"].append(o.time)
        o.step(1)
    return seed, {k: np.array(v) for k, v in rows.items()}


def _load(name, fn):
    a = np.loadtxt(os.path.join(REF, name, fn))
    return a


# cases sized for the GPU only (the benchmark model at full size) are left to
# tests/test_gpu_cli.py: the CPU oracle would take minutes on them
CPU_CASES = sorted(n for n, c in ref_cases.CASES.items() if not c.get("gpu_only"))


@pytest.mark.parametrize("name", CPU_CASES)
def test_oracle_matches_reference(po, pkg, tmp_path, name):
    case = ref_cases.CASES[name]
    meta = json.load(open(os.path.join(REF, name, "meta.json")))
    seed, got = _oracle_outputs(po, pkg, case, tmp_path)
    # the model the reference read is the one regenerated here
    assert ref_cases.sha256(seed + "_tb.dat") == meta["model_sha256"]
    assert meta["input"]["coulomb"] == case["coulomb"]
    for fn in ("Population.txt", "Population_wannier.txt", "Velocity.txt"):
        ref = _load(name, fn)
        assert ref.shape == got[fn].shape, fn
        err = np.abs(ref - got[fn]).max()
        assert err < 1e-10, f"{name} {fn}: max |oracle - reference| = {err:.3e}"
    # Laser.txt: E(t) at the printed times (8 printed digits in the reference)
    las = _load(name, "Laser.txt")
    assert np.allclose(got["Laser.txt"], las, rtol=1e-7, atol=1e-14)
    t = _load(name, "Time.txt")
    assert np.allclose(got["Time.txt"], t, rtol=1e-5, atol=1e-12)


@pytest.mark.parametrize("name", [n for n in CPU_CASES if ref_cases.CASES[n]["coulomb"]])
def test_reference_outputs_depend_on_hsex(po, pkg, tmp_path, name):
    """The pin has teeth: the same run without the HSEX term misses the
    reference's populations by far more than the tolerance."""
    _, ipa = _oracle_outputs(po, pkg, ref_cases.CASES[name], tmp_path, coulomb=False)
    ref = _load(name, "Population.txt")
    assert np.abs(ref - ipa["Population.txt"]).max() > 1e-7


REF_EXE = os.path.join(os.path.dirname(GOLDEN), os.pardir, "oracle", "_ref", "EDUS")


def _run_reference(inp, d):
    import subprocess

    with open(os.path.join(d, "input.json"), "w") as f:
        json.dump(inp, f)
    r = subprocess.run([os.path.abspath(REF_EXE), "input.json"], cwd=d, capture_output=True, text=True,
                       env=dict(os.environ, OMP_NUM_THREADS="4"), timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return os.path.join(d, "Output")


@pytest.mark.skipif(not os.path.exists(REF_EXE), reason="oracle/_ref/EDUS not built (oracle/build_ref.py)")
def test_reference_build_reproduces_checked_in_hbn_outputs(pkg, hbn_golden_model, tmp_path):
    """The stand-ins do not move the reference's answer: the stand-in build of
    the reference reproduces the reference's own checked-in outputs of its
    hBN integration test (ci-test/outputs/hBN) at compare.py's 1e-10.  The
    input is ci-test/inputs/hBN.json.in with r0 as a list (the current schema
    rejects the bare number that file still has)."""
    inp = pkg.workloads.hbn_golden_input(hbn_golden_model)
    inp["r0"] = [inp["r0"]]
    out = _run_reference(inp, str(tmp_path))
    for fn in ("Population.txt", "Velocity.txt", "Laser.txt", "Time.txt"):
        got = np.loadtxt(os.path.join(out, fn))
        gold = np.loadtxt(os.path.join(GOLDEN, "hBN", fn))
        assert got.shape == gold.shape, fn
        assert np.abs(got - gold).max() < 1e-10, fn


@pytest.mark.skipif(not os.path.exists(REF_EXE), reason="oracle/_ref/EDUS not built (oracle/build_ref.py)")
def test_reference_build_reproduces_fixture(pkg, tmp_path):
    """The committed fixtures are what the current build of the reference prints."""
    name = "rand4_rk4"
    case = ref_cases.CASES[name]
    seed = ref_cases.write_model(pkg.workloads, case, str(tmp_path))
    out = _run_reference(ref_cases.make_input(case, seed), str(tmp_path))
    for fn in ref_cases.OUTPUTS:
        assert np.array_equal(np.loadtxt(os.path.join(out, fn)), _load(name, fn)), fn
