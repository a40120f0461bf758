"""bench.py's form bookkeeping (CPU): which form the line names as the fastest
within 1e-8 of plain FP64, and the command-line switches that select the
workload, the grid and the form of the timed loop."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_best_form_prefers_the_fastest_form_within_the_bar():
    forms = {
        "batched_fp64": {"max_abs_drho": 0.0},
        "batched_hplanes": {"solve_steps_per_s": 1858.2, "max_abs_drho": 1e-14, "meets_1e-8": True},
        "split32": {"steps_per_s": 1000.0, "max_abs_drho": 1e-6, "meets_1e-8": False},
        "hplanes": {"steps_per_s": 1500.0, "max_abs_drho": 1e-14, "meets_1e-8": True},
    }
    b = bench.best_form(forms, 1535.0, 1188.0)
    assert b["form"] == "batched HPLANES"
    assert abs(b["vs_fp64_ratio"] - 1858.2 / 1188.0) < 1e-3


def test_best_form_ignores_forms_that_miss_the_bar():
    forms = {
        "batched_fp64": {"max_abs_drho": 0.0},
        "batched_hplanes": {"solve_steps_per_s": 2463.1, "max_abs_drho": 1.2e-2, "meets_1e-8": False},
        "hplanes": {"steps_per_s": 2036.0, "max_abs_drho": 1.2e-2, "meets_1e-8": False},
    }
    b = bench.best_form(forms, 2039.5, 1589.4)
    assert b["form"] == "batched FP64"
    assert b["steps_per_s"] == 2039.5


def test_command_line_lists_the_workloads_grid_and_form():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0
    for flag in ("--workload", "--grid", "--form", "--batch", "--impl"):
        assert flag in r.stdout
