import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")
# the reference sources, where they are mounted (no default: tests needing them skip)
REFERENCE = os.environ.get("EDUS_REFERENCE_DIR", "")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def pkg():
    import __graft_entry__ as ge

    return ge.load_package()


@pytest.fixture(scope="session")
def po():
    import pyoracle

    pyoracle.build_lib()
    return pyoracle


def reference_available() -> bool:
    return bool(REFERENCE) and os.path.isdir(os.path.join(REFERENCE, "src"))


@pytest.fixture(scope="session")
def hbn_golden_model(tmp_path_factory, pkg):
    """The reference's hBN test model, regenerated from its parameters."""
    d = tmp_path_factory.mktemp("hbn")
    uc, Rs, H, r = pkg.workloads.hexagonal_two_band(a=2.5, onsite=3.625, t=-2.3, centre=1.44337567297406441)
    seed = os.path.join(str(d), "hBN_gap7.25eV_a2.5A")
    pkg.workloads.write_tb(seed + "_tb.dat", uc, Rs, H, r)
    return seed
