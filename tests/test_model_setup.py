"""Product host set-up (edus_2.0_b200/model.py) against the oracle's set-up,
on CPU: the arrays the GPU receives must equal the reference's (1e-12)."""
import os

import numpy as np
import pytest


def _cmp(a, b, tol=1e-12):
    return float(np.abs(a - b).max() / max(1.0, np.abs(b).max())) < tol


@pytest.mark.parametrize("coulomb,fix", [(False, False), (True, False), (True, True)])
def test_model_matches_oracle(pkg, po, tmp_path, coulomb, fix):
    uc, Rs, H, r = pkg.workloads.random_model(4, 3)
    seed = os.path.join(str(tmp_path), "m")
    pkg.workloads.write_tb(seed + "_tb.dat", uc, Rs, H, r)
    inp = pkg.workloads._input(seed, (9, 8, 1), 2, 0.05, 10, "RK",
                               [pkg.workloads.gaussian_laser(1.5, 2.0, 0.01, 1.0)], coulomb=coulomb,
                               epsilon=1.5, r0_A=12.0)
    inp["coulomb_fix_centres"] = fix
    m = pkg.model.Model(pkg.model.parse_input(inp))
    o = po.Oracle(po.load_input(inp))
    assert _cmp(m.H0k, o.get("H0k"))
    for d, n in enumerate(("xk", "yk", "zk")):
        assert _cmp(m.xik[d], o.get(n))
    assert _cmp(m.rho0k, o.get("rho"))
    assert np.allclose(m.eval, o.eigenvalues(), atol=1e-12)
    assert _cmp(m.Rcart, o.rcart())
    assert _cmp(m.A, o.lattice())
    if coulomb:
        assert _cmp(m.W, o.get("W"))
        assert _cmp(m.DM0R, o.get("DM0R"))
        assert _cmp(m.hartree, o.hartree())


def test_struve_vectorised_matches_oracle(pkg, po):
    xs = np.array([0.0, 1e-3, 0.5, 3.0, 19.9, 20.0, 20.01, 35.0, 49.9, 50.0, 120.0])
    got = pkg.model.struve0(xs)
    ref = np.array([po.struve0(x) for x in xs])
    assert np.abs(got - ref).max() < 1e-15 * 10


def test_lasers_parsed_like_oracle(pkg, po):
    inp = {"tb_file": "x", "grid": [4, 4, 1], "dt": 0.01, "dt_units": "fs",
           "lasers": [pkg.workloads.gaussian_laser(1.5, 10.0, 0.01, 10.0),
                      pkg.workloads.sin2_laser(3.0, 1e11, 2, 1.0, pol=(1, 1, 0))]}
    a = pkg.model.parse_input(inp)
    b = po.load_input(inp)
    assert a.dt == b.dt
    for La, Lb in zip(a.lasers, b.lasers):
        assert (La.intensity, La.omega, La.t0, La.fwhm, La.envelope, La.cycles) == \
               (Lb.intensity, Lb.omega, Lb.t0, Lb.fwhm, Lb.envelope, Lb.cycles)
