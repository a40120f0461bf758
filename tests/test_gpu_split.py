"""GPU parity of the split-precision form (EDUS_PREC_SPLIT32).

The form computes the reference's full generator (every band pair, the
reference's own gradient and self-energy on every grid, so the unmodified
oracle is the comparison) with rho = rho_ref + delta, the terms of rho_ref in
FP64 and the plane transforms of delta in FP32.  Its rounding error scales
with |delta| <= |rho(t) - rho(t_anchor)|: after n steps the tests require
max|rho - rho_oracle| < 5e-7 * max|rho(n) - rho(0)|, about 8 FP32 units of the
change per step, and an FP64-exact right-hand side when delta = 0.
"""
import numpy as np
import pytest

from test_gpu_parity import lasers_of, model_input, rel

pytestmark = pytest.mark.gpu


def make_split(pkg, po, inp, batch=1, anchor=None):
    cfg = po.load_input(inp)
    o = po.Oracle(cfg)
    E = pkg.edus
    s = pkg.Solver(cfg.grid, o.nb, cfg.dt, solver=cfg.solver, order=cfg.order, coulomb=cfg.coulomb, batch=batch,
                   precision=E.PREC_SPLIT32)
    xi = np.stack([o.get("xk"), o.get("yk"), o.get("zk")])
    if cfg.coulomb:
        s.upload_model(o.get("H0k"), xi, o.lattice(), o.get("W"), o.get("DM0R"), o.hartree())
    else:
        s.upload_model(o.get("H0k"), xi, o.lattice())
    for b in range(batch):
        s.set_lasers(lasers_of(pkg, cfg), b)
        s.set_state(o.get("rho"), b)
    if anchor is not None:
        s.set_anchor_interval(anchor)
    return cfg, o, s


CASES = [
    # name, grid, nb, dims, coulomb, solver, order, anchor interval
    ("s2d", (6, 10, 1), 3, 2, False, "RK", 4, None),
    ("s2d_hsex", (8, 6, 1), 4, 2, True, "RK", 4, 5),
    ("s_ab4", (10, 9, 1), 4, 2, True, "AB", 4, None),
    ("s1d", (9, 1, 1), 2, 1, False, "RK", 4, 3),
    ("s3d", (4, 3, 5), 2, 3, False, "RK", 4, None),
    ("s12", (12, 8, 1), 12, 2, True, "RK", 4, 7),     # TMA commutator, 2x2 tiles
    ("s17", (8, 6, 1), 17, 2, True, "RK", 4, None),   # TMA commutator, 3x3 tiles
    ("s72", (72, 8, 1), 6, 2, True, "RK", 4, 4),      # radix 8 x 9 plane variant
]


@pytest.mark.parametrize("name,grid,nb,dims,coulomb,solver,order,anchor", CASES)
def test_split_matches_oracle(pkg, po, tmp_path, name, grid, nb, dims, coulomb, solver, order, anchor):
    inp = model_input(pkg, tmp_path, name, grid, nb=nb, dims=dims, coulomb=coulomb, solver=solver, order=order,
                      dt=0.01, envelope="gauss")
    cfg, o, s = make_split(pkg, po, inp, anchor=anchor)
    rho0 = o.get("rho")
    assert rel(s.get_state(), rho0) < 1e-15
    s.step(16)
    o.step(16)
    got, ref = s.get_state(), o.get("rho")
    err = float(np.abs(got - ref).max())
    assert err < 5e-7 * float(np.abs(ref - rho0).max()), (name, err)
    assert abs(s.time - o.time) < 1e-12


def test_split_rhs_exact_at_anchor(pkg, po, tmp_path):
    """delta = 0: the right-hand side is the FP64 one of the anchor."""
    inp = model_input(pkg, tmp_path, "srhs", (8, 6, 1), nb=4, coulomb=True, dt=0.01, envelope="gauss")
    cfg, o, s = make_split(pkg, po, inp)
    rho = o.get("rho")
    for t in (0.3, 7.0):
        assert rel(s.rhs(t, rho), o.rhs(t, rho)) < 1e-12


def test_split_batch_equals_separate(pkg, po, tmp_path):
    inp = model_input(pkg, tmp_path, "sbatch", (8, 8, 1), nb=3, coulomb=True, dt=0.01, envelope="gauss")
    cfg, o, s = make_split(pkg, po, inp, batch=3, anchor=3)
    base = lasers_of(pkg, cfg)[0]
    for b in range(3):
        L = pkg.Laser(base.intensity * (1 + b), base.omega, base.pol, base.cycles, base.t0, base.phase, base.fwhm,
                      base.envelope)
        s.set_lasers([L], b)
    s.step(8)
    for b in range(3):
        cfgb = po.load_input(inp)
        cfgb.lasers[0].intensity = base.intensity * (1 + b)
        ob = po.Oracle(cfgb)
        rho0 = ob.get("rho")
        ob.step(8)
        ref = ob.get("rho")
        assert np.abs(s.get_state(b) - ref).max() < 5e-7 * np.abs(ref - rho0).max()


def test_split_anchor_interval_arguments(pkg, po, tmp_path):
    E = pkg.edus
    inp = model_input(pkg, tmp_path, "sarg", (6, 6, 1), nb=2)
    cfg, o, s = make_split(pkg, po, inp)
    with pytest.raises(E.EdusError):
        s.set_anchor_interval(0)
    s2 = E.Solver(cfg.grid, 2, cfg.dt)
    with pytest.raises(E.EdusError):
        s2.set_anchor_interval(8)
