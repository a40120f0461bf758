"""GPU parity of gradient_space "k" (the finite-difference k gradient of
kGradient.cpp) against the oracle's restatement, at the FP64 bar (1e-10
relative): the stencil comes from model.kgradient_stencil, the oracle builds
its own shells and weights, so the test pins both."""
import numpy as np
import pytest

from test_gpu_parity import lasers_of, model_input, rel

pytestmark = pytest.mark.gpu

CASES = [
    # name, grid, nb, dims, coulomb, solver, order
    ("k2d", (12, 12, 1), 3, 2, False, "RK", 4),
    ("k2d_hsex", (8, 6, 1), 4, 2, True, "RK", 4),
    ("k1d", (9, 1, 1), 2, 1, False, "RK", 4),
    ("k3d", (4, 3, 5), 2, 3, False, "RK", 4),
    ("k_ab4", (10, 9, 1), 3, 2, True, "AB", 4),
    ("k13", (8, 9, 1), 13, 2, True, "RK", 4),
]


@pytest.mark.parametrize("name,grid,nb,dims,coulomb,solver,order", CASES)
def test_kgradient_matches_oracle(pkg, po, tmp_path, name, grid, nb, dims, coulomb, solver, order):
    E = pkg.edus
    inp = model_input(pkg, tmp_path, name, grid, nb=nb, dims=dims, coulomb=coulomb, solver=solver, order=order,
                      dt=0.01, envelope="gauss")
    inp["gradient_space"] = "k"
    cfg = po.load_input(inp)
    o = po.Oracle(cfg)
    m = pkg.model.Model(pkg.model.parse_input(inp))
    s = E.Solver(cfg.grid, o.nb, cfg.dt, solver=cfg.solver, order=cfg.order, coulomb=cfg.coulomb)
    xi = np.stack([o.get("xk"), o.get("yk"), o.get("zk")])
    if cfg.coulomb:
        s.upload_model(o.get("H0k"), xi, o.lattice(), o.get("W"), o.get("DM0R"), o.hartree())
    else:
        s.upload_model(o.get("H0k"), xi, o.lattice())
    s.set_kgradient(*m.kgradient_stencil())
    s.set_lasers(lasers_of(pkg, cfg))
    s.set_state(o.get("rho"))
    rng = np.random.default_rng(4)
    x = rng.normal(size=o.shape) + 1j * rng.normal(size=o.shape)
    for t in (0.3 * 41.341373335182113, 7.0):
        assert rel(s.rhs(t, x), o.rhs(t, x)) < 1e-10
    s.step(10)
    o.step(10)
    assert rel(s.get_state(), o.get("rho")) < 1e-10
    # the k stencil differs from the R-space gradient (this is not a no-op)
    cfgR = po.load_input({**inp, "gradient_space": "R"})
    oR = po.Oracle(cfgR)
    assert rel(oR.rhs(7.0, x), o.rhs(7.0, x)) > 1e-6


def test_kgradient_model_solver_and_reset(pkg, po, tmp_path):
    """Model.solver applies gradient_space "k" from the input; set_kgradient()
    without arguments returns to the R-space gradient."""
    inp = model_input(pkg, tmp_path, "kms", (12, 12, 1), nb=2, dt=0.01, envelope="gauss")
    inp["gradient_space"] = "k"
    m = pkg.model.Model(pkg.model.parse_input(inp))
    s = m.solver()
    ok = po.Oracle(po.load_input(inp))
    oR = po.Oracle(po.load_input({**inp, "gradient_space": "R"}))
    rho = ok.get("rho")
    t = 7.0
    assert rel(s.rhs(t, rho), ok.rhs(t, rho)) < 1e-10
    s.set_kgradient()
    assert rel(s.rhs(t, rho), oR.rhs(t, rho)) < 1e-10
