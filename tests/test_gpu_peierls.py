"""GPU tests of the Peierls gauge ("peierls": true): no gradient term and
H(R) = (H0 + E.xi + Hee[rho(R) e^{-iA.R}]) e^{+iA.R}, with A(t) integrated as
Laser::VectorPotential does (Functional_SourceTerm.hpp:15-50,
Simulation.cpp:876-899, Laser.cpp:136-151).

Every case runs the same input through the oracle with "peierls" set and
compares at the FP64 bar (1e-10 relative to the array maximum).
"""
import numpy as np
import pytest

from test_gpu_parity import lasers_of, model_input, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10


def pair(pkg, po, tmp_path, name, grid, nb, coulomb, solver="RK", order=4, batch=1, dt=0.01):
    inp = model_input(pkg, tmp_path, name, grid, nb=nb, coulomb=coulomb, solver=solver, order=order, dt=dt,
                      envelope="gauss")
    inp["peierls"] = True
    cfg = po.load_input(inp)
    o = po.Oracle(cfg)
    s = pkg.Solver(cfg.grid, o.nb, cfg.dt, solver=cfg.solver, order=cfg.order, coulomb=cfg.coulomb, batch=batch)
    xi = np.stack([o.get("xk"), o.get("yk"), o.get("zk")])
    if cfg.coulomb:
        s.upload_model(o.get("H0k"), xi, o.lattice(), o.get("W"), o.get("DM0R"), o.hartree())
    else:
        s.upload_model(o.get("H0k"), xi, o.lattice())
    for b in range(batch):
        s.set_lasers(lasers_of(pkg, cfg), b)
        s.set_state(o.get("rho"), b)
    s.set_peierls(True)
    return inp, cfg, o, s


@pytest.mark.parametrize("nb,grid,coulomb", [(2, (8, 6, 1), False), (3, (6, 10, 1), True), (13, (8, 9, 1), True),
                                             (14, (6, 6, 1), False)])
def test_rhs_matches_oracle(pkg, po, tmp_path, nb, grid, coulomb):
    _, cfg, o, s = pair(pkg, po, tmp_path, f"prhs{nb}{int(coulomb)}", grid, nb, coulomb)
    rng = np.random.default_rng(nb)
    rho = o.get("rho") + 0.05 * (rng.normal(size=o.get("rho").shape) + 1j * rng.normal(size=o.get("rho").shape))
    # times inside the pulse, increasing: each call is one request to both integrators
    for t in (cfg.lasers[0].t0 - 0.3 * cfg.lasers[0].fwhm, cfg.lasers[0].t0, cfg.lasers[0].t0 + 0.2 * cfg.lasers[0].fwhm):
        ref = o.rhs(t, rho)
        assert rel(s.rhs(t, rho), ref) < TOL, t
    assert np.allclose(s.vector_potential(cfg.lasers[0].t0 + cfg.lasers[0].fwhm),
                       o.vector_potential(cfg.lasers[0].t0 + cfg.lasers[0].fwhm), rtol=0, atol=1e-14)


@pytest.mark.parametrize("solver,order", [("RK", 4), ("AB", 4)])
@pytest.mark.parametrize("coulomb", [False, True])
def test_steps_match_oracle(pkg, po, tmp_path, solver, order, coulomb):
    _, cfg, o, s = pair(pkg, po, tmp_path, f"pst{solver}{int(coulomb)}", (8, 6, 1), 3, coulomb, solver=solver,
                        order=order)
    t0 = cfg.lasers[0].t0 - 1.5 * cfg.lasers[0].fwhm
    s.time = t0
    o.time = t0
    for chunk in (1, 5, 20):
        s.step(chunk)
        o.step(chunk)
        assert rel(s.get_state(), o.get("rho")) < TOL
        assert s.time == pytest.approx(o.time, rel=0, abs=1e-12)
    # the field has acted: the state moved away from the initial one
    assert rel(s.get_state(), po.Oracle(cfg).get("rho")) > 1e-6


def test_tensor_core_commutators(pkg, po, tmp_path):
    """HSEX with 22 bands (warp-specialised TMA commutator) and 14 bands without
    HSEX (tensor-core commutator with the fused Hamiltonian)."""
    for nb, coulomb, grid in ((22, True, (6, 4, 1)), (14, False, (6, 6, 1))):
        _, cfg, o, s = pair(pkg, po, tmp_path, f"ptc{nb}", grid, nb, coulomb)
        t0 = cfg.lasers[0].t0 - 0.5 * cfg.lasers[0].fwhm
        s.time = t0
        o.time = t0
        s.step(6)
        o.step(6)
        assert rel(s.get_state(), o.get("rho")) < TOL, nb


def test_batch_each_solve_its_own_vector_potential(pkg, po, tmp_path):
    inp, cfg, o, s = pair(pkg, po, tmp_path, "pbatch", (8, 6, 1), 3, True, batch=2)
    base = lasers_of(pkg, cfg)[0]
    L1 = pkg.Laser(base.intensity * 2.0, base.omega * 1.1, base.pol, base.cycles, base.t0, base.phase, base.fwhm,
                   base.envelope)
    s.set_lasers([L1], 1)
    s.set_peierls(True)  # restart both integrators after the laser change
    t0 = cfg.lasers[0].t0 - cfg.lasers[0].fwhm
    s.time = t0
    s.step(12)
    o.time = t0
    o.step(12)
    assert rel(s.get_state(0), o.get("rho")) < TOL
    cfg1 = po.load_input(inp)
    cfg1.lasers[0].intensity = L1.intensity
    cfg1.lasers[0].omega = L1.omega
    o1 = po.Oracle(cfg1)
    o1.time = t0
    o1.step(12)
    assert rel(s.get_state(1), o1.get("rho")) < TOL


def test_observables_in_peierls_gauge(pkg, po, tmp_path):
    _, cfg, o, s = pair(pkg, po, tmp_path, "pobs", (8, 6, 1), 3, True)
    s.upload_observables(U=o.get("U"), vel=np.stack([o.get("vx"), o.get("vy"), o.get("vz")]))
    t0 = cfg.lasers[0].t0 - 0.5 * cfg.lasers[0].fwhm
    s.time = t0
    o.time = t0
    for _ in range(3):
        s.step(4)
        o.step(4)
        pb, pw, v = s.observables(0, cfg.filledbands)
        rb, rw, rv = o.observables()
        assert np.abs(pb - rb).max() < 1e-12
        assert np.abs(pw - rw).max() < 1e-12
        assert np.abs(np.array([x for c in v for x in (c.real, c.imag)]) - rv).max() < 1e-12


def test_unsupported_forms_refused(pkg, po, tmp_path):
    E = pkg.edus
    inp = model_input(pkg, tmp_path, "pref", (6, 6, 1), nb=2)
    cfg = po.load_input(inp)
    o = po.Oracle(cfg)
    p = E.Solver(cfg.grid, 2, cfg.dt, precision=E.PREC_HERM64)
    p.upload_model(o.get("H0k"), np.stack([o.get("xk"), o.get("yk"), o.get("zk")]), o.lattice())
    with pytest.raises(E.EdusError) as ei:
        p.set_peierls(True)
    assert ei.value.code == 5
