"""GPU parity of the packed-Hermitian forms.

The packed forms propagate the Hermitian part of the reference's generator.
The two differ only on an even grid, on the planes of the Gamma-centred index
N/2 (coordinate -N/2 for both R and -R), where the reference's k-gradient and
self-energy are not Hermitian-preserving.  The oracle's `hermitian_nyquist`
switch computes the Hermitian part exactly; on odd grids it changes nothing
and the packed forms are compared with the unmodified oracle.

HERM64 keeps FP64 everywhere: it must match the oracle at the FP64 bar (1e-10
relative to the array max), which checks the packing and the split
rho = rho_ref + delta algebra.  MIXED stores the per-step intermediates in
FP32 and works on delta = rho - rho_ref, so its rounding error scales with
|delta|, not |rho|: after 16 steps it must stay below 5e-7 * max|delta|
(about 8 FP32 units of delta per step).
"""
import os

import numpy as np
import pytest

from test_gpu_parity import lasers_of, model_input, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10


def make_packed(pkg, po, inp, precision, batch=1, hermitian_nyquist=True):
    cfg = po.load_input(inp)
    cfg.hermitian_nyquist = hermitian_nyquist
    o = po.Oracle(cfg)
    s = pkg.Solver(cfg.grid, o.nb, cfg.dt, solver=cfg.solver, order=cfg.order, coulomb=cfg.coulomb, batch=batch,
                   precision=precision)
    xi = np.stack([o.get("xk"), o.get("yk"), o.get("zk")])
    if cfg.coulomb:
        s.upload_model(o.get("H0k"), xi, o.lattice(), o.get("W"), o.get("DM0R"), o.hartree())
    else:
        s.upload_model(o.get("H0k"), xi, o.lattice())
    for b in range(batch):
        s.set_lasers(lasers_of(pkg, cfg), b)
        s.set_state(o.get("rho"), b)
    return cfg, o, s


CASES = [
    # name, grid, nb, dims, coulomb, solver, order
    ("p2d", (6, 10, 1), 3, 2, False, "RK", 4),
    ("p2d_hsex", (8, 6, 1), 4, 2, True, "RK", 4),
    ("p_ab4", (10, 9, 1), 4, 2, True, "AB", 4),
    ("p_ab5", (8, 8, 1), 5, 2, False, "AB", 5),
    ("p1d", (9, 1, 1), 2, 1, False, "RK", 4),
    ("p3d", (4, 3, 5), 2, 3, False, "RK", 4),
    ("p13", (8, 9, 1), 13, 2, True, "RK", 4),
    ("p72", (72, 8, 1), 6, 2, True, "RK", 4),   # radix 8 x 9 axis (specialised plane kernel)
]


@pytest.mark.parametrize("coulomb", [False, True])
def test_herm64_odd_grid_matches_reference_oracle(pkg, po, tmp_path, coulomb):
    """No N/2 index on an odd grid: the packed form reproduces the unmodified
    reference algorithm."""
    E = pkg.edus
    inp = model_input(pkg, tmp_path, "podd", (7, 9, 1), nb=4, coulomb=coulomb, dt=0.01, envelope="gauss")
    cfg, o, s = make_packed(pkg, po, inp, E.PREC_HERM64, hermitian_nyquist=False)
    s.step(10)
    o.step(10)
    assert rel(s.get_state(), o.get("rho")) < TOL


@pytest.mark.parametrize("name,grid,nb,dims,coulomb,solver,order", CASES)
def test_herm64_matches_oracle(pkg, po, tmp_path, name, grid, nb, dims, coulomb, solver, order):
    E = pkg.edus
    inp = model_input(pkg, tmp_path, name, grid, nb=nb, dims=dims, coulomb=coulomb, solver=solver, order=order,
                      dt=0.01, envelope="gauss")
    cfg, o, s = make_packed(pkg, po, inp, E.PREC_HERM64)
    assert rel(s.get_state(), o.get("rho")) < 1e-14  # rho_ref + 0 round trip
    for chunk in (1, 3, 12):
        s.step(chunk)
        o.step(chunk)
        assert rel(s.get_state(), o.get("rho")) < TOL, (name, chunk)
    assert abs(s.time - o.time) < 1e-12


@pytest.mark.parametrize("name,grid,nb,dims,coulomb,solver,order", CASES)
def test_mixed_error_bound(pkg, po, tmp_path, name, grid, nb, dims, coulomb, solver, order):
    E = pkg.edus
    inp = model_input(pkg, tmp_path, name, grid, nb=nb, dims=dims, coulomb=coulomb, solver=solver, order=order,
                      dt=0.01, envelope="gauss")
    cfg, o, s = make_packed(pkg, po, inp, E.PREC_MIXED)
    rho_ref = o.get("rho")
    s.step(16)
    o.step(16)
    got, ref = s.get_state(), o.get("rho")
    err = float(np.abs(got - ref).max())
    assert err < 5e-7 * float(np.abs(ref - rho_ref).max()), (name, err)
    # Hermitian to rounding
    assert np.abs(got - np.conj(np.transpose(got, (0, 2, 1)))).max() < 1e-13


def test_packed_batch(pkg, po, tmp_path):
    E = pkg.edus
    inp = model_input(pkg, tmp_path, "pbatch", (8, 8, 1), nb=3, coulomb=True, dt=0.01, envelope="gauss")
    cfg, o, s = make_packed(pkg, po, inp, E.PREC_HERM64, batch=3)
    base = lasers_of(pkg, cfg)[0]
    for b in range(3):
        L = pkg.Laser(base.intensity * (1 + b), base.omega, base.pol, base.cycles, base.t0, base.phase, base.fwhm,
                      base.envelope)
        s.set_lasers([L], b)
    s.step(6)
    for b in range(3):
        cfgb = po.load_input(inp)
        cfgb.hermitian_nyquist = True
        cfgb.lasers[0].intensity = base.intensity * (1 + b)
        ob = po.Oracle(cfgb)
        ob.step(6)
        assert rel(s.get_state(b), ob.get("rho")) < TOL


def test_packed_population(pkg, po, tmp_path):
    E = pkg.edus
    inp = model_input(pkg, tmp_path, "ppop", (6, 6, 1), nb=4, coulomb=True, dt=0.01, envelope="gauss")
    cfg, o, s = make_packed(pkg, po, inp, E.PREC_MIXED)
    s.step(5)
    rho = s.get_state()
    assert np.abs(s.population_wannier() - np.real(np.einsum("knn->n", rho)) / o.Nk).max() < 1e-14


def test_packed_refuses_non_hermitian_self_energy(pkg, po, tmp_path):
    """Two off-origin Wannier centres make the reference's cumulative r_nm
    (ModelCoulomb.cpp:76-79) break W_nm(R) = W_mn(-R): the packed forms refuse
    the model, the FP64 form takes it."""
    E = pkg.edus
    uc, Rs, H, r = pkg.workloads.random_model(3, 7)
    r[0, 0, 0, 0] = 0.4  # a second off-origin centre
    seed = os.path.join(str(tmp_path), "badw")
    pkg.workloads.write_tb(seed + "_tb.dat", uc, Rs, H, r)
    inp = pkg.workloads._input(seed, (6, 6, 1), 1, 0.01, 10, "RK", [], coulomb=True, epsilon=2.0, r0_A=10.0)
    cfg = po.load_input(inp)
    o = po.Oracle(cfg)
    xi = np.stack([o.get("xk"), o.get("yk"), o.get("zk")])
    s = E.Solver(cfg.grid, o.nb, cfg.dt, coulomb=True, precision=E.PREC_MIXED)
    with pytest.raises(E.EdusError) as ei:
        s.upload_model(o.get("H0k"), xi, o.lattice(), o.get("W"), o.get("DM0R"), o.hartree())
    assert ei.value.code == 5
    s2 = E.Solver(cfg.grid, o.nb, cfg.dt, coulomb=True)
    s2.upload_model(o.get("H0k"), xi, o.lattice(), o.get("W"), o.get("DM0R"), o.hartree())


def test_packed_needs_state_before_step(pkg, po, tmp_path):
    E = pkg.edus
    inp = model_input(pkg, tmp_path, "pord", (6, 6, 1), nb=2)
    cfg = po.load_input(inp)
    o = po.Oracle(cfg)
    s = E.Solver(cfg.grid, 2, cfg.dt, precision=E.PREC_HERM64)
    xi = np.stack([o.get("xk"), o.get("yk"), o.get("zk")])
    s.upload_model(o.get("H0k"), xi, o.lattice())
    with pytest.raises(E.EdusError):
        s.step(1)
