"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Tolerance for the FP64 form: 1e-10 relative to the largest element of the
compared array (the bar stated for the FP64 drop-in), per RHS and per step.
Cases cover 1-D, 2-D and 3-D grids, radices 2/3/4/5/7/8, IPA and HSEX,
RK4 / AB4 / AB5, batched solves, and the reference's hBN golden run.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def lasers_of(pkg, cfg):
    return [pkg.Laser(L.intensity, L.omega, L.pol, L.cycles, L.t0, L.phase, L.fwhm, L.envelope) for L in cfg.lasers]


def make_pair(pkg, po, inp, batch=1):
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
    return cfg, o, s


def random_hermitian_state(shape, seed):
    rng = np.random.default_rng(seed)
    a = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    return 0.5 * (a + np.conj(np.transpose(a, (0, 2, 1))))


def model_input(pkg, tmp_path, name, grid, nb=3, seed=0, dims=2, coulomb=False, solver="RK", order=4,
                dt=0.05, envelope="sin2"):
    uc, Rs, H, r = pkg.workloads.random_model(nb, seed, dims=dims)
    seedp = os.path.join(str(tmp_path), name)
    pkg.workloads.write_tb(seedp + "_tb.dat", uc, Rs, H, r)
    if envelope == "sin2":
        las = [pkg.workloads.sin2_laser(2.0, 5e12, 3, pol=(1.0, 0.4, 0.2))]
    else:
        las = [pkg.workloads.gaussian_laser(1.5, 0.5, 0.02, 0.3, pol=(0.6, 1.0, 0.0))]
    inp = pkg.workloads._input(seedp, grid, max(1, nb // 2), dt, 10, solver, las, coulomb=coulomb,
                               epsilon=2.0, r0_A=10.0)
    inp["order"] = order
    return inp


CASES = [
    # name, grid, nb, dims, coulomb
    ("g2d", (6, 10, 1), 3, 2, False),
    ("g2d_hsex", (8, 6, 1), 4, 2, True),
    ("g1d", (9, 1, 1), 2, 1, False),
    ("g3d", (4, 3, 5), 2, 3, False),
    ("g7", (7, 14, 1), 2, 2, True),
    ("g50", (50, 50, 1), 2, 2, True),
    ("g64", (64, 8, 1), 3, 2, False),
    ("g36", (36, 12, 1), 2, 2, True),     # radix 12 then 3, and radix 12 alone
    ("g3d_6x9x4", (6, 9, 4), 2, 3, False),
    ("g120", (120, 120, 1), 2, 2, False),  # 230 KB plane in shared memory; radices 12 and 10
    ("g96", (96, 20, 1), 5, 2, True),      # odd nb: padded 2x2 commutator tiles
    # tensor-core (FP64 MMA) commutator from 12 bands: padded 8x8 tiles, TK 4 / 2
    ("mma12", (12, 8, 1), 12, 2, True),
    ("mma14", (10, 6, 1), 14, 2, False),
    ("mma17", (8, 6, 1), 17, 2, True),
    ("mma33", (6, 4, 1), 33, 2, True),
    # planes of 4096 points and more arrive by bulk copies; without HSEX, G
    # leaves by a bulk store and the next plane's bulk load into the same
    # buffer must wait for that store's reads
    ("bulk_ipa", (72, 64, 1), 3, 2, False),
    ("bulk_ipa_70x60", (70, 60, 1), 2, 2, False),
    # generic odd radices 11 and 13
    ("g11x13", (11, 13, 1), 3, 2, True),
    ("g3d_13x3x11", (13, 3, 11), 2, 3, False),
]


@pytest.mark.parametrize("name,grid,nb,dims,coulomb", CASES)
def test_rhs_parity(pkg, po, tmp_path, name, grid, nb, dims, coulomb):
    inp = model_input(pkg, tmp_path, name, grid, nb=nb, dims=dims, coulomb=coulomb, envelope="gauss")
    cfg, o, s = make_pair(pkg, po, inp)
    for seed, t in [(1, 0.3), (2, 4.0)]:
        rho = random_hermitian_state(o.shape, seed)
        ref = o.rhs(t, rho)
        got = s.rhs(t, rho)
        assert rel(got, ref) < TOL, (name, t)
    # a non-Hermitian input is handled like the reference (no symmetry assumed)
    rng = np.random.default_rng(5)
    rho = rng.normal(size=o.shape) + 1j * rng.normal(size=o.shape)
    assert rel(s.rhs(1.0, rho), o.rhs(1.0, rho)) < TOL


@pytest.mark.parametrize("solver,order", [("RK", 4), ("AB", 4), ("AB", 5)])
@pytest.mark.parametrize("coulomb", [False, True])
def test_steps_parity(pkg, po, tmp_path, solver, order, coulomb):
    # dt = 0.01 fs keeps AB5 inside its stability region for this model
    inp = model_input(pkg, tmp_path, f"st_{solver}{order}{int(coulomb)}", (10, 9, 1), nb=4, coulomb=coulomb,
                      solver=solver, order=order, dt=0.01)
    cfg, o, s = make_pair(pkg, po, inp)
    n0 = np.abs(o.get("rho")).max()
    for chunk in (1, 3, 8, 20):
        s.step(chunk)
        o.step(chunk)
        ref = o.get("rho")
        assert np.abs(ref).max() < 10 * n0  # a bounded (physical) trajectory
        assert rel(s.get_state(), ref) < TOL
        assert s.time == pytest.approx(o.time, rel=0, abs=1e-12)


# the fused HSEX commutator for 12 <= nb <= 24: 8x8 tiles in 2x2 (nb 13) and 3x3
# (nb 17, 19, 24) blocks; k counts 72, 35, 25 and 30 (0, 3, 1 and 2 mod 4) end the
# last update tile of 4 k points full, one short, with its second product tile
# wholly past the grid, and two short
@pytest.mark.parametrize("nb,grid", [(13, (8, 9, 1)), (19, (7, 5, 1)), (24, (5, 5, 1)), (17, (5, 6, 1))])
@pytest.mark.parametrize("solver,order", [("RK", 4), ("AB", 4)])
def test_steps_parity_mma(pkg, po, tmp_path, solver, order, nb, grid):
    inp = model_input(pkg, tmp_path, f"stm_{solver}{order}_{nb}", grid, nb=nb, coulomb=True, solver=solver,
                      order=order, dt=0.01)
    cfg, o, s = make_pair(pkg, po, inp, batch=2)
    for chunk in (1, 4, 10):
        s.step(chunk)
        o.step(chunk)
        ref = o.get("rho")
        assert rel(s.get_state(0), ref) < TOL
        assert rel(s.get_state(1), ref) < TOL


def test_batch_equals_separate_solves(pkg, po, tmp_path):
    inp = model_input(pkg, tmp_path, "batch", (8, 8, 1), nb=3, coulomb=True, dt=0.01)
    cfg, o, s = make_pair(pkg, po, inp, batch=3)
    base = lasers_of(pkg, cfg)[0]
    las = []
    for b in range(3):
        L = pkg.Laser(base.intensity * (1 + b), base.omega * (1 + 0.1 * b), base.pol, base.cycles, base.t0,
                      base.phase, base.fwhm, base.envelope)
        las.append(L)
        s.set_lasers([L], b)
    s.step(5)
    for b in range(3):
        _, o1, s1 = make_pair(pkg, po, inp)
        s1.set_lasers([las[b]], 0)
        s1.step(5)
        assert np.array_equal(s.get_state(b), s1.get_state(0))
        # and against the oracle with the same laser
        cfgb = po.load_input(inp)
        cfgb.lasers[0].intensity = las[b].intensity
        cfgb.lasers[0].omega = las[b].omega
        ob = po.Oracle(cfgb)
        ob.step(5)
        assert rel(s.get_state(b), ob.get("rho")) < TOL


def test_hbn_golden_on_gpu(pkg, po, hbn_golden_model):
    """The reference's hBN IPA integration test run on the GPU path:
    Population.txt and Velocity.txt reproduced at 1e-10 (ci-test/compare.py)."""
    cfg, o, s = make_pair(pkg, po, pkg.workloads.hbn_golden_input(hbn_golden_model))
    U = o.get("U")
    vel = [o.get("vx"), o.get("vy"), o.get("vz")]
    pops, vels = [], []
    for _ in range(cfg.nsteps):
        rho = s.get_state()
        rb = np.einsum("kji,kjl,klm->kim", U.conj(), rho, U)
        pb = np.real(np.einsum("knn->n", rb)) / o.Nk
        pb[: cfg.filledbands] = 1.0 - pb[: cfg.filledbands]
        pops.append(pb)
        v = [np.einsum("knl,kln->", vd, rho) / o.Nk for vd in vel]
        vels.append([x for c in v for x in (c.real, c.imag)])
        s.step(1)
    gp = np.loadtxt(os.path.join(GOLDEN, "hBN", "Population.txt"))
    gv = np.loadtxt(os.path.join(GOLDEN, "hBN", "Velocity.txt"))
    assert np.abs(np.array(pops) - gp).max() < 1e-10
    assert np.abs(np.array(vels) - gv).max() < 1e-10


def test_population_wannier_kernel(pkg, po, tmp_path):
    inp = model_input(pkg, tmp_path, "pop", (12, 10, 1), nb=4)
    cfg, o, s = make_pair(pkg, po, inp)
    s.step(3)
    rho = s.get_state()
    ref = np.real(np.einsum("knn->n", rho)) / o.Nk
    assert np.abs(s.population_wannier() - ref).max() < 1e-14


def test_tmd22_rhs_full_size(pkg, po, tmp_path):
    """The benchmark workload itself (22 orbitals, 72x72, HSEX): one RHS and two
    RK4 steps against the oracle."""
    inp = pkg.workloads.make("tmd22_rk4", str(tmp_path), nsteps=4)
    cfg, o, s = make_pair(pkg, po, inp)
    rho = o.get("rho")
    t = 10.0 * 41.341373335182113  # 10 fs, pulse centre
    assert rel(s.rhs(t, rho), o.rhs(t, rho)) < TOL
    s.time = t
    o.time = t
    s.step(2)
    o.step(2)
    assert rel(s.get_state(), o.get("rho")) < TOL


def test_unsupported_sizes_fail_cleanly(pkg):
    E = pkg.edus
    with pytest.raises(E.EdusError) as ei:
        E.Solver((17, 4, 1), 2, dt=0.1)
    assert ei.value.code == 5
    # a plane pair larger than shared memory is refused, not faulted
    with pytest.raises(E.EdusError) as ei:
        E.Solver((128, 128, 1), 2, dt=0.1, coulomb=True)
    assert ei.value.code == 5


def test_errors_are_reported(pkg, po, tmp_path):
    E = pkg.edus
    inp = model_input(pkg, tmp_path, "err", (6, 6, 1), nb=2, coulomb=True)
    cfg = po.load_input(inp)
    o = po.Oracle(cfg)
    s = E.Solver(cfg.grid, 2, cfg.dt, coulomb=True)
    with pytest.raises(E.EdusError) as ei:
        s.step(1)  # model not uploaded yet
    assert ei.value.code == 1
    xi = np.stack([o.get("xk"), o.get("yk"), o.get("zk")])
    with pytest.raises(E.EdusError):
        s.upload_model(o.get("H0k"), xi, o.lattice())  # coulomb needs W, rho0, hartree
    W = o.get("W").copy()
    W[0, 0, 0] += 1j
    with pytest.raises(E.EdusError):
        s.upload_model(o.get("H0k"), xi, o.lattice(), W, o.get("DM0R"), o.hartree())
    with pytest.raises(E.EdusError):
        s.set_state(o.get("rho"), b=1)
