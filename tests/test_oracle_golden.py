"""Pin the CPU oracle to the reference's own golden vectors and known answers.

Runs on CPU.  The oracle (oracle/edus_oracle.cpp) is the checker of every GPU
parity test, so it is checked here first against:
  * ci-test/outputs/hBN/{Population,Velocity,Laser,Time}.txt of the reference,
    with ci-test/compare.py semantics (1e-10 absolute, column 0 skipped) and,
    stricter, on every column;
  * ci-test/Reference/Struve.txt (6 printed decimals);
  * analytic answers restated from ci-test/test_DEsolver2.cpp (phase rotation),
    test_Gradient_R.cpp (plane-wave gradient) and test_fft_mpi.cpp (transform).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, reference_available, REFERENCE


def compare_py(a, b, tol=1e-10):
    """ci-test/compare.py:1-23: skip column 0, fail if |a-b| > tol while either exceeds tol."""
    a = np.atleast_2d(a).T[1:].flatten()
    b = np.atleast_2d(b).T[1:].flatten()
    bad = (np.abs(a - b) > tol) & ((np.abs(a) > tol) | (np.abs(b) > tol))
    return not bad.any()


@pytest.fixture(scope="module")
def hbn_run(po, pkg, hbn_golden_model):
    cfg = po.load_input(pkg.workloads.hbn_golden_input(hbn_golden_model))
    o = po.Oracle(cfg)
    pops, vels, las, times = [], [], [], []
    for _ in range(cfg.nsteps):
        pb, pw, v = o.observables()
        pops.append(pb)
        vels.append(v)
        las.append(o.efield(o.time))
        times.append(o.time)
        o.step(1)
    return cfg, np.array(pops), np.array(vels), np.array(las), np.array(times)


def test_hbn_nsteps(hbn_run):
    cfg = hbn_run[0]
    assert cfg.nsteps == 102  # int((1 fs - 0)/0.01 fs) + 2


def test_hbn_population_golden(hbn_run):
    gold = np.loadtxt(os.path.join(GOLDEN, "hBN", "Population.txt"))
    pops = hbn_run[1]
    assert pops.shape == gold.shape
    assert compare_py(pops, gold)
    assert np.abs(pops - gold).max() < 1e-10


def test_hbn_velocity_golden(hbn_run):
    gold = np.loadtxt(os.path.join(GOLDEN, "hBN", "Velocity.txt"))
    vels = hbn_run[2]
    assert vels.shape == gold.shape
    assert compare_py(vels, gold)
    assert np.abs(vels - gold).max() < 1e-10
    # the signal itself is far above the tolerance: this is a real check
    assert np.abs(gold[:, 0]).max() > 1e-5


def test_hbn_laser_and_time_golden(hbn_run):
    las = np.loadtxt(os.path.join(GOLDEN, "hBN", "Laser.txt"))
    t = np.loadtxt(os.path.join(GOLDEN, "hBN", "Time.txt"))
    assert np.abs(hbn_run[3] - las).max() < 1e-16
    # Time.txt is printed with 6 significant digits
    assert np.allclose(hbn_run[4], t, rtol=1e-5, atol=1e-12)


def test_struve_table(po):
    rows = [l.split() for l in open(os.path.join(GOLDEN, "Struve.txt")).read().splitlines()[2:] if l.strip()]
    for row in rows:
        x = float(row[0].split("=")[1])
        h0 = float(row[1])
        assert abs(po.struve0(x) - h0) <= 6e-7, (x, po.struve0(x), h0)


def test_struve_large_argument(po):
    # asymptotic branch (x > 20) against scipy's H0
    from scipy.special import struve

    for x in (20.5, 31.0, 49.0, 75.0):
        assert abs(po.struve0(x) - struve(0, x)) < 1e-6


def test_fft_matches_numpy(po):
    rng = np.random.default_rng(0)
    for dims in [(6, 10, 1), (72, 72, 1), (5, 4, 3), (64, 1, 1), (7, 1, 1)]:
        Nk = dims[0] * dims[1] * dims[2]
        a = rng.normal(size=(Nk, 3)) + 1j * rng.normal(size=(Nk, 3))
        got = po.fft(a, dims, -1)
        ref = np.fft.fftn(a.reshape(*dims, 3), axes=(0, 1, 2)).reshape(Nk, 3) / Nk
        assert np.abs(got - ref).max() < 1e-13 * max(1, np.abs(ref).max())
        got = po.fft(a, dims, +1)
        ref = np.fft.ifftn(a.reshape(*dims, 3), axes=(0, 1, 2)).reshape(Nk, 3) * Nk
        assert np.abs(got - ref).max() < 1e-12 * np.abs(ref).max()


def test_fft_gaussian_known_answer(po):
    # test_fft_mpi.cpp: a Gaussian sampled on a periodic grid transforms into a
    # Gaussian; checked here against the closed form at 0.5 % like the reference.
    N = 100
    sigma = 6.0
    x = np.arange(N)
    xc = np.where(x < N // 2, x, x - N)
    g = np.exp(-(xc[:, None] ** 2 + xc[None, :] ** 2) / (2 * sigma ** 2)).reshape(N * N, 1)
    out = po.fft(g.astype(complex), (N, N, 1), -1).reshape(N, N)
    kc = 2 * np.pi * xc / N
    ana = (2 * np.pi * sigma ** 2) * np.exp(-(kc[:, None] ** 2 + kc[None, :] ** 2) * sigma ** 2 / 2) / (N * N)
    assert np.abs(out - ana).max() <= 5e-3 * ana.max()


def test_eigh_matches_numpy(po):
    rng = np.random.default_rng(1)
    for n in (1, 2, 5, 22):
        A = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        A = A + A.conj().T
        w, V = po.eigh(A)
        assert np.allclose(w, np.linalg.eigvalsh(A), atol=1e-12)
        assert np.abs(A @ V - V * w).max() < 1e-12
        assert np.abs(V.conj().T @ V - np.eye(n)).max() < 1e-13


def test_units_and_defaults(po):
    # unknown unit strings give the reference's silent NullUnit (value 0)
    assert po.unit("Wcm2") == 0.0
    assert po.unit("wcm2") == 1e4
    cfg = po.load_input({"tb_file": "x", "grid": [4, 4, 1], "dt": 0.01, "dt_units": "fs",
                         "finaltime": 1.0, "finaltime_units": "fs",
                         "lasers": [{"intensity": 1e10, "frequency": 1.0, "polarization": [1, 0, 0], "cycles": 1}]})
    assert cfg.lasers[0].intensity == 0.0  # default units "Wcm2" -> NullUnit
    assert cfg.lasers[0].omega == 0.0      # default units "eV" -> NullUnit
    assert cfg.nsteps == int((cfg.finaltime - cfg.initialtime) / cfg.dt) + 2


def _two_level_cfg(po, pkg, tmp_path, grid=(4, 4, 1), solver="RK", order=4, dt=0.05):
    # k-independent two-level system, no field: rho_01(t) = rho_01(0) exp(-i (e0-e1) t)
    uc = [[2.0, 0, 0], [0, 2.0, 0], [0, 0, 20.0]]
    H = np.zeros((1, 2, 2), complex)
    H[0, 0, 0], H[0, 1, 1] = -1.0, 1.5
    r = np.zeros((3, 1, 2, 2), complex)
    seed = os.path.join(str(tmp_path), "twolevel")
    pkg.workloads.write_tb(seed + "_tb.dat", uc, [(0, 0, 0)], H, r)
    inp = pkg.workloads._input(seed, grid, 1, dt, 10, solver, [])
    inp["order"] = order
    return po.load_input(inp)


def discrete_rotation(lam, h, nsteps, solver, order, y0=0.5):
    """Exact iterate of the reference's steppers on y' = lam y (DESolver.hpp:154-220),
    AB history starting at zero (DESolver.cpp:26-29)."""
    y = complex(y0)
    if solver == "RK":
        z = lam * h
        R = 1 + z + z * z / 2 + z ** 3 / 6 + z ** 4 / 24
        return y * R ** nsteps
    beta = {4: [55 / 24, -59 / 24, 37 / 24, -3 / 8], 5: [1901 / 720, -2774 / 720, 2616 / 720, -1274 / 720, 251 / 720]}[order]
    hist = [0j] * order
    for _ in range(nsteps):
        hist = [lam * y] + hist[:-1]
        for i in range(order):
            y = y + h * beta[i] * hist[i]
    return y


@pytest.mark.parametrize("solver,order", [("RK", 4), ("AB", 4), ("AB", 5)])
def test_phase_rotation_stepper(po, pkg, tmp_path, solver, order):
    # restates ci-test/test_DEsolver2.cpp (y' = 2 i H00 y): the oracle's stepper
    # must reproduce the exact discrete iterate of RK4 / AB4 / AB5
    cfg = _two_level_cfg(po, pkg, tmp_path, solver=solver, order=order, dt=0.05)
    o = po.Oracle(cfg)
    rho = np.full(o.shape, 0.5, dtype=complex)
    o.set_state(rho)
    nst = 200
    o.step(nst)
    de = (-1.0 - 1.5) * 1.602176634e-19 / (2 * 2.1798723611035e-18)
    exact = discrete_rotation(-1j * de, cfg.dt, nst, solver, order)
    got = o.get("rho")[:, 0, 1]
    assert np.abs(got - exact).max() / 0.5 < 1e-12
    assert abs(o.time - nst * cfg.dt) < 1e-9


def test_phase_rotation_analytic(po, pkg, tmp_path):
    # continuous solution at a small step: relative error < 1e-8 % as in test_DEsolver2
    cfg = _two_level_cfg(po, pkg, tmp_path, solver="RK", order=4, dt=0.001)
    o = po.Oracle(cfg)
    o.set_state(np.full(o.shape, 0.5, dtype=complex))
    o.step(1000)
    de = (-1.0 - 1.5) * 1.602176634e-19 / (2 * 2.1798723611035e-18)
    exact = 0.5 * np.exp(-1j * de * o.time)
    assert np.abs(o.get("rho")[:, 0, 1] - exact).max() / 0.5 < 1e-10


def test_gradient_plane_wave_known_answer(po, pkg, tmp_path):
    # restates ci-test/test_Gradient_R.cpp: for rho(k) = exp(2 pi i k.m) the R-space
    # gradient gives E.grad_k rho = i (R_m . E) rho exactly
    uc = [[2.1650635094610966, 1.25, 0.0], [2.1650635094610966, -1.25, 0.0], [0, 0, 20.0]]
    H = np.zeros((1, 1, 1), complex)
    r = np.zeros((3, 1, 1, 1), complex)
    seed = os.path.join(str(tmp_path), "flat")
    pkg.workloads.write_tb(seed + "_tb.dat", uc, [(0, 0, 0)], H, r)
    N = 12
    inp = pkg.workloads._input(seed, (N, N, 1), 0, 0.01, 10, "RK",
                               [pkg.workloads.sin2_laser(3.0, 1e12, 4, pol=(0.3, 1.0, 0))])
    cfg = po.load_input(inp)
    o = po.Oracle(cfg)
    t = 7.0
    E = o.efield(t)
    assert np.abs(E).max() > 0
    A = o.lattice()
    for m in [(1, 0), (2, -3), (-5, 4)]:
        i0, i1 = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
        phase = np.exp(2j * np.pi * (i0 * m[0] + i1 * m[1]) / N).reshape(-1, 1, 1)
        out = o.rhs(t, phase)
        Rm = A @ np.array([m[0], m[1], 0.0])
        ana = 1j * (Rm @ E) * phase
        assert np.abs(out - ana).max() < 1e-12 * max(1.0, np.abs(ana).max())


def _hsex_cfg(po, pkg, tmp_path, grid, name):
    uc, Rs, H, r = pkg.workloads.random_model(3, 5)
    seed = os.path.join(str(tmp_path), name)
    pkg.workloads.write_tb(seed + "_tb.dat", uc, Rs, H, r)
    inp = pkg.workloads._input(seed, grid, 1, 0.01, 10, "RK",
                               [pkg.workloads.gaussian_laser(1.5, 0.5, 0.02, 0.3, pol=(0.6, 1.0, 0.0))],
                               coulomb=True, epsilon=2.0, r0_A=10.0)
    return po.load_input(inp)


def _herm_part_error(o, t, rho):
    f = o.rhs(t, rho)
    return np.abs(f - np.conj(np.transpose(f, (0, 2, 1)))).max() / np.abs(f).max()


def test_hermitian_nyquist_switch(po, pkg, tmp_path):
    """On an even grid the reference's generator (gradient at the Gamma-centred
    index -N/2, and W there) is not Hermitian-preserving; the oracle's
    hermitian_nyquist switch gives its Hermitian part, which the packed GPU
    forms propagate.  On an odd grid the switch changes nothing."""
    rng = np.random.default_rng(3)
    t = 0.3 / 0.02418884326585747  # near the pulse centre, a.u.
    for grid, even in (((6, 8, 1), True), ((7, 9, 1), False)):
        cfg = _hsex_cfg(po, pkg, tmp_path, grid, "hn%d" % grid[0])
        ref = po.Oracle(cfg)
        cfg.hermitian_nyquist = True
        herm = po.Oracle(cfg)
        x = rng.normal(size=ref.shape) + 1j * rng.normal(size=ref.shape)
        rho = ref.get("rho") + 0.05 * (x + np.conj(np.transpose(x, (0, 2, 1))))
        assert _herm_part_error(herm, t, rho) < 1e-13
        if even:
            assert _herm_part_error(ref, t, rho) > 1e-6
        else:
            assert np.array_equal(ref.rhs(t, rho), herm.rhs(t, rho))
            assert np.array_equal(ref.get("W"), herm.get("W"))


@pytest.mark.skipif(not reference_available(), reason="reference sources not mounted")
def test_hbn_generator_matches_reference_model(po, hbn_golden_model):
    import pyoracle

    ref = os.path.join(REFERENCE, "tb_models", "hBN_gap7.25eV_a2.5A")
    base = dict(grid=[6, 6, 1], filledbands=1, dt=0.01, lasers=[])
    a = pyoracle.Oracle(pyoracle.load_input({**base, "tb_file": ref}))
    b = pyoracle.Oracle(pyoracle.load_input({**base, "tb_file": hbn_golden_model}))
    for name in ("H0k", "xk", "yk", "zk", "rho"):
        assert np.array_equal(a.get(name), b.get(name)), name
    assert np.array_equal(a.lattice(), b.lattice())


def test_k_gradient_converges_to_R_gradient(po, pkg, tmp_path):
    """gradient_space "k" (the finite-difference shells of kGradient.cpp) on a
    plane wave rho(k) = exp(i k.R0): it tends to the exact R-space gradient
    i (R0.E) rho as the grid is refined, with error O((b.R0)^2)."""
    uc = [[2.1650635094610966, 1.25, 0.0], [2.1650635094610966, -1.25, 0.0], [0, 0, 20.0]]
    H = np.zeros((1, 1, 1), complex)
    r = np.zeros((3, 1, 1, 1), complex)
    seed = os.path.join(str(tmp_path), "flatk")
    pkg.workloads.write_tb(seed + "_tb.dat", uc, [(0, 0, 0)], H, r)
    errs = []
    for N in (12, 24, 48):
        inp = pkg.workloads._input(seed, (N, N, 1), 0, 0.01, 10, "RK",
                                   [pkg.workloads.sin2_laser(3.0, 1e12, 4, pol=(0.3, 1.0, 0))])
        inp["gradient_space"] = "k"
        cfg = po.load_input(inp)
        o = po.Oracle(cfg)
        t = 7.0
        E = o.efield(t)
        A = o.lattice()
        i0, i1 = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
        phase = np.exp(2j * np.pi * (i0 * 1 + i1 * 0) / N).reshape(-1, 1, 1)
        out = o.rhs(t, phase)
        ana = 1j * ((A @ np.array([1.0, 0.0, 0.0])) @ E) * phase
        errs.append(np.abs(out - ana).max() / np.abs(ana).max())
    assert errs[0] > errs[1] > errs[2] and errs[2] < 3e-3
    assert errs[1] / errs[2] > 3.5  # second order


def test_k_gradient_stencil_model_equals_property(pkg, tmp_path):
    """The stencil of model.py satisfies sum_b w b_alpha b_beta = delta (per periodic axis)."""
    for grid in ((12, 12, 1), (9, 1, 1), (4, 3, 5)):
        dims = 1 if grid[1] == 1 else (3 if grid[2] > 1 else 2)
        uc, Rs, H, r = pkg.workloads.random_model(2, 0, dims=dims)
        seed = os.path.join(str(tmp_path), f"ks{grid[0]}")
        pkg.workloads.write_tb(seed + "_tb.dat", uc, Rs, H, r)
        inp = pkg.workloads._input(seed, grid, 1, 0.01, 10, "RK", [])
        m = pkg.model.Model(pkg.model.parse_input(inp))
        sh, b, w = m.kgradient_stencil()
        M = np.einsum("i,ia,ib->ab", w, b, b)
        want = np.diag([1.0 if n > 1 else 0.0 for n in grid])
        assert np.abs(M - want).max() < 1e-8
        assert np.abs(np.einsum("i,ia->a", w, b)).max() < 1e-8  # symmetric shells


def _peierls_oracle(po, pkg, tmp_path, name, coulomb, envelope="sin2"):
    uc, Rs, H, r = pkg.workloads.random_model(3, 7)
    seed = os.path.join(str(tmp_path), name)
    pkg.workloads.write_tb(seed + "_tb.dat", uc, Rs, H, r)
    las = ([pkg.workloads.sin2_laser(2.0, 5e12, 3, pol=(1.0, 0.4, 0.2))] if envelope == "sin2" else
           [pkg.workloads.gaussian_laser(1.5, 0.5, 0.02, 0.3, pol=(0.6, 1.0, 0.0))])
    inp = pkg.workloads._input(seed, (6, 8, 1), 1, 0.01, 10, "RK", las, coulomb=coulomb, epsilon=2.0, r0_A=10.0)
    inp["peierls"] = True
    cfg = po.load_input(inp)
    inp2 = dict(inp)
    inp2["peierls"] = False
    return po.Oracle(cfg), po.Oracle(po.load_input(inp2))


def test_peierls_vector_potential_integrator(po, pkg, tmp_path):
    """Laser::VectorPotential (Laser.cpp:136-151): one Simpson step from the
    previous request, none below 1e-7, from A = 0 at t = 0; close to -int E dt."""
    o, _ = _peierls_oracle(po, pkg, tmp_path, "pvec", False, envelope="gauss")
    A = np.zeros(3)
    prev = 0.0
    ts = np.concatenate([np.linspace(0.0, 400.0, 401), [400.0, 400.0 + 5e-8, 401.0]])
    for t in ts:
        got = o.vector_potential(t)
        dT = t - prev
        if dT >= 1e-7:
            A = A - dT / 6.0 * (o.efield(prev) + 4.0 * o.efield(prev + dT / 2.0) + o.efield(t))
            prev = t
        assert np.array_equal(got, A)
    # the rule integrates the field: against a fine trapezoid sum of -E
    fine = np.linspace(0.0, 401.0, 40101)
    Ef = np.array([o.efield(t) for t in fine])
    ref = -np.trapezoid(Ef, fine, axis=0)
    assert np.abs(A - ref).max() < 1e-6 * max(np.abs(ref).max(), 1e-3)


@pytest.mark.parametrize("coulomb", [False, True])
def test_peierls_without_field_is_the_length_gauge(po, pkg, tmp_path, coulomb):
    """Before a sin^2 pulse E = 0 and A = 0: the two gauges give the same source term."""
    op, ol = _peierls_oracle(po, pkg, tmp_path, f"pzero{int(coulomb)}", coulomb)
    rng = np.random.default_rng(3)
    rho = op.get("rho") + 0.1 * (rng.normal(size=op.get("rho").shape) + 1j * rng.normal(size=op.get("rho").shape))
    t = 0.5 * op.cfg.lasers[0].t0
    assert np.array_equal(op.efield(t), np.zeros(3))
    a, b = op.rhs(t, rho), ol.rhs(t, rho)
    assert np.abs(a - b).max() <= 1e-15 * np.abs(b).max()
