"""edus_rhs_noalloc: the right-hand side for callers that cannot let the
library allocate device memory (their GPU memory belongs to another
allocator, or their loop cannot afford cudaMalloc's device-wide sync).

The test owns every device buffer (inputs and output, allocated here with
torch); the entry point keeps its intermediates in the array built into the
library.  Its result must equal the handle-based edus_rhs within the parity
tolerance of the other tests, on two consecutive calls (the second call
reuses the array the first one left behind).  This file is collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _setup(pkg, po, tmp_path, coulomb, nb=3, grid=(12, 10, 1)):
    import os

    uc, Rs, H, r = pkg.workloads.random_model(nb, 11)
    seed = os.path.join(str(tmp_path), f"na{nb}_{grid[0]}x{grid[1]}")
    pkg.workloads.write_tb(seed + "_tb.dat", uc, Rs, H, r)
    inp = pkg.workloads._input(seed, grid, max(1, nb // 2), 0.01, 10, "RK",
                               [pkg.workloads.gaussian_laser(1.5, 0.5, 0.02, 0.3, pol=(0.6, 1.0, 0.0))],
                               coulomb=coulomb, epsilon=2.0, r0_A=10.0)
    cfg = po.load_input(inp)
    o = po.Oracle(cfg)
    s = pkg.Solver(cfg.grid, o.nb, cfg.dt, coulomb=coulomb)
    xi = np.stack([o.get("xk"), o.get("yk"), o.get("zk")])
    if coulomb:
        s.upload_model(o.get("H0k"), xi, o.lattice(), o.get("W"), o.get("DM0R"), o.hartree())
    else:
        s.upload_model(o.get("H0k"), xi, o.lattice())
    s.set_lasers([pkg.Laser(L.intensity, L.omega, L.pol, L.cycles, L.t0, L.phase, L.fwhm, L.envelope)
                  for L in cfg.lasers])
    return cfg, o, s, xi


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.complex128)).cuda()


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


# nb = 3: the CUDA-core commutator; nb = 13: the FP64 tensor-core commutator
@pytest.mark.parametrize("coulomb", [True, False])
@pytest.mark.parametrize("nb,grid", [(3, (12, 10, 1)), (13, (8, 9, 1))])
def test_noalloc_matches_handle_rhs_twice(pkg, po, tmp_path, coulomb, nb, grid):
    torch = pytest.importorskip("torch")
    cfg, o, s, xi = _setup(pkg, po, tmp_path, coulomb, nb, grid)
    lib = pkg.edus.load_library()
    H0 = _dev(torch, o.get("H0k"))
    XI = _dev(torch, xi)
    W = _dev(torch, o.get("W")) if coulomb else None
    R0 = _dev(torch, o.get("DM0R")) if coulomb else None
    HA = _dev(torch, o.hartree()) if coulomb else None
    grid = (ctypes.c_int * 3)(*cfg.grid)
    lat = np.ascontiguousarray(o.lattice(), dtype=np.float64)
    err = ctypes.create_string_buffer(512)
    rng = np.random.default_rng(3)
    for call, t in enumerate((0.2, 3.0)):
        rho = rng.normal(size=o.shape) + 1j * rng.normal(size=o.shape)
        rho = 0.5 * (rho + np.conj(np.transpose(rho, (0, 2, 1))))
        ref = s.rhs(t, rho)                      # the existing entry point
        E = np.ascontiguousarray(o.efield(t), dtype=np.float64)
        din = _dev(torch, rho)
        dout = torch.empty_like(din)
        rc = lib.edus_rhs_noalloc(grid, o.nb, int(coulomb), lat.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                  E.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _ptr(H0), _ptr(XI), _ptr(W),
                                  _ptr(R0), _ptr(HA), _ptr(din), _ptr(dout), None, err, len(err))
        assert rc == 0, err.value.decode()
        torch.cuda.synchronize()
        got = dout.cpu().numpy()
        assert _rel(got, ref) < TOL, (call, _rel(got, ref))


def test_noalloc_rejects_oversized_problem(pkg):
    torch = pytest.importorskip("torch")
    lib = pkg.edus.load_library()
    nb, grid = 22, (72, 72, 1)  # ~40 MB per array: the intermediates exceed the built-in array
    Nk = grid[0] * grid[1] * grid[2]
    dummy = torch.zeros(2, dtype=torch.complex128, device="cuda")
    g = (ctypes.c_int * 3)(*grid)
    lat = np.eye(3)
    E = np.zeros(3)
    err = ctypes.create_string_buffer(512)
    p = ctypes.c_void_p(dummy.data_ptr())
    rc = lib.edus_rhs_noalloc(g, nb, 1, lat.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                              E.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), p, p, p, p, p, p, p, None, err,
                              len(err))
    assert rc == 5  # EDUS_ERR_UNSUPPORTED, before any device work
    assert b"scratch" in err.value
    assert Nk * nb * nb * 16 * 6 > 64 * 1024 * 1024


def _call(lib, torch, cfg, o, xi, coulomb, W_host, rho, t):
    H0 = _dev(torch, o.get("H0k"))
    XI = _dev(torch, xi)
    W = _dev(torch, W_host) if coulomb else None
    R0 = _dev(torch, o.get("DM0R")) if coulomb else None
    HA = _dev(torch, o.hartree()) if coulomb else None
    grid = (ctypes.c_int * 3)(*cfg.grid)
    lat = np.ascontiguousarray(o.lattice(), dtype=np.float64)
    E = np.ascontiguousarray(o.efield(t), dtype=np.float64)
    err = ctypes.create_string_buffer(512)
    din = _dev(torch, rho)
    dout = torch.empty_like(din)
    rc = lib.edus_rhs_noalloc(grid, o.nb, int(coulomb), lat.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                              E.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _ptr(H0), _ptr(XI), _ptr(W),
                              _ptr(R0), _ptr(HA), _ptr(din), _ptr(dout), None, err, len(err))
    assert rc == 0, err.value.decode()
    torch.cuda.synchronize()
    return dout.cpu().numpy()


def test_noalloc_grid_change_and_complex_w(pkg, po, tmp_path):
    """Calls on alternating grids (each change copies that grid's FFT tables
    again) match the handle path; a W with an imaginary part is refused with
    NaN, and the next call with a real W is clean again."""
    torch = pytest.importorskip("torch")
    lib = pkg.edus.load_library()
    rng = np.random.default_rng(5)
    a = _setup(pkg, po, tmp_path, True, 4, (10, 6, 1))
    b = _setup(pkg, po, tmp_path, True, 4, (7, 9, 1))
    for (cfg, o, s, xi), t in ((a, 0.3), (b, 0.5), (a, 0.7)):
        rho = rng.normal(size=o.shape) + 1j * rng.normal(size=o.shape)
        got = _call(lib, torch, cfg, o, xi, True, o.get("W"), rho, t)
        assert _rel(got, s.rhs(t, rho)) < TOL
    cfg, o, s, xi = a
    rho = rng.normal(size=o.shape) + 1j * rng.normal(size=o.shape)
    Wc = o.get("W").copy()
    Wc[3, 1, 2] += 1e-3j
    assert np.isnan(_call(lib, torch, cfg, o, xi, True, Wc, rho, 0.4)).all()
    got = _call(lib, torch, cfg, o, xi, True, o.get("W"), rho, 0.4)
    assert _rel(got, s.rhs(0.4, rho)) < TOL
