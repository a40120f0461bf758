"""GPU tests of the learned self-energy (no reference counterpart) and of the
two entry points it uses.

* edus_state_rspace: rho(R) of the state equals the k->R transform of
  get_state (1e-12);
* edus_set_fock_override with the exact Fock term on every lattice vector
  reproduces the oracle's right-hand side (1e-10): the override path is exact;
* the network's forward pass and gradients match the CPU checker
  (oracle/mlp_ref.py) within BF16 accumulation differences;
* the gain test: a network trained on data of the exact path, used in the
  predictor-corrector AB4 run (exact term every 8 steps), against the same
  run with the Fock term held from the last exact step (the method without
  the network) and against the exact method.
"""
import os
import sys
import time

import numpy as np
import pytest

from test_gpu_parity import model_input, rel

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import mlp_ref  # noqa: E402

pytestmark = pytest.mark.gpu


def small_hsex(pkg, tmp_path, name, solver="AB", order=4, grid=(12, 12, 1), nb=4):
    # AB4 is stable for |lambda dt| < ~0.43 on the imaginary axis; the gradient
    # term i (R.E) reaches ~0.4 / (0.01 fs) here at the base field, so 0.005 fs
    inp = model_input(pkg, tmp_path, name, grid, nb=nb, coulomb=True, solver=solver, order=order, dt=0.005,
                      envelope="gauss")
    cfg = pkg.model.parse_input(inp)
    return inp, cfg, pkg.model.Model(cfg)


def test_state_rspace_matches_transform(pkg, tmp_path):
    sur = pkg.surrogate
    inp, cfg, m = small_hsex(pkg, tmp_path, "srs")
    s = m.solver()
    s.step(10)
    rho = s.get_state()
    idx = np.arange(m.Nk, dtype=np.int32)[::5]
    got = sur.state_rspace(s, idx)
    ref = pkg.model.fft_k_to_R(rho, m.grid)[idx]
    assert np.abs(got - ref).max() < 1e-12 * max(1.0, np.abs(ref).max())


def test_fock_override_exact_on_all_R(pkg, po, tmp_path):
    sur = pkg.surrogate
    inp, cfg, m = small_hsex(pkg, tmp_path, "sfo", solver="RK")
    o = po.Oracle(po.load_input(inp))
    s = m.solver()
    rng = np.random.default_rng(2)
    x = rng.normal(size=o.shape) + 1j * rng.normal(size=o.shape)
    rho = o.get("rho") + 0.05 * (x + np.conj(np.transpose(x, (0, 2, 1))))
    rho_R = pkg.model.fft_k_to_R(rho, m.grid)
    fock = -np.real(m.W) * (rho_R - m.DM0R)
    idx = np.arange(m.Nk, dtype=np.int32)
    sur.set_fock(s, idx, fock)
    t = 7.0
    assert rel(s.rhs(t, rho), o.rhs(t, rho)) < 1e-10
    # a different Fock term changes the result; clearing restores the exact one
    sur.set_fock(s, idx, 0.5 * fock)
    assert rel(s.rhs(t, rho), o.rhs(t, rho)) > 1e-6
    sur.set_fock(s, idx, None)
    assert rel(s.rhs(t, rho), o.rhs(t, rho)) < 1e-10


# (n_in, n_out, batch): single and multiple 128-wide tiles of the tensor-core
# GEMM in M and N, K chunks of 64 partly filled
@pytest.mark.parametrize("n_in,n_out,batch", [(37, 21, 300), (300, 260, 129)])
def test_mlp_forward_and_gradients_match_cpu_checker(pkg, n_in, n_out, batch):
    sur = pkg.surrogate
    rng = np.random.default_rng(3)
    net = sur.MLP(n_in, n_out, hidden=128, seed=5)
    dims = [n_in, 128, 128, 128, n_out]
    p = net.params()
    assert p.size == net.nparams == sum(dims[i] * dims[i + 1] + dims[i + 1] for i in range(4))
    # non-zero biases so that every term is exercised
    off = 0
    for i in range(4):
        off += dims[i] * dims[i + 1]
        p[off:off + dims[i + 1]] = rng.normal(scale=0.1, size=dims[i + 1])
        off += dims[i + 1]
    net.set_params(p)
    x = rng.normal(size=(batch, n_in)).astype(np.float32)
    t = rng.normal(size=(batch, n_out)).astype(np.float32)
    y_gpu = net.forward(x).cpu().numpy()
    y_ref = mlp_ref.forward(p, dims, x)[0]
    assert np.abs(y_gpu - y_ref).max() < 1e-2 * np.abs(y_ref).max()
    g_gpu, loss_gpu = net.gradients(x, t)
    g_ref, loss_ref = mlp_ref.gradients(p, dims, x, t)
    assert abs(loss_gpu - loss_ref) < 1e-3 * loss_ref
    off = 0
    for i in range(4):
        for n in (dims[i] * dims[i + 1], dims[i + 1]):
            a, b = g_gpu[off:off + n], g_ref[off:off + n]
            assert np.linalg.norm(a - b) < 2e-2 * np.linalg.norm(b), (i, n)
            off += n


def test_mlp_learns_a_linear_map(pkg):
    torch = pytest.importorskip("torch")
    sur = pkg.surrogate
    rng = np.random.default_rng(4)
    A = rng.normal(size=(16, 8)) / 4
    net = sur.MLP(16, 8, seed=1)
    X = rng.normal(size=(4096, 16)).astype(np.float32)
    Y = (X @ A).astype(np.float32)
    Xd, Yd = torch.as_tensor(X, device="cuda"), torch.as_tensor(Y, device="cuda")
    first = net.train_step(Xd, Yd, 1e-3)
    for _ in range(1500):
        last = net.train_step(Xd, Yd, 1e-3)
    assert last < 1e-2 * first


def test_surrogate_gain(pkg, tmp_path):
    """What the trained network gains over the method without it.

    Both predictor-corrector runs make the same calls per step (gather rho(R),
    set the Fock term, step); they differ in where the Fock term of the seven
    steps between exact ones comes from: the network, or the last exact term.
    The exact method recomputes the term every step inside the plane kernel."""
    sur = pkg.surrogate
    inp, cfg, m = small_hsex(pkg, tmp_path, "sgain")
    hs = sur.HseSurrogate(m, r_cut=3.0, seed=0)
    rng = np.random.default_rng(7)
    base = cfg.lasers[0]

    def lasers(r):
        L = pkg.Laser(base.intensity * r.uniform(0.2, 1.5), base.omega * r.uniform(0.7, 1.3),
                      tuple(r.normal(size=2).tolist()) + (0.0,), base.cycles, base.t0, r.uniform(0, 6.28),
                      base.fwhm, base.envelope)
        return [L]

    train = hs.generate(n_runs=6, steps=960, every=16, rng=rng, laser_factory=lasers)
    held = hs.generate(n_runs=1, steps=960, every=16, rng=rng, laser_factory=lasers)
    losses = hs.fit(train, iters=3000, batch=1024, lr=2e-3, rng=rng)
    assert losses[-1] < 0.05 * losses[0]
    err_held = hs.relative_error(held)

    nsteps = 960
    ref = m.solver()
    t0 = time.perf_counter()
    ref.step(nsteps)
    ref.synchronize()
    t_exact = time.perf_counter() - t0
    rho_exact = ref.get_state()

    s_net = m.solver()
    t_net, judged_net, fb_net = sur.run_predictor_corrector(s_net, hs, nsteps, judge_every=8, fallback_tol=1.0)
    s_frz = m.solver()
    t_frz, judged_frz, fb_frz = sur.run_predictor_corrector(s_frz, hs, nsteps, judge_every=8, fallback_tol=1.0,
                                                            frozen=True)
    scale = np.abs(rho_exact - m.rho0k).max()
    e_net = np.abs(s_net.get_state() - rho_exact).max() / scale
    e_frz = np.abs(s_frz.get_state() - rho_exact).max() / scale
    print(f"\nsurrogate gain: held-out Fock error {err_held:.3e}; trajectory error vs exact "
          f"(relative to the change of rho): network {e_net:.3e}, held Fock term {e_frz:.3e}; "
          f"judged Fock error network {judged_net:.3e}, held {judged_frz:.3e}; "
          f"wall s/step: exact {t_exact / nsteps:.2e}, network {t_net / nsteps:.2e}, held {t_frz / nsteps:.2e}")
    assert err_held < 0.2
    assert e_net < e_frz  # the network beats the term held from the last exact step
    assert judged_net < judged_frz
