"""The benchmark configurations themselves, GPU against the oracle (FP64 bar).

  c0  two-band linear chain, 64x1x1, IPA, Gaussian pulse, RK4 dt = 0.01 fs, all
      2000 steps, state and observables compared along the way;
  c1  hBN-like two bands (t = -2.7 eV), 120x120, IPA, RK4 dt = 0.01 fs, 200
      steps through the pulse in FP64; the SPLIT32 form beside it with its
      error against the FP64 oracle stated and bounded;
  c2  22-orbital TMD-like model, 72x72, HSEX, its own solver (AB4, dt =
      0.005 fs), 20 steps from the pulse centre at full size;
  c3  the batched laser sweep: 16 solves drawn (seeded) from the 256 of the
      sweep (shapes up to 8 bands on 72x72 or the same work, 20 steps), grouped by
      shape into handles with a model per solve and stepped together by
      edus_sweep_step, each against its own oracle.

The oracle itself is pinned to the reference's outputs (test_oracle_reference).
"""
import numpy as np
import pytest

from test_gpu_parity import TOL, lasers_of, make_pair, rel

pytestmark = pytest.mark.gpu
FS = 41.341373335182113  # a.u. of time per fs


def test_c0_chain_2000_steps(pkg, po, tmp_path):
    inp = pkg.workloads.make("chain2", str(tmp_path))
    cfg, o, s = make_pair(pkg, po, inp)
    assert cfg.grid == (64, 1, 1) and cfg.nsteps == 2000
    done = 0
    for chunk in (1, 99, 400, 500, 1000):
        s.step(chunk)
        o.step(chunk)
        done += chunk
        assert rel(s.get_state(), o.get("rho")) < TOL, done
        _, pw, _ = o.observables()
        assert np.abs(s.population_wannier() - pw).max() < 1e-12
    assert done == 2000
    # the pulse did something
    assert np.abs(o.get("rho") - po.Oracle(cfg).get("rho")).max() > 1e-4


def test_c1_hbn_120_fp64_and_split32(pkg, po, tmp_path):
    inp = pkg.workloads.make("hbn2", str(tmp_path), nsteps=200)
    cfg, o, s = make_pair(pkg, po, inp)
    assert cfg.grid == (120, 120, 1)
    t0 = cfg.lasers[0].t0 - 0.5 * cfg.lasers[0].fwhm  # enter the pulse
    s.time = t0
    o.time = t0
    E = pkg.edus
    sp = E.Solver(cfg.grid, o.nb, cfg.dt, precision=E.PREC_SPLIT32)
    xi = np.stack([o.get("xk"), o.get("yk"), o.get("zk")])
    sp.upload_model(o.get("H0k"), xi, o.lattice())
    sp.set_lasers(lasers_of(pkg, cfg))
    sp.set_state(o.get("rho"))
    sp.time = t0
    rho0 = o.get("rho")
    for chunk in (50, 150):
        s.step(chunk)
        sp.step(chunk)
        o.step(chunk)
        ref = o.get("rho")
        assert rel(s.get_state(), ref) < TOL
        err = np.abs(sp.get_state() - ref).max()
        # stated bound of the FP32-transform form on this config
        assert err < 5e-7, err
    assert np.abs(ref - rho0).max() > 1e-3  # the state moved far more than either bound


def test_c2_tmd22_ab4_full_size(pkg, po, tmp_path):
    inp = pkg.workloads.make("tmd22", str(tmp_path), nsteps=20)
    cfg, o, s = make_pair(pkg, po, inp)
    assert cfg.grid == (72, 72, 1) and o.nb == 22 and cfg.coulomb and cfg.solver == 0  # AB
    t = 10.0 * FS  # pulse centre
    s.time = t
    o.time = t
    for chunk in (4, 16):
        s.step(chunk)
        o.step(chunk)
        assert rel(s.get_state(), o.get("rho")) < TOL


def test_c3_sweep_sample_against_oracle(pkg, po, tmp_path):
    E = pkg.edus
    specs = pkg.workloads.sweep_specs(256, seed=2024)
    rng = np.random.default_rng(7)
    # 16 of the 256, the largest shapes left out to keep the oracle's share short
    pool = [i for i, sp in enumerate(specs) if sp["nb"] * sp["nb"] * sp["N"] ** 2 <= 8 * 8 * 72 * 72]
    pick = sorted(rng.choice(pool, size=16, replace=False))
    groups = {}
    for i in pick:
        groups.setdefault((specs[i]["nb"], specs[i]["N"]), []).append(i)
    assert len(groups) >= 5
    nsteps = 20
    handles, members = [], []
    for (nb, N), idx in sorted(groups.items()):
        inps = [pkg.workloads.sweep_input(specs[i], str(tmp_path), nsteps=nsteps) for i in idx]
        oracles = []
        for b, inp in enumerate(inps):
            cfg = po.load_input(inp)
            oracles.append((cfg, po.Oracle(cfg)))
        cfg0, o0 = oracles[0]
        s = E.Solver(cfg0.grid, nb, cfg0.dt, batch=len(idx))
        xi0 = np.stack([o0.get("xk"), o0.get("yk"), o0.get("zk")])
        s.upload_model(o0.get("H0k"), xi0, o0.lattice())
        for b, (cfg, o) in enumerate(oracles):
            if b:
                s.upload_model_solve(b, o.get("H0k"), np.stack([o.get("xk"), o.get("yk"), o.get("zk")]))
            s.set_lasers(lasers_of(pkg, cfg), b)
            s.set_state(o.get("rho"), b)
        s.autotune()
        handles.append(s)
        members.append(oracles)
    E.sweep_step(handles, nsteps, graph=True)
    for s, oracles in zip(handles, members):
        for b, (cfg, o) in enumerate(oracles):
            o.step(nsteps)
            assert rel(s.get_state(b), o.get("rho")) < TOL, (s.nb, b)
