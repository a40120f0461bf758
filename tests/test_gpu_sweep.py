"""GPU tests of sweeps: a model per solve, several handles stepped together
(one CUDA graph per chunk of steps), and the launch-variant autotuner.

The sweep must be invisible in the results: every solve equals the same solve
stepped alone (bit for bit: the same kernels on the same data), and solves
with models of their own match the oracle at the FP64 bar (1e-10 relative).
"""
import numpy as np
import pytest

from test_gpu_parity import lasers_of, model_input, rel

pytestmark = pytest.mark.gpu


def oracle_of(po, inp):
    cfg = po.load_input(inp)
    return cfg, po.Oracle(cfg)


def upload(s, o, coulomb=False):
    xi = np.stack([o.get("xk"), o.get("yk"), o.get("zk")])
    if coulomb:
        s.upload_model(o.get("H0k"), xi, o.lattice(), o.get("W"), o.get("DM0R"), o.hartree())
    else:
        s.upload_model(o.get("H0k"), xi, o.lattice())


def test_model_per_solve_matches_oracle(pkg, po, tmp_path):
    E = pkg.edus
    pairs = [oracle_of(po, model_input(pkg, tmp_path, f"ms{seed}", (8, 6, 1), nb=3, seed=seed, dt=0.01,
                                       envelope="gauss")) for seed in (0, 1, 2)]
    cfg0, o0 = pairs[0]
    s = E.Solver(cfg0.grid, o0.nb, cfg0.dt, batch=3)
    upload(s, o0)
    for b, (cfg, o) in enumerate(pairs):
        if b:
            s.upload_model_solve(b, o.get("H0k"), np.stack([o.get("xk"), o.get("yk"), o.get("zk")]))
        s.set_lasers(lasers_of(pkg, cfg), b)
        s.set_state(o.get("rho"), b)
    s.step(10)
    for b, (cfg, o) in enumerate(pairs):
        o.step(10)
        assert rel(s.get_state(b), o.get("rho")) < 1e-10, b


def test_model_per_solve_refused_with_hsex(pkg, po, tmp_path):
    E = pkg.edus
    cfg, o = oracle_of(po, model_input(pkg, tmp_path, "msh", (6, 6, 1), nb=2, coulomb=True))
    s = E.Solver(cfg.grid, o.nb, cfg.dt, coulomb=True, batch=2)
    upload(s, o, coulomb=True)
    with pytest.raises(E.EdusError) as ei:
        s.upload_model_solve(1, o.get("H0k"), np.stack([o.get("xk"), o.get("yk"), o.get("zk")]))
    assert ei.value.code == 5


SHAPES = [  # nb, grid, seed
    (2, (24, 24, 1), 3),
    (4, (12, 12, 1), 4),
    (8, (8, 6, 1), 5),
]


def make_sweep(pkg, po, tmp_path, tag):
    E = pkg.edus
    out = []
    for nb, grid, seed in SHAPES:
        inp = model_input(pkg, tmp_path, f"sw{tag}{nb}", grid, nb=nb, seed=seed, dt=0.01, envelope="gauss")
        cfg, o = oracle_of(po, inp)
        s = E.Solver(cfg.grid, o.nb, cfg.dt, batch=2)
        upload(s, o)
        for b in range(2):
            s.set_lasers(lasers_of(pkg, cfg), b)
            s.set_state(o.get("rho"), b)
        out.append(s)
    return out


@pytest.mark.parametrize("graph", [True, False])
def test_sweep_equals_separate_steps(pkg, po, tmp_path, graph):
    E = pkg.edus
    swept = make_sweep(pkg, po, tmp_path, "a")
    alone = make_sweep(pkg, po, tmp_path, "b")
    E.sweep_step(swept, 70, graph=graph)  # two full chunks of 32 and a partial one
    for s in alone:
        s.step(70)
    for s1, s2 in zip(swept, alone):
        assert abs(s1.time - s2.time) == 0.0
        for b in range(2):
            assert np.array_equal(s1.get_state(b), s2.get_state(b))
    # the sweep handles keep stepping normally afterwards
    for s in swept:
        s.step(3)
        assert np.isfinite(s.get_state()).all()


# shapes for the fused sweep: small planes (two CTAs per SM), a plane above
# 110 KB (96 x 96: the large-plane launch), CUDA-core and FP64 tensor-core
# commutators (13 and 14 bands), odd and even band counts
FUSED_SHAPES = [  # nb, grid, seed, batch
    (2, (96, 96, 1), 21, 2),
    (3, (24, 24, 1), 22, 3),
    (13, (8, 6, 1), 23, 2),
    (14, (12, 12, 1), 24, 1),
    (4, (36, 36, 1), 25, 2),
]


def make_fused_sweep(pkg, po, tmp_path, tag, tune=False):
    E = pkg.edus
    out = []
    for nb, grid, seed, batch in FUSED_SHAPES:
        inp = model_input(pkg, tmp_path, f"fs{tag}{nb}", grid, nb=nb, seed=seed, dt=0.01, envelope="gauss")
        cfg, o = oracle_of(po, inp)
        s = E.Solver(cfg.grid, o.nb, cfg.dt, batch=batch)
        upload(s, o)
        for b in range(batch):
            s.set_lasers(lasers_of(pkg, cfg), b)
            s.set_state(o.get("rho"), b)
        if tune:
            s.autotune()
        out.append((s, cfg, o))
    return out


def _uses_plane3(s):
    """A handle alone spreads each plane over many CTAs (axis 1 first) when a
    2-D grid of 1024+ points has fewer planes x solves than SMs; its sums then
    run in another order than the whole-plane transform of the fused launch."""
    import torch

    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    N = s.grid
    return N[2] == 1 and N[1] > 1 and N[0] * N[1] >= 1024 and s.nb * s.nb * s.batch < nsm


def test_fused_sweep_equals_separate_and_oracle(pkg, po, tmp_path):
    """One persistent launch per stage for every solve of every shape: bit for
    bit what stepping each handle alone gives (to rounding where the handle
    alone takes the many-CTA plane path), and the oracle at 1e-10."""
    E = pkg.edus
    fused = make_fused_sweep(pkg, po, tmp_path, "a")
    alone = make_fused_sweep(pkg, po, tmp_path, "b")
    E.sweep_step([s for s, _, _ in fused], 37, fused=True)  # a captured chunk of 32 and 5 steps more
    for s, _, _ in alone:
        s.step(37)
    for (s1, cfg, o), (s2, _, _) in zip(fused, alone):
        assert s1.time == s2.time
        for b in range(s1.batch):
            if _uses_plane3(s2):
                assert rel(s1.get_state(b), s2.get_state(b)) < 1e-13, (s1.nb, b)
            else:
                assert np.array_equal(s1.get_state(b), s2.get_state(b)), (s1.nb, b)
        o.step(37)
        assert rel(s1.get_state(0), o.get("rho")) < 1e-10


def test_fused_sweep_after_autotune(pkg, po, tmp_path):
    """The autotuner's choices (thread counts, tensor-core commutator down to
    small band counts) carry over to the fused launches."""
    E = pkg.edus
    fused = make_fused_sweep(pkg, po, tmp_path, "c", tune=True)
    E.sweep_step([s for s, _, _ in fused], 10, fused=True)
    for s, cfg, o in fused:
        o.step(10)
        for b in range(s.batch):
            assert rel(s.get_state(b), o.get("rho")) < 1e-10, (s.nb, b)


def test_fused_sweep_refuses_hsex(pkg, po, tmp_path):
    E = pkg.edus
    cfg, o = oracle_of(po, model_input(pkg, tmp_path, "fsh", (6, 6, 1), nb=2, coulomb=True))
    s = E.Solver(cfg.grid, o.nb, cfg.dt, coulomb=True)
    upload(s, o, coulomb=True)
    s.set_state(o.get("rho"))
    with pytest.raises(E.EdusError) as ei:
        E.sweep_step([s], 4, fused=True)
    assert ei.value.code == 5


def test_sweep_rejects_duplicates_and_packed(pkg, po, tmp_path):
    E = pkg.edus
    sw = make_sweep(pkg, po, tmp_path, "c")
    with pytest.raises(E.EdusError):
        E.sweep_step([sw[0], sw[0]], 4)
    cfg, o = oracle_of(po, model_input(pkg, tmp_path, "swp", (6, 6, 1), nb=2))
    p = E.Solver(cfg.grid, 2, cfg.dt, precision=E.PREC_HERM64)
    upload(p, o)
    p.set_state(o.get("rho"))
    with pytest.raises(E.EdusError) as ei:
        E.sweep_step([sw[1], p], 4)
    assert ei.value.code == 5


@pytest.mark.parametrize("nb,grid,coulomb", [(4, (12, 12, 1), False), (13, (8, 9, 1), True), (2, (72, 8, 1), False)])
def test_autotune_keeps_results(pkg, po, tmp_path, nb, grid, coulomb):
    E = pkg.edus
    inp = model_input(pkg, tmp_path, f"at{nb}", grid, nb=nb, coulomb=coulomb, dt=0.01, envelope="gauss")
    cfg, o = oracle_of(po, inp)
    s = E.Solver(cfg.grid, o.nb, cfg.dt, coulomb=coulomb)
    upload(s, o, coulomb)
    s.set_lasers(lasers_of(pkg, cfg))
    s.set_state(o.get("rho"))
    threads, tensor = s.autotune()
    assert 128 <= threads <= 768 and threads % 32 == 0
    assert rel(s.get_state(), o.get("rho")) < 1e-15  # the state is untouched
    s.step(6)
    o.step(6)
    assert rel(s.get_state(), o.get("rho")) < 1e-10
