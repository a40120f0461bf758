"""Sharding of a laser sweep across ranks (CPU; world size 2 over gloo).

The partition deals whole solves to ranks by predicted cost (no data-path
collective); the ranks meet once at the end to gather observables.  Here each
rank propagates its share with the oracle (a stand-in for its GPU, which this
test does not need), and the gathered results must equal a one-process run
of the whole sweep, solve for solve.
"""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _specs(pkg, n=12):
    # small shapes so the oracle propagates them in a fraction of a second
    specs = pkg.workloads.sweep_specs(n, seed=11)
    for i, sp in enumerate(specs):
        sp["nb"] = (2, 3, 4)[i % 3]
        sp["N"] = (6, 8, 9, 10)[i % 4]
    return specs


def _propagate(po, pkg, spec, tmp, steps=5):
    inp = pkg.workloads.sweep_input(spec, tmp, nsteps=steps)
    o = po.Oracle(po.load_input(inp))
    o.step(steps)
    _, pw, _ = o.observables()
    return pw


def test_partition_is_complete_disjoint_and_balanced(pkg):
    sw = pkg.sweep
    specs = pkg.workloads.sweep_specs(256, seed=2024)
    for world in (1, 2, 3, 8):
        parts = sw.partition(specs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        L = sw.loads(specs, parts)
        # LPT: the heaviest rank exceeds the mean by at most the largest single solve
        assert max(L) - sum(L) / world <= max(sw.solve_cost(s) for s in specs) + 1e-6
    assert sw.partition(specs, 4) == sw.partition(specs, 4)


def _rank_main(rank, world, port, root, tmp, out):
    import sys

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import torch.distributed as dist

    import __graft_entry__ as ge
    import pyoracle as po

    pkg = ge.load_package()
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs = _specs(pkg)
        mine = pkg.sweep.partition(specs, world)[rank]
        local = {i: _propagate(po, pkg, specs[i], os.path.join(tmp, f"r{rank}")) for i in mine}
        merged = pkg.sweep.gather(local, world)
        if rank == 0:
            np.save(out, np.concatenate([merged[i] for i in range(len(specs))]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_match_one_process(pkg, po, tmp_path):
    import torch.multiprocessing as mp

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = os.path.join(str(tmp_path), "merged.npy")
    mp.spawn(_rank_main, args=(2, _free_port(), root, str(tmp_path), out), nprocs=2, join=True)
    merged = np.load(out)
    specs = _specs(pkg)
    serial = np.concatenate([_propagate(po, pkg, sp, os.path.join(str(tmp_path), "serial")) for sp in specs])
    assert merged.shape == serial.shape
    assert np.array_equal(merged, serial)


def test_gather_rejects_a_solve_on_two_ranks(pkg, monkeypatch):
    import torch.distributed as dist

    def fake_all_gather(parts, local):
        parts[0] = {0: 1.0}
        parts[1] = {0: 2.0}

    monkeypatch.setattr(dist, "all_gather_object", fake_all_gather)
    with pytest.raises(RuntimeError):
        pkg.sweep.gather({0: 1.0}, 2)
