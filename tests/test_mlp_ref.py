"""CPU pin of the network checker (oracle/mlp_ref.py): with every operand in
FP64 its gradients equal central finite differences of its loss."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import mlp_ref  # noqa: E402


def test_reference_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    dims = [5, 7, 7, 7, 3]
    n = sum(dims[i] * dims[i + 1] + dims[i + 1] for i in range(4))
    p = rng.normal(scale=0.5, size=n)
    x = rng.normal(size=(6, dims[0]))
    t = rng.normal(size=(6, dims[-1]))
    g, loss = mlp_ref.gradients(p, dims, x, t, round_ops=False)
    h = 1e-6
    for i in rng.choice(n, size=40, replace=False):
        e = np.zeros(n)
        e[i] = h
        lp = mlp_ref.gradients(p + e, dims, x, t, round_ops=False)[1]
        lm = mlp_ref.gradients(p - e, dims, x, t, round_ops=False)[1]
        assert abs((lp - lm) / (2 * h) - g[i]) < 1e-7 * max(1.0, abs(g[i])), i


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-3], dtype=np.float32)
    r = mlp_ref.bf16(x)
    # spacing 2^-7 at 1: 1 + 2^-8 is a tie that rounds to even (1), so is 1 + 3 2^-8 (to 1 + 2^-6)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5
    assert abs(r[4] - 3.0e-3) < 3.0e-3 * 2 ** -8
