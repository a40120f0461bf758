"""Learned HSEX self-energy (no reference counterpart).

The exact Fock term of the reference (Coulomb.cpp:162-171) is, per lattice
vector R and band pair (n, m),

    Hee_nm(R) = -W_nm(R) (rho_nm(R) - rho0_nm(R)),

an elementwise map whose cost is nothing next to the transforms that produce
rho(R) and carry Hee(R) back to k.  The surrogate stands in for it on the R
shells |R| <= r_cut (in lattice vectors):

* factorisation: ONE network shared by all band pairs.  The input of a pair
  is delta rho_nm(R) = rho_nm(R) - rho0_nm(R) on the shells (real and
  imaginary parts), the pair's centre offset c_n - c_m (on which W_nm
  depends) and n/nb, m/nb; the output is Hee_nm(R) on the same shells.  A
  whole state is one batch of nb^2 rows.
* network: `MLP` (3 hidden layers of 128, GELU, BF16 weights, FP32
  accumulation; forward, backward and Adam are the library's CUDA kernels).
* data: (delta rho(R), Hee(R)) pairs generated by the exact FP64 path itself
  under random pulses (`edus_state_rspace` gathers rho(R) on the shells).
* use: `run_predictor_corrector` steps AB4 with the network's Fock term
  (through `edus_set_fock_override`) and recomputes the exact term every
  `judge_every` steps, where it also measures the network's error and falls
  back to the exact term for good when the error exceeds `fallback_tol`.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import edus

HIDDEN = 128


def _torch():
    import torch  # device buffers only: the arithmetic is the library's

    return torch


class MLP:
    """The library's BF16 multilayer perceptron (`edus_mlp_*`)."""

    def __init__(self, n_in: int, n_out: int, hidden: int = HIDDEN, seed: int = 0, device: int = 0):
        self._L = edus.load_library()
        self.n_in, self.n_out, self.hidden, self.device = n_in, n_out, hidden, device
        h = ctypes.c_void_p()
        rc = self._L.edus_mlp_create(n_in, hidden, n_out, seed, device, ctypes.byref(h))
        if rc:
            raise edus.EdusError(rc, self._L.edus_mlp_last_error(None).decode())
        self._h = h
        self.nparams = int(self._L.edus_mlp_param_count(self._h))

    def close(self):
        if getattr(self, "_h", None):
            self._L.edus_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def _check(self, rc):
        if rc:
            raise edus.EdusError(rc, self._L.edus_mlp_last_error(self._h).decode())

    def _dev(self, x):
        torch = _torch()
        t = torch.as_tensor(x, dtype=torch.float32, device=f"cuda:{self.device}").contiguous()
        return t

    def params(self) -> np.ndarray:
        out = np.empty(self.nparams, dtype=np.float32)
        self._check(self._L.edus_mlp_get_params(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparams
        self._check(self._L.edus_mlp_set_params(self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def layer_shapes(self):
        d = [self.n_in, self.hidden, self.hidden, self.hidden, self.n_out]
        return [(d[i], d[i + 1]) for i in range(4)]

    def forward(self, x):
        torch = _torch()
        xd = self._dev(x)
        y = torch.empty((xd.shape[0], self.n_out), dtype=torch.float32, device=xd.device)
        self._check(self._L.edus_mlp_forward(self._h, xd.shape[0], ctypes.c_void_p(xd.data_ptr()),
                                             ctypes.c_void_p(y.data_ptr())))
        return y

    def gradients(self, x, target):
        xd, td = self._dev(x), self._dev(target)
        g = np.empty(self.nparams, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        self._check(self._L.edus_mlp_gradients(self._h, xd.shape[0], ctypes.c_void_p(xd.data_ptr()),
                                               ctypes.c_void_p(td.data_ptr()), g.ctypes.data_as(fp),
                                               loss.ctypes.data_as(fp)))
        return g, float(loss[0])

    def train_step(self, x, target, lr: float) -> float:
        loss = np.zeros(1, dtype=np.float32)
        self._check(self._L.edus_mlp_train_step(self._h, int(x.shape[0]), ctypes.c_void_p(x.data_ptr()),
                                                ctypes.c_void_p(target.data_ptr()), ctypes.c_float(lr),
                                                loss.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return float(loss[0])


def shell_indices(model, r_cut: float):
    """Natural R indices (j0 N1 + j1) N2 + j2 with |R| <= r_cut lattice vectors
    (Cartesian length over the first lattice vector's length)."""
    a1 = np.linalg.norm(model.A[:, 0])
    R = model.Rcart.reshape(-1, 3)
    idx = np.nonzero(np.linalg.norm(R, axis=1) <= r_cut * a1 + 1e-9)[0]
    return idx.astype(np.int32)


class HseSurrogate:
    """Network + feature map for one model (grid, bands, Wannier centres)."""

    def __init__(self, model, r_cut: float = 3.0, seed: int = 0, device: int = 0):
        if not model.cfg.coulomb:
            raise ValueError("the surrogate stands in for the HSEX term: the model needs coulomb=true")
        self.model = model
        self.idx = shell_indices(model, r_cut)
        self.S = len(self.idx)
        nb = model.nb
        self.nb = nb
        # W_nm(R) depends on the pair through the centre offset c_n - c_m (and,
        # under the cumulative-r quirk, on the pair itself): both are features
        c = model.centres
        self.pair_feat = np.array([[*(c[n] - c[m]), n / nb, m / nb] for n in range(nb) for m in range(nb)],
                                  dtype=np.float32)
        self.rho0_R = model.DM0R[self.idx]  # [S][nb][nb]
        self.W_R = np.real(model.W[self.idx])  # [S][nb][nb]
        self.net = MLP(2 * self.S + 5, 2 * self.S, seed=seed, device=device)
        self.x_scale = 1.0
        self.y_scale = 1.0

    # ---- features -------------------------------------------------------
    def features(self, rho_R: np.ndarray) -> np.ndarray:
        """rho_R [S][nb][nb] -> network input [nb^2][2S + 5] (scaled)."""
        d = (rho_R - self.rho0_R).reshape(self.S, -1).T  # [P][S]
        x = np.concatenate([d.real / self.x_scale, d.imag / self.x_scale, self.pair_feat], axis=1)
        return x.astype(np.float32)

    def exact(self, rho_R: np.ndarray) -> np.ndarray:
        """The reference's Fock term on the shells, [S][nb][nb]."""
        return -self.W_R * (rho_R - self.rho0_R)

    def targets(self, hee: np.ndarray) -> np.ndarray:
        h = hee.reshape(self.S, -1).T
        return (np.concatenate([h.real, h.imag], axis=1) / self.y_scale).astype(np.float32)

    def decode(self, y: np.ndarray) -> np.ndarray:
        y = np.asarray(y, dtype=np.float64) * self.y_scale
        h = y[:, : self.S] + 1j * y[:, self.S:]
        return h.T.reshape(self.S, self.nb, self.nb)

    def predict(self, rho_R: np.ndarray) -> np.ndarray:
        y = self.net.forward(self.features(rho_R)).cpu().numpy()
        return self.decode(y)

    # ---- data and training ---------------------------------------------
    def generate(self, n_runs: int, steps: int, every: int, rng: np.random.Generator, laser_factory):
        """(rho(R) on the shells) snapshots of the exact FP64 path under random
        pulses: n_runs runs of `steps` steps, a snapshot every `every` steps."""
        snaps = []
        for _ in range(n_runs):
            s = self.model.solver()
            s.set_lasers(laser_factory(rng))
            for _ in range(steps // every):
                s.step(every)
                snaps.append(state_rspace(s, self.idx))
            del s
        return snaps

    def fit(self, snaps, iters: int = 2000, batch: int = 512, lr: float = 2e-3, rng=None):
        torch = _torch()
        rng = rng or np.random.default_rng(0)
        d = np.stack([r - self.rho0_R for r in snaps])
        if not np.isfinite(d).all():
            raise ValueError("non-finite snapshot: the exact runs that produced the data diverged")
        self.x_scale = float(np.abs(d).max()) or 1.0
        hs = [self.exact(r) for r in snaps]
        self.y_scale = float(max(np.abs(h).max() for h in hs)) or 1.0
        X = np.concatenate([self.features(r) for r in snaps])
        Y = np.concatenate([self.targets(h) for h in hs])
        Xd = torch.as_tensor(X, device=f"cuda:{self.net.device}")
        Yd = torch.as_tensor(Y, device=f"cuda:{self.net.device}")
        losses = []
        n = X.shape[0]
        for it in range(iters):
            sel = torch.as_tensor(rng.integers(0, n, size=min(batch, n)), device=Xd.device)
            losses.append(self.net.train_step(Xd[sel].contiguous(), Yd[sel].contiguous(), lr))
        return losses

    def relative_error(self, snaps) -> float:
        """max |Hee_net - Hee_exact| / max |Hee_exact| over the snapshots."""
        err, ref = 0.0, 0.0
        for r in snaps:
            e = self.exact(r)
            err = max(err, float(np.abs(self.predict(r) - e).max()))
            ref = max(ref, float(np.abs(e).max()))
        return err / max(ref, 1e-300)


def state_rspace(s: "edus.Solver", idx: np.ndarray, b: int = 0) -> np.ndarray:
    """rho(R) of solve b on the natural R indices idx, [len(idx)][nb][nb]."""
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    out = np.empty((len(idx), s.nb, s.nb), dtype=np.complex128)
    s._check(s._L.edus_state_rspace(s._h, b, len(idx), idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                    out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return out


def set_fock(s: "edus.Solver", idx, values):
    """Fock term of the following right-hand sides: `values` [len(idx)][nb][nb]
    on the R indices idx, zero elsewhere; values None restores the exact term."""
    if values is None:
        s._check(s._L.edus_set_fock_override(s._h, 0, None, None))
        return
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    v = np.ascontiguousarray(values, dtype=np.complex128)
    s._check(s._L.edus_set_fock_override(s._h, len(idx), idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                         v.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))


def run_predictor_corrector(s: "edus.Solver", sur: HseSurrogate | None, nsteps: int, judge_every: int = 8,
                            fallback_tol: float = 0.05, frozen: bool = False):
    """AB steps where the Fock term comes from the network (or, with
    frozen=True and no network, is held from the last exact step), with the
    exact term every `judge_every` steps.  At those steps the prediction is
    compared with the exact term; above `fallback_tol` (relative) the run
    falls back to the exact term for the remaining steps.
    The judged error is max|predicted - exact| over max(max|exact|, the largest
    |Hee| of the training data).  Returns (wall seconds, max judged error,
    fell_back)."""
    idx = sur.idx if sur is not None else None
    t0 = time.perf_counter()
    worst, fell_back, held = 0.0, False, None
    for n in range(nsteps):
        if n % judge_every == 0 or fell_back:
            set_fock(s, idx, None)
            if not fell_back and sur is not None:
                rho_R = state_rspace(s, idx)
                exact = sur.exact(rho_R)
                pred = held if frozen else sur.predict(rho_R)
                if pred is not None:
                    # relative to the exact term, or to the training scale of
                    # the term where the exact one is small (delta rho ~ 0)
                    e = float(np.abs(pred - exact).max() / max(np.abs(exact).max(), sur.y_scale))
                    worst = max(worst, e)
                    fell_back = e > fallback_tol
                held = exact
            s.step(1)
            continue
        rho_R = state_rspace(s, idx)
        set_fock(s, idx, held if frozen else sur.predict(rho_R))
        s.step(1)
    set_fock(s, idx, None)
    s.synchronize()
    return time.perf_counter() - t0, worst, fell_back
