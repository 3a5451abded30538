"""Learned warm start of the circulation solve (no counterpart in the reference).

A per-panel MLP (8 features -> 3 x 256 GELU -> 1; BF16 weights, FP32
accumulation; forward, backward and Adam run as the library's own CUDA
kernels) predicts the correction of the extrapolation 2 G_n - G_{n-1}.  The
training pairs come from the solver itself: ``SimpleSimulator`` records them
with ``collect_training_data`` while a run advances.

Typical use::

    X, T = collect(make_sim, kinematics_list, steps, dt)    # plain FP64 solver
    net = MLP(seed=0); net.fit_normalization(X, T); net.train(X, T, epochs=20)
    sim = SimpleSimulator(precision="mixed", warm_start="mlp"); sim.set_mlp(net)
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import check, lib

N_FEATURES = 8
FEATURES = ("gamma_n", "gamma_n - gamma_n-1", "rhs_n+1", "rhs_n+1 - rhs_n", "sin phase", "cos phase",
            "chord position", "span position")

_F = C.POINTER(C.c_float)


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _pf(a):
    return a.ctypes.data_as(_F)


class MLP:
    """Handle of a uvlm_mlp on the current CUDA device."""

    def __init__(self, seed: int = 0):
        h = C.c_void_p()
        check(lib().uvlm_mlp_create(int(seed), C.byref(h)))
        self._h = h
        self.mean = np.zeros(N_FEATURES, np.float32)
        self.std = np.ones(N_FEATURES, np.float32)
        self.out_scale = 1.0

    @property
    def handle(self):
        return self._h

    def num_params(self) -> int:
        return int(lib().uvlm_mlp_num_params(self._h))

    def params(self) -> np.ndarray:
        p = np.zeros(self.num_params(), np.float32)
        check(lib().uvlm_mlp_get_params(self._h, _pf(p)))
        return p

    def set_params(self, p) -> None:
        p = _f32(p)
        assert p.size == self.num_params()
        check(lib().uvlm_mlp_set_params(self._h, _pf(p)))

    def set_normalization(self, mean, std, out_scale) -> None:
        self.mean, self.std, self.out_scale = _f32(mean), _f32(std), float(out_scale)
        check(lib().uvlm_mlp_set_normalization(self._h, _pf(self.mean), _pf(self.std), C.c_float(self.out_scale)))

    def fit_normalization(self, X, T) -> None:
        X = np.asarray(X, np.float64)
        std = X.std(axis=0)
        std[std < 1e-12] = 1.0
        out = float(np.std(T)) or 1.0
        self.set_normalization(X.mean(axis=0), std, out)

    def forward(self, X) -> np.ndarray:
        X = _f32(X).reshape(-1, N_FEATURES)
        y = np.zeros(X.shape[0], np.float32)
        check(lib().uvlm_mlp_forward(self._h, _pf(X), X.shape[0], _pf(y)))
        return y

    def forward_tc(self, X) -> np.ndarray:
        """The same network on the tcgen05 tensor cores (BF16 activations in the hidden layers): the inference
        the time-stepper uses for its learned warm start."""
        X = _f32(X).reshape(-1, N_FEATURES)
        y = np.zeros(X.shape[0], np.float32)
        check(lib().uvlm_mlp_forward_tc(self._h, _pf(X), X.shape[0], _pf(y)))
        return y

    def gradients(self, X, T):
        X = _f32(X).reshape(-1, N_FEATURES)
        T = _f32(T).reshape(-1)
        g = np.zeros(self.num_params(), np.float32)
        loss = C.c_double()
        check(lib().uvlm_mlp_gradients(self._h, _pf(X), _pf(T), X.shape[0], _pf(g), C.byref(loss)))
        return g, loss.value

    def train(self, X, T, epochs=10, batch=4096, lr=1e-3, seed=0) -> float:
        X = _f32(X).reshape(-1, N_FEATURES)
        T = _f32(T).reshape(-1)
        loss = C.c_double()
        check(lib().uvlm_mlp_train(self._h, _pf(X), _pf(T), X.shape[0], int(epochs), int(batch), float(lr),
                                   int(seed), C.byref(loss)))
        return loss.value

    def save(self, path) -> None:
        np.savez_compressed(path, params=self.params(), mean=self.mean, std=self.std, out_scale=self.out_scale)

    @classmethod
    def load(cls, path) -> "MLP":
        d = np.load(path)
        net = cls()
        net.set_params(d["params"])
        net.set_normalization(d["mean"], d["std"], float(d["out_scale"]))
        return net

    def layers(self):
        """(W, b) per layer from the parameter vector (W is [in][out])."""
        p = self.params()
        dims = [N_FEATURES, 256, 256, 256, 1]
        out, off = [], 0
        for i in range(4):
            W = p[off:off + dims[i] * dims[i + 1]].reshape(dims[i], dims[i + 1])
            off += dims[i] * dims[i + 1]
            b = p[off:off + dims[i + 1]]
            off += dims[i + 1]
            out.append((W, b))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().uvlm_mlp_destroy(h)
            except Exception:
                pass
            self._h = None


def collect(make_sim, variants, steps, dt, max_samples=None):
    """Runs ``make_sim(variant)`` for each variant with data collection on and
    returns the concatenated (X [n][8], T [n]) training pairs."""
    Xs, Ts = [], []
    for v in variants:
        sim = make_sim(v)
        n_panels = None
        sim.begin()
        num, rows, cols, _, _ = sim.sizes()
        n_panels = num * rows * cols
        cap = max_samples or n_panels * (steps + 1)
        sim.collect_training_data(True, cap)
        for s in range(steps + 1):
            sim.step(s, dt)
        X, T = sim.training_data()
        Xs.append(X)
        Ts.append(T)
        sim.close()
    return np.concatenate(Xs), np.concatenate(Ts)
