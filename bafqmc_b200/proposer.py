"""Learned global proposer: the convolutional network of libbafqmc_b200.so
(bafqmc_net_*), its training on configurations of the plain sampler, and
its parameter files.

The network maps the HS field phi[t][site][aux] of one chain to a Gaussian
proposal phi' = mu(phi) + exp(lsig(phi)) xi, i.e. a Gaussian displacement
mu - phi + exp(lsig) xi from phi (4-layer periodic 3x3x3
convolution over imaginary time and the lattice, 2 -> width -> width ->
width -> 4 channels, bf16 weights, float32 accumulation).  Moves are
accepted by the exact Metropolis-Hastings ratio under the true weight
(Ensemble.learned_move), so the sampler stays unbiased whatever the network
has learned.  The reference has no counterpart: its only global move is the
dead global_update.f90 (accept rule global_update.f90:237-249).
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np

from . import _lib

NTAP = 27
C_IN, C_OUT = 2, 4


def layer_shapes(width: int = 64):
    return [(C_IN, width), (width, width), (width, width), (width, C_OUT)]


def init_params(width: int = 64, seed: int = 0) -> np.ndarray:
    """He-uniform weights (bound sqrt(6 / (27 cin))), zero biases, and a zero
    last layer: the untrained network proposes the prior N(0, 1) for every
    field independently of phi (mu = 0, lsig = 0), a move whose Hastings term
    cancels the Gaussian part of the weight exactly."""
    rng = np.random.default_rng(seed)
    parts = []
    for l, (ci, co) in enumerate(layer_shapes(width)):
        bound = math.sqrt(6.0 / (NTAP * ci)) * (0.0 if l == 3 else 1.0)
        parts.append(rng.uniform(-bound, bound, size=NTAP * co * ci).astype(np.float32))
        parts.append(np.zeros(co, dtype=np.float32))
    return np.concatenate(parts)


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Proposer:
    """One network on one device (bafqmc_net_create)."""

    def __init__(self, Lx: int, Ly: int, Ltrot: int, width: int = 64, device: int = 0, params=None, seed: int = 0):
        self.lib = _lib.load()
        self.Lx, self.Ly, self.Ltrot, self.width = int(Lx), int(Ly), int(Ltrot), int(width)
        h = C.c_void_p()
        _lib.check(self.lib.bafqmc_net_create(self.Lx, self.Ly, self.Ltrot, self.width, int(device), C.byref(h)))
        self.h = h
        self.nparams = int(self.lib.bafqmc_net_num_params(h))
        self.set_params(init_params(self.width, seed) if params is None else params)

    def close(self):
        if getattr(self, "h", None):
            self.lib.bafqmc_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- parameters
    def set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == self.nparams, (p.size, self.nparams)
        _lib.check(self.lib.bafqmc_net_set_params(self.h, _f(p)))

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.nparams, dtype=np.float32)
        _lib.check(self.lib.bafqmc_net_get_params(self.h, _f(p)))
        return p

    def set_tensor_cores(self, enable: bool):
        _lib.check(self.lib.bafqmc_net_set_tensor_cores(self.h, 1 if enable else 0))

    def set_wait_test(self, enable: bool):
        """Test hook: the tensor-core kernels skip their MMAs so their bounded waits expire."""
        _lib.check(self.lib.bafqmc_net_set_wait_test(self.h, 1 if enable else 0))

    def status(self) -> int:
        st = C.c_int32()
        _lib.check(self.lib.bafqmc_net_status(self.h, C.byref(st)))
        return int(st.value)

    # ---- evaluation (host buffers)
    def forward(self, phi: np.ndarray) -> np.ndarray:
        """phi [B, Ltrot, Ns, 2] -> [B, Ltrot, Ns, 4] (mu_0, mu_1, lsig_0, lsig_1)."""
        x = np.ascontiguousarray(phi, dtype=np.float64)
        B = x.shape[0]
        assert x.shape == (B, self.Ltrot, self.Lx * self.Ly, 2)
        out = np.zeros((B, self.Ltrot, self.Lx * self.Ly, 4), dtype=np.float32)
        _lib.check(self.lib.bafqmc_net_forward(self.h, B, _d(x), _f(out)))
        return out

    def loss_grad(self, phi: np.ndarray, target: np.ndarray):
        x = np.ascontiguousarray(phi, dtype=np.float64)
        t = np.ascontiguousarray(target, dtype=np.float64)
        assert x.shape == t.shape
        loss = np.zeros(1, dtype=np.float64)
        grad = np.zeros(self.nparams, dtype=np.float32)
        _lib.check(self.lib.bafqmc_net_loss_grad(self.h, x.shape[0], _d(x), _d(t), _d(loss), _f(grad)))
        return float(loss[0]), grad

    def time_layers(self, chains: int, reps: int = 5) -> np.ndarray:
        """Milliseconds per launch of each forward layer for `chains` chains (CUDA events)."""
        ms = np.zeros(4, dtype=np.float64)
        _lib.check(self.lib.bafqmc_net_time_layers(self.h, int(chains), int(reps), _d(ms)))
        return ms

    # ---- training on the plain sampler's configurations
    def reserve(self, chains: int, slots: int):
        _lib.check(self.lib.bafqmc_net_reserve_data(self.h, int(chains), int(slots)))

    def collect(self, ens):
        _lib.check(self.lib.bafqmc_net_collect(self.h, ens.h))

    def train(self, steps: int, batch: int, lag: int, lr: float, seed: int = 1) -> np.ndarray:
        losses = np.zeros(int(steps), dtype=np.float64)
        _lib.check(self.lib.bafqmc_net_train(self.h, int(steps), int(batch), int(lag), float(lr), int(seed),
                                             _d(losses)))
        return losses

    # ---- files
    def save(self, path, **meta):
        np.savez_compressed(Path(path), params=self.get_params(),
                            shape=np.array([self.Lx, self.Ly, self.Ltrot, self.width], dtype=np.int64),
                            meta=np.array(repr(meta)))

    @classmethod
    def load(cls, path, device: int = 0) -> "Proposer":
        d = np.load(Path(path), allow_pickle=False)
        lx, ly, lt, w = (int(v) for v in d["shape"])
        return cls(lx, ly, lt, w, device=device, params=d["params"])
