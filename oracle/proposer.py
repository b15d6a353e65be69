"""CPU oracle of the learned global proposer (convolutional network over the
(imaginary time x site) HS field) and of its Metropolis-Hastings move.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU legs of ``bench.py`` may import it; the product path (``bafqmc_b200``)
never does.

The reference has no learned proposer.  Its only global move is the dead
``src/number_conserving/src/global_update.f90`` (not in the Makefile), whose
accept rule ``exp(log w' - log w) >= u`` (global_update.f90:237-249) the move
below keeps, with the Hastings factor q(phi|phi') / q(phi'|phi) of a
non-symmetric proposal added to the exponent.  This module defines the network
that the CUDA kernels must reproduce, and is itself pinned by finite
differences of its float64 form (``tests/test_proposer_oracle.py``).

Network (one chain; fields phi[t][site][aux] in the confin order, site =
y*Lx + x, periodic in t, y and x):

  x0 = bf16(phi)                                        (2 channels)
  pre_l[p][o] = b_l[o] + sum_{tap, i} W_l[tap][o][i] x_{l-1}[nbr(p, tap)][i]
  x_l = bf16(relu(pre_l))                               l = 1, 2, 3 (C channels)
  out = pre_4                                           4 channels: mu_0, mu_1, lsig_0, lsig_1

with taps (a, b, c) in {-1, 0, 1}^3, nbr((t, y, x), (a, b, c)) =
((t + a) mod L, (y + b) mod Ly, (x + c) mod Lx), and the tap index
k = 3 * ((b + 1) * 3 + (c + 1)) + (a + 1).  Weights are bf16 values (the
float32 master copy rounded), accumulation is float32 on the device.

Proposal: phi' = mu(phi) + exp(lsig(phi)) * xi, xi ~ N(0, 1) per field, i.e.
the Gaussian displacement phi' - phi = (mu - phi) + exp(lsig) xi: the network
emits the mean mu of the proposed field (a skip connection from the input),
so a network whose last layer is zero proposes the prior N(0, 1)
independently of phi, a move the Gaussian part of the weight accepts with
ratio 1 exactly.  xi is drawn from the chain's LCG by the reference's
Box-Muller form (two draws per value, fields.f90:280-288) in the field
order.  log q(phi'|phi) = sum(-xi^2 / 2 - lsig(phi)) (constants cancel in
the ratio).

Training loss for a pair (phi, phi_target) (a configuration of the plain
sampler and one `lag` sweeps later in the same chain):
  L = mean over fields of [ z^2 / 2 + lsig ],  z = (phi_target - mu) exp(-lsig)
(the Gaussian negative log-likelihood of the transition), averaged over the
batch.  Backward: gradients of the pre-activations are rounded to bf16 before
they feed the transposed convolutions (the device stores them in bf16).
"""
from __future__ import annotations

import math

import numpy as np

NTAP = 27
C_IN = 2
C_OUT = 4


def tap_offsets():
    """(a, b, c) for tap index k = 3 * ((b + 1) * 3 + (c + 1)) + (a + 1)."""
    out = []
    for k in range(NTAP):
        a = k % 3 - 1
        bc = k // 3
        b = bc // 3 - 1
        c = bc % 3 - 1
        out.append((a, b, c))
    return out


TAPS = tap_offsets()


def layer_shapes(width: int = 64):
    """(cin, cout) per layer."""
    return [(C_IN, width), (width, width), (width, width), (width, C_OUT)]


def num_params(width: int = 64) -> int:
    return sum(NTAP * co * ci + co for ci, co in layer_shapes(width))


def unpack(params: np.ndarray, width: int = 64):
    """Flat float32 parameter vector -> [(W [27][cout][cin], b [cout])] per layer."""
    out, off = [], 0
    for ci, co in layer_shapes(width):
        n = NTAP * co * ci
        W = params[off:off + n].reshape(NTAP, co, ci)
        off += n
        b = params[off:off + co]
        off += co
        out.append((W, b))
    assert off == params.size
    return out


def init_params(width: int = 64, seed: int = 0, last_scale: float = 0.0) -> np.ndarray:
    """He-uniform weights (bound sqrt(6 / (27 cin))), zero biases; the last
    layer scaled by last_scale (0: the prior's independence sampler)."""
    rng = np.random.default_rng(seed)
    parts = []
    for l, (ci, co) in enumerate(layer_shapes(width)):
        bound = math.sqrt(6.0 / (NTAP * ci)) * (last_scale if l == 3 else 1.0)
        parts.append(rng.uniform(-bound, bound, size=NTAP * co * ci).astype(np.float32))
        parts.append(np.zeros(co, dtype=np.float32))
    return np.concatenate(parts)


# ---------------------------------------------------------------------------
def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (round to nearest even), returned as float32."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(f.shape)


def _shift(x: np.ndarray, a: int, b: int, c: int) -> np.ndarray:
    """y[t, y, x] = x[t + a, y + b, x + c] (periodic) for x of shape [B, L, Ly, Lx, C]."""
    return np.roll(x, shift=(-a, -b, -c), axis=(1, 2, 3))


def conv(x: np.ndarray, W: np.ndarray, b: np.ndarray, dtype=np.float64) -> np.ndarray:
    """Periodic 3x3x3 convolution: x [B, L, Ly, Lx, cin] -> [B, L, Ly, Lx, cout]."""
    out = np.broadcast_to(b.astype(dtype), x.shape[:4] + (W.shape[1],)).copy()
    xd = x.astype(dtype)
    for k, (a, bb, c) in enumerate(TAPS):
        out += _shift(xd, a, bb, c) @ W[k].T.astype(dtype)
    return out


def conv_transpose(g: np.ndarray, W: np.ndarray, dtype=np.float64) -> np.ndarray:
    """Gradient w.r.t. the input of `conv` for output gradient g [.., cout] -> [.., cin]."""
    out = np.zeros(g.shape[:4] + (W.shape[2],), dtype=dtype)
    gd = g.astype(dtype)
    for k, (a, bb, c) in enumerate(TAPS):
        out += _shift(gd, -a, -bb, -c) @ W[k].astype(dtype)
    return out


def conv_wgrad(x: np.ndarray, g: np.ndarray, dtype=np.float64) -> np.ndarray:
    """dW[k][o][i] = sum_p g[p][o] x[nbr(p, k)][i]."""
    cin, cout = x.shape[-1], g.shape[-1]
    gd = g.astype(dtype).reshape(-1, cout)
    dW = np.zeros((NTAP, cout, cin), dtype=dtype)
    xd = x.astype(dtype)
    for k, (a, bb, c) in enumerate(TAPS):
        dW[k] = gd.T @ _shift(xd, a, bb, c).reshape(-1, cin)
    return dW


def to_grid(phi: np.ndarray, Lx: int, Ly: int) -> np.ndarray:
    """phi [B, L, Ns, 2] (confin order, site = y*Lx + x) -> [B, L, Ly, Lx, 2]."""
    B, L, ns, na = phi.shape
    assert ns == Lx * Ly and na == 2
    return phi.reshape(B, L, Ly, Lx, 2)


def forward(params: np.ndarray, phi: np.ndarray, Lx: int, Ly: int, width: int = 64, rounding: bool = True,
            keep: bool = False):
    """Network output [B, L, Ns, 4] (mu_0, mu_1, lsig_0, lsig_1) for fields [B, L, Ns, 2].

    rounding=True mirrors the device (bf16 weights and activations, float32
    outputs); rounding=False is the float64 network the finite-difference
    check differentiates."""
    layers = unpack(np.asarray(params, dtype=np.float32 if rounding else np.float64), width)
    r = bf16 if rounding else (lambda v: np.asarray(v, dtype=np.float64))
    x = r(to_grid(np.asarray(phi, dtype=np.float64 if not rounding else np.float32), Lx, Ly))
    acts = [x]
    out = None
    for l, (W, b) in enumerate(layers):
        Wr = bf16(W) if rounding else W.astype(np.float64)
        pre = conv(x, Wr, b.astype(np.float64))
        if l < 3:
            x = r(np.maximum(pre, 0.0))
            acts.append(x)
        else:
            out = pre.astype(np.float32) if rounding else pre
    B, L = phi.shape[:2]
    out = out.reshape(B, L, Lx * Ly, C_OUT)
    return (out, acts) if keep else out


def loss_and_grad(params: np.ndarray, phi: np.ndarray, target: np.ndarray, Lx: int, Ly: int, width: int = 64,
                  rounding: bool = True):
    """Mean Gaussian NLL of target under N(mu, exp(lsig)^2) and its
    gradient w.r.t. the flat parameter vector (same layout as params)."""
    layers = unpack(np.asarray(params, dtype=np.float32 if rounding else np.float64), width)
    out, acts = forward(params, phi, Lx, Ly, width, rounding, keep=True)
    B, L, ns, _ = phi.shape
    nf = B * L * ns * 2
    o = out.astype(np.float64)
    m, ls = o[..., 0:2], o[..., 2:4]
    z = (np.asarray(target, np.float64) - m) * np.exp(-ls)
    loss = float(np.sum(0.5 * z * z + ls) / nf)
    g = np.empty_like(o)
    g[..., 0:2] = -z * np.exp(-ls) / nf
    g[..., 2:4] = (1.0 - z * z) / nf
    g = g.reshape(B, L, Ly, Lx, C_OUT)
    r = bf16 if rounding else (lambda v: v)
    grads = [None] * 4
    for l in range(3, -1, -1):
        W, b = layers[l]
        Wr = bf16(W) if rounding else W.astype(np.float64)
        gl = r(g)
        x = acts[l]
        grads[l] = (conv_wgrad(x, gl), np.asarray(gl, np.float64).sum(axis=(0, 1, 2, 3)))
        if l > 0:
            dx = conv_transpose(gl, Wr)
            g = dx * (acts[l] > 0)
    flat = np.concatenate([np.concatenate([dW.ravel(), db.ravel()]) for dW, db in grads])
    return loss, flat


# ---------------------------------------------------------------------------
# the move
def gaussians(seed: int, n: int) -> tuple[int, np.ndarray]:
    """n values of the reference's Box-Muller form (fields.f90:280-288) from the LCG."""
    LCG_A, LCG_M = 48828125, 2147483648
    out = np.empty(n)
    for k in range(n):
        seed = (LCG_A * seed) % LCG_M
        x1 = seed / LCG_M
        seed = (LCG_A * seed) % LCG_M
        x2 = seed / LCG_M
        out[k] = math.sqrt(-2.0 * math.log(x1)) * math.cos(2.0 * math.pi * x2)
    return seed, out


def log_q(phi_from: np.ndarray, phi_to: np.ndarray, out_from: np.ndarray) -> float:
    """log q(phi_to | phi_from) up to the constant, from the network output at
    phi_from (phi_from enters only through it)."""
    o = np.asarray(out_from, np.float64)
    m, ls = o[..., 0:2], o[..., 2:4]
    z = (np.asarray(phi_to, np.float64) - m) * np.exp(-ls)
    return float(np.sum(-0.5 * z * z - ls))


def propose(seed: int, phi: np.ndarray, out: np.ndarray):
    """phi' = mu + exp(lsig) xi for one chain ([L, Ns, 2] arrays); returns
    (seed after the draws, phi', log q(phi'|phi))."""
    seed, xi = gaussians(seed, phi.size)
    xi = xi.reshape(phi.shape)
    o = np.asarray(out, np.float64)
    prop = o[..., 0:2] + np.exp(o[..., 2:4]) * xi
    return seed, prop, float(np.sum(-0.5 * xi * xi - o[..., 2:4]))


def accept(seed: int, log_w: float, log_w_prop: float, hastings: float) -> tuple[int, bool]:
    """global_update.f90:237-249 with the Hastings term: accept if
    exp(log w' - log w + log q(phi|phi') - log q(phi'|phi)) >= u."""
    seed = (48828125 * seed) % 2147483648
    u = seed / 2147483648
    return seed, math.exp(log_w_prop - log_w + hastings) >= u
