"""The proposer oracle (oracle/proposer.py) checked against itself on the CPU:
finite differences of its float64 network pin the backward pass, the
transposed convolution is the adjoint of the convolution, and the proposal's
log q agrees with the density it draws from."""
import math

import numpy as np

from oracle import proposer as P


def _small(width=4, Lx=3, Ly=2, L=4, B=2, seed=0):
    rng = np.random.default_rng(seed)
    # a last layer as large as the others, so every output depends on every layer
    params = P.init_params(width, seed=seed, last_scale=1.0)
    layers = P.unpack(params, width)
    for _, b in layers:
        b[...] = rng.normal(0, 0.1, size=b.shape)
    phi = rng.normal(size=(B, L, Lx * Ly, 2))
    target = phi + rng.normal(scale=0.7, size=phi.shape)
    return params.astype(np.float64), phi, target, (Lx, Ly, width)


def test_zero_last_layer_is_the_prior_independence_sampler():
    """mu = 0, lsig = 0: q(phi'|phi) = N(0, 1) whatever phi, and the Gaussian
    part of the weight cancels the Hastings term exactly."""
    rng = np.random.default_rng(2)
    params = P.init_params(8, seed=4)
    phi = rng.normal(size=(1, 4, 6, 2))
    out = P.forward(params, phi, 3, 2, width=8)
    assert np.all(out == 0.0)
    seed, prop, lqf = P.propose(99, phi[0], out[0])
    lqr = P.log_q(prop, phi[0], out[0])
    log_prior_ratio = -0.5 * np.sum(prop ** 2) + 0.5 * np.sum(phi[0] ** 2)
    assert abs(log_prior_ratio + lqr - lqf) < 1e-9


def test_tap_order():
    assert P.TAPS[0] == (-1, -1, -1)
    assert P.TAPS[13] == (0, 0, 0)
    assert P.TAPS[1] == (0, -1, -1)
    assert P.TAPS[3] == (-1, -1, 0)
    assert len(set(P.TAPS)) == 27


def test_transpose_is_adjoint():
    rng = np.random.default_rng(3)
    x = rng.normal(size=(2, 4, 3, 5, 3))
    g = rng.normal(size=(2, 4, 3, 5, 6))
    W = rng.normal(size=(27, 6, 3))
    lhs = np.sum(P.conv(x, W, np.zeros(6)) * g)
    rhs = np.sum(x * P.conv_transpose(g, W))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)
    # the weight gradient: d<conv(x, W), g>/dW
    dW = P.conv_wgrad(x, g)
    k, o, i = 17, 4, 2
    E = np.zeros_like(W)
    E[k, o, i] = 1.0
    assert abs(np.sum(P.conv(x, E, np.zeros(6)) * g) - dW[k, o, i]) < 1e-10


def test_gradient_matches_finite_differences():
    params, phi, target, (Lx, Ly, w) = _small()
    loss, grad = P.loss_and_grad(params, phi, target, Lx, Ly, w, rounding=False)
    rng = np.random.default_rng(7)
    idx = rng.choice(params.size, size=60, replace=False)
    h = 1e-6
    for j in idx:
        pp, pm = params.copy(), params.copy()
        pp[j] += h
        pm[j] -= h
        lp, _ = P.loss_and_grad(pp, phi, target, Lx, Ly, w, rounding=False)
        lm, _ = P.loss_and_grad(pm, phi, target, Lx, Ly, w, rounding=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - grad[j]) <= 1e-6 * max(1.0, abs(fd)), (j, fd, grad[j])


def test_rounded_network_tracks_float64():
    params, phi, target, (Lx, Ly, w) = _small(width=8)
    o64 = P.forward(params, phi, Lx, Ly, w, rounding=False)
    o16 = P.forward(params, phi, Lx, Ly, w, rounding=True)
    assert np.max(np.abs(o64 - o16)) <= 0.05 * np.max(np.abs(o64))
    _, g64 = P.loss_and_grad(params, phi, target, Lx, Ly, w, rounding=False)
    _, g16 = P.loss_and_grad(params, phi, target, Lx, Ly, w, rounding=True)
    assert np.linalg.norm(g64 - g16) <= 0.05 * np.linalg.norm(g64)


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -3.14159, 1e-30], dtype=np.float32)
    r = P.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0          # tie to even
    assert r[2] == np.float32(1.0 + 2 ** -7)     # tie to even (upwards)
    assert abs(r[3] + 3.140625) < 1e-7
    assert np.all(r.view(np.uint32) & 0xFFFF == 0)


def test_proposal_log_q_and_draws():
    rng = np.random.default_rng(5)
    phi = rng.normal(size=(4, 6, 2))
    out = rng.normal(scale=0.3, size=(4, 6, 4))
    seed, prop, lq = P.propose(12345, phi, out)
    assert abs(lq - P.log_q(phi, prop, out)) < 1e-9
    s2, xi = P.gaussians(12345, phi.size)
    assert s2 == seed
    s = 12345
    for _ in range(2 * phi.size):
        s = (48828125 * s) % 2147483648
    assert s == seed
    np.testing.assert_allclose(prop, out[..., :2] + np.exp(out[..., 2:]) * xi.reshape(phi.shape))
    # the accept rule: exp(x) >= u with u the chain's next draw
    s3, acc = P.accept(seed, 0.0, -1.0, 0.5)
    u = s3 / 2147483648
    assert acc == (math.exp(-0.5) >= u)
