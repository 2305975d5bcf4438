"""The scheduler network: the CPU oracle is pinned by finite differences; the
GPU forward/backward kernels match the oracle; training lowers the loss."""
import numpy as np
import pytest

import scaph_b200 as S
from oracle import mlp_oracle as M


def _problem(n=96, n_in=40, n_out=9, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, n_in)).astype(np.float32)
    T = (rng.random((n, n_out)) < 0.4).astype(np.float32)
    W = rng.uniform(0.2, 1.0, size=(n, n_out)).astype(np.float32) / n
    p = (rng.normal(size=M.num_params(n_in, n_out)) * 0.2).astype(np.float32)
    return X, T, W, p, n_in, n_out


def test_oracle_gradient_matches_finite_differences():
    X, T, W, p, n_in, n_out = _problem(n=8, n_in=6, n_out=3)
    p64 = p.astype(np.float64)
    _, g = M.loss_grad(p64, X, T, W, n_in, n_out, rnd=False, dtype=np.float64)
    rng = np.random.default_rng(1)
    for i in rng.choice(p.size, 40, replace=False):
        e = np.zeros_like(p64)
        e[i] = 1e-6
        lp, _ = M.loss_grad(p64 + e, X, T, W, n_in, n_out, rnd=False, dtype=np.float64)
        lm, _ = M.loss_grad(p64 - e, X, T, W, n_in, n_out, rnd=False, dtype=np.float64)
        assert abs((lp - lm) / 2e-6 - g[i]) < 1e-6 + 1e-5 * abs(g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e38], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie 1 + 2^-8 rounds to even (1.0)
    assert r[2] == np.float32(1.0078125) and r[3] == -2.5


@pytest.mark.gpu
def test_gpu_forward_and_gradients_match_oracle():
    """Tolerance: bf16 operands are identical on both sides; only the float32
    accumulation order differs (rtol 2e-3 on outputs, 1e-2 on gradients)."""
    X, T, W, p, n_in, n_out = _problem(n=200, n_in=80, n_out=33)
    net = S.Mlp(n_in, n_out, seed=3)
    net.set_params(p)
    pb = M.bf16(p)  # the network stores bf16 weights
    assert np.array_equal(net.params(), pb)
    _, _, Yr = M.forward(pb, X, n_in, n_out)
    Y = net.forward(X)
    np.testing.assert_allclose(Y, Yr, rtol=2e-3, atol=2e-3)
    loss_r, g_r = M.loss_grad(pb, X, T, W, n_in, n_out)
    loss, g = net.loss_grad(X, T, W)
    assert abs(loss - loss_r) < 1e-3 * max(1.0, abs(loss_r))
    scale = np.abs(g_r).max()
    np.testing.assert_allclose(g, g_r, rtol=1e-2, atol=1e-2 * scale)


@pytest.mark.gpu
def test_gpu_training_fits_a_separable_task(tmp_path):
    rng = np.random.default_rng(4)
    n, n_in, n_out = 512, 24, 5
    X = rng.normal(size=(n, n_in)).astype(np.float32)
    Wtrue = rng.normal(size=(n_in, n_out))
    T = (X @ Wtrue > 0).astype(np.float32)
    Wt = np.full((n, n_out), 1.0 / n, np.float32)
    net = S.Mlp(n_in, n_out, seed=5)
    l0, _ = net.loss_grad(X, T, Wt)
    l1 = net.train(X, T, Wt, epochs=60, batch=128, lr=3e-3)
    acc = ((net.forward(X) > 0) == (T > 0.5)).mean()
    assert l1 < 0.5 * l0 and acc > 0.9
    # checkpoint round trip
    path = str(tmp_path / "net.bin")
    net.save(path)
    other = S.Mlp(n_in, n_out, seed=9)
    other.load(path)
    assert np.array_equal(other.params(), net.params())


@pytest.mark.gpu
def test_device_timing_leaves_the_network_unchanged():
    """scaph_mlp_time reports CUDA-event times of a forward pass, a training
    step and the single-row inference kernel, and restores the parameters."""
    net = S.Mlp(16 + 40, 41, seed=9)
    p0 = net.params().copy()
    t = net.time(n=128, reps=5)
    assert t["forward_us"] > 0 and t["train_step_us"] > t["forward_us"] and t["infer1_us"] > 0
    assert np.array_equal(net.params(), p0)
