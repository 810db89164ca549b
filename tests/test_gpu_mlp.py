"""The learned-MDF network on the tensor cores against the CPU oracle
(oracle/mlp.py): forward outputs, gradients (the oracle follows the GPU's
BF16 rounding points; the exact FP64 gradients bound the BF16 effect), Adam
updates and deterministic training."""
import numpy as np
import pytest

from oracle import mlp as Q

pytestmark = pytest.mark.gpu


def _net(seed=3):
    from softflow_b200.learned import MDFNetwork
    net = MDFNetwork(0, seed=seed)
    return net


def _data(n, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.normal(0, 1, (n, 8)).astype(np.float32)
    T = np.stack([np.tanh(X[:, 0] - 0.5 * X[:, 1]) + 0.1 * X[:, 4],
                  X[:, 2] * X[:, 3] * 0.3 - X[:, 7]], 1).astype(np.float32)
    return X, T


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def test_forward_matches_oracle(sfg):
    net = _net()
    p = net.params()
    X, _ = _data(1000)      # not a multiple of 128: ragged last tile
    y = net.forward(X).cpu().numpy()
    yq, _ = Q.forward_q(p, X)
    ye, _ = Q.forward_exact(p, X)
    assert rel(y, yq) < 5e-3
    assert rel(y, ye) < 3e-2


def test_forward_normalisation(sfg):
    net = _net()
    rng = np.random.default_rng(1)
    im, isd = rng.normal(0, 1, 8), rng.uniform(0.5, 2.0, 8)
    om, osd = rng.normal(0, 1, 2), rng.uniform(0.5, 2.0, 2)
    net.set_normalization(im, isd, om, osd)
    X, _ = _data(300, 2)
    y = net.forward(X).cpu().numpy()
    Xn = ((X - im.astype(np.float32)) / isd.astype(np.float32)).astype(np.float32)
    yq, _ = Q.forward_q(net.params(), Xn)
    assert rel(y, yq * osd + om) < 5e-3


@pytest.mark.parametrize("n", [128, 1000, 8192])
def test_gradients_match_oracle(sfg, n):
    net = _net()
    p = net.params()
    X, T = _data(n, 4)
    g, loss = net.gradients(X, T)
    gq = Q.gradients_q(p, X, T)
    ge = Q.gradients_exact(p, X, T)
    assert rel(g, gq) < 2e-2, "vs BF16-rounding oracle"
    assert rel(g, ge) < 6e-2, "vs exact FP64"
    assert abs(loss - Q.loss_exact(p, X, T)) / Q.loss_exact(p, X, T) < 2e-2
    # every block of the parameter vector carries gradient
    W1, b1, W2, b2, W3, b3 = Q.unpack(g)
    for blk in (W1, b1, W2, b2, W3, b3):
        assert np.linalg.norm(blk) > 0


def test_adam_step_matches_oracle(sfg):
    net = _net()
    p0 = net.params()
    X, T = _data(8192, 5)
    g, _ = net.gradients(X, T)
    net.train(X, T, epochs=1, batch=8192, lr=1e-3, seed=0)   # one step, whole batch
    p1 = net.params()
    # the shuffled batch is the same set, so the gradient is the same sum
    pe, _, _ = Q.adam(p0, g, np.zeros_like(p0), np.zeros_like(p0), 1, lr=1e-3)
    assert np.max(np.abs(p1 - pe)) < 2e-5
    assert net.steps() == 1


def test_training_reduces_loss_and_is_deterministic(sfg):
    X, T = _data(65536, 6)
    a, b = _net(7), _net(7)
    la = a.train(X, T, epochs=3, batch=8192, lr=1e-3, seed=11)
    lb = b.train(X, T, epochs=3, batch=8192, lr=1e-3, seed=11)
    assert np.array_equal(la, lb)
    assert np.array_equal(a.params(), b.params())
    assert la[-1] < 0.5 * la[0]
    # the trained network generalises to fresh samples of the same law
    Xv, Tv = _data(4096, 8)
    yv = a.forward(Xv).cpu().numpy()
    assert np.mean((yv - Tv) ** 2) < 0.5 * np.mean((Q.forward_exact(Q.he_init(7), Xv)[0] - Tv) ** 2)
