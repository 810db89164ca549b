"""CPU checker of the learned multi-direct-forcing network (test
infrastructure only: imported by tests/ and nothing else).

The network is the per-marker MLP 8 -> 64 -> 64 -> 2 with ReLU, the shape of
the reference's surrogate `SimpleNN` (src/ml/simple_nn.cpp:45-79, forward;
:151-262, mean-squared-error backpropagation with the gradient
2 (out - y) / n_out per sample, averaged over the batch; He initialisation
:19-43; inputs and outputs normalised by mean and standard deviation
:156-165).  The reference trains it in FP64 with plain SGD; the GPU trains it
with BF16 operands, FP32 accumulation and Adam.

Two restatements:

* ``forward_q`` / ``gradients_q`` follow the GPU's rounding points: inputs,
  weights, hidden activations and the back-propagated errors are rounded to
  BF16 (round to nearest even) where the GPU rounds them, products are
  accumulated in FP64 here and rounded to FP32 (the tensor cores accumulate
  in FP32 in another order, so results agree to FP32 rounding, and hidden
  activations can differ by one BF16 step where a sum lies on a rounding
  boundary);
* ``forward_exact`` / ``gradients_exact`` are the same formulas in FP64 with
  no rounding, checked against finite differences.

``features`` restates the per-marker input features computed on the GPU.

Parameter vector layout (4866 FP32 values): W1 [64 x 8], b1 [64],
W2 [64 x 64], b2 [64], W3 [2 x 64], b3 [2].
"""
from __future__ import annotations

import numpy as np

N_IN, N_H, N_OUT = 8, 64, 2
N_PARAMS = N_H * N_IN + N_H + N_H * N_H + N_H + N_OUT * N_H + N_OUT   # 4866


def bf16(x):
    """Round FP32 values to BF16 (nearest even), returned as float32."""
    u = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) & 0xFFFF0000).astype(np.uint32).view(np.float32)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    out = []
    for shape in ((N_H, N_IN), (N_H,), (N_H, N_H), (N_H,), (N_OUT, N_H), (N_OUT,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    return out


def pack(W1, b1, W2, b2, W3, b3):
    return np.concatenate([np.ravel(a) for a in (W1, b1, W2, b2, W3, b3)]).astype(np.float32)


def he_init(seed):
    """He initialisation with zero biases (simple_nn.cpp:19-43)."""
    rng = np.random.default_rng(seed)
    W1 = rng.normal(0.0, np.sqrt(2.0 / N_IN), (N_H, N_IN))
    W2 = rng.normal(0.0, np.sqrt(2.0 / N_H), (N_H, N_H))
    W3 = rng.normal(0.0, np.sqrt(2.0 / N_H), (N_OUT, N_H))
    return pack(W1, np.zeros(N_H), W2, np.zeros(N_H), W3, np.zeros(N_OUT))


def _f32(x):
    return np.asarray(x, dtype=np.float64).astype(np.float32).astype(np.float64)


# ---------------------------------------------------------------- exact (FP64)

def forward_exact(p, X):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    Z1 = X @ W1.T + b1
    H1 = np.maximum(Z1, 0.0)
    Z2 = H1 @ W2.T + b2
    H2 = np.maximum(Z2, 0.0)
    return H2 @ W3.T + b3, (H1, H2)


def loss_exact(p, X, T):
    Y, _ = forward_exact(p, X)
    return float(np.mean((Y - T) ** 2))


def gradients_exact(p, X, T):
    """d loss / d p for loss = mean over samples and outputs of (y - t)^2."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    B = X.shape[0]
    Y, (H1, H2) = forward_exact(p, X)
    dY = 2.0 * (Y - T) / N_OUT / B
    dW3 = dY.T @ H2
    db3 = dY.sum(0)
    dZ2 = (dY @ W3) * (H2 > 0)
    dW2 = dZ2.T @ H1
    db2 = dZ2.sum(0)
    dZ1 = (dZ2 @ W2) * (H1 > 0)
    dW1 = dZ1.T @ X
    db1 = dZ1.sum(0)
    return pack(dW1, db1, dW2, db2, dW3, db3).astype(np.float64)


# ------------------------------------------------------- GPU rounding points

def forward_q(p, X):
    """Forward pass with the GPU's BF16 rounding points.  Returns Y (FP32)
    and the BF16 activations (H1, H2) the backward pass reuses."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    Xq = bf16(X).astype(np.float64)
    # layer 1 carries its bias as a ninth input fixed at 1 (BF16 bias)
    Z1 = _f32(Xq @ bf16(W1).astype(np.float64).T + bf16(b1).astype(np.float64))
    H1 = bf16(np.maximum(Z1, 0.0)).astype(np.float64)
    Z2 = _f32(_f32(H1 @ bf16(W2).astype(np.float64).T) + _f32(b2))
    H2 = bf16(np.maximum(Z2, 0.0)).astype(np.float64)
    Y = _f32(_f32(H2 @ bf16(W3).astype(np.float64).T) + _f32(b3))
    return Y, (Xq, H1, H2)


def gradients_q(p, X, T):
    """Gradients as the GPU forms them (BF16 operands, FP32 sums)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    B = np.asarray(X).shape[0]
    Y, (Xq, H1, H2) = forward_q(p, X)
    dY = _f32((Y - _f32(T)) * np.float32(1.0 / B))   # 2 (y - t) / 2 / B
    dW3 = _f32(dY.T @ H2)
    db3 = _f32(dY.sum(0))
    dYq = bf16(dY).astype(np.float64)
    dZ2 = bf16(_f32(dYq @ bf16(W3).astype(np.float64)) * (H2 > 0)).astype(np.float64)
    dW2 = _f32(dZ2.T @ H1)
    db2 = _f32(dZ2.sum(0))
    dZ1 = bf16(_f32(dZ2 @ bf16(W2).astype(np.float64)) * (H1 > 0)).astype(np.float64)
    dW1 = _f32(dZ1.T @ Xq)
    db1 = _f32(dZ1.sum(0))
    return pack(dW1, db1, dW2, db2, dW3, db3).astype(np.float64)


def adam(p, g, m, v, t, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam update in FP32 (Kingma and Ba, 2015, Algorithm 1)."""
    p = np.asarray(p, np.float32).copy()
    g = np.asarray(g, np.float32)
    m = (np.float32(beta1) * m + np.float32(1 - beta1) * g).astype(np.float32)
    v = (np.float32(beta2) * v + np.float32(1 - beta2) * g * g).astype(np.float32)
    mh = m / np.float32(1 - beta1 ** t)
    vh = v / np.float32(1 - beta2 ** t)
    p -= np.float32(lr) * mh / (np.sqrt(vh) + np.float32(eps))
    return p, m, v


# ------------------------------------------------------------------ features

def features(pos, nxt, prv, rest_prev, rest_next, u_interp, u_target, dF_prev, Lx):
    """Per-marker network inputs in the marker's local frame.

    pos, nxt, prv : (M, 2) positions of the marker and its ring neighbours;
    rest_prev, rest_next : rest lengths of the edges (k-1, k) and (k, k+1);
    u_interp : velocity interpolated after the membrane-force spread;
    u_target : the marker's velocity from the previous step (the multi-direct
               forcing target, immersed_boundary.cpp:255);
    dF_prev  : the marker's forcing correction of the previous step before
               its last sweep.

    Tangent t = normalised (e_prev + e_next), normal n = (-t_y, t_x);
    features = [slip.t, slip.n, dF_prev.t, dF_prev.n, stretch, curvature,
    u_target.t, u_target.n] with slip = u_interp - u_target,
    stretch = (|e_prev| + |e_next|) / (rest_prev + rest_next) - 1 and
    curvature = atan2(e_prev x e_next, e_prev . e_next) / (0.5 (|e_prev| + |e_next|)).
    Returns (features (M, 8), t (M, 2), n (M, 2)).
    """
    def mimg(d):
        d = d.copy()
        d[:, 0] -= Lx * np.round(d[:, 0] / Lx)
        return d
    ep = mimg(pos - prv)
    en = mimg(nxt - pos)
    tv = ep + en
    tl = np.hypot(tv[:, 0], tv[:, 1])
    tl = np.where(tl > 0, tl, 1.0)
    t = tv / tl[:, None]
    n = np.stack([-t[:, 1], t[:, 0]], 1)
    lp = np.hypot(ep[:, 0], ep[:, 1])
    ln = np.hypot(en[:, 0], en[:, 1])
    stretch = (lp + ln) / (rest_prev + rest_next) - 1.0
    cross = ep[:, 0] * en[:, 1] - ep[:, 1] * en[:, 0]
    dot = ep[:, 0] * en[:, 0] + ep[:, 1] * en[:, 1]
    curv = np.arctan2(cross, dot) / (0.5 * (lp + ln))
    slip = u_interp - u_target
    dot2 = lambda a, b: a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1]
    F = np.stack([dot2(slip, t), dot2(slip, n), dot2(dF_prev, t), dot2(dF_prev, n),
                  stretch, curv, dot2(u_target, t), dot2(u_target, n)], 1)
    return F, t, n
