"""Learned multi-direct forcing: the per-marker network and its training.

``MDFNetwork`` owns a trainer object of the library (``sfg_mlp_*``): FP32
master parameters, Adam state and the normalisation constants; forward,
gradients and Adam steps run on the GPU's tensor cores.  Its shape and
conventions follow the reference surrogate ``SimpleNN``
(src/ml/simple_nn.cpp:10-262): 8 -> 64 -> 64 -> 2 with ReLU, He
initialisation, inputs and outputs normalised by mean and standard deviation,
mean-squared-error loss.

Inputs per marker (local frame of the membrane: tangent t, normal n):
slip = u_interp - u_target (t, n), previous-step forcing correction (t, n),
stretch, curvature, u_target (t, n).  Output: the multi-direct forcing
correction (t, n) that the plain iteration of K sweeps accumulates before its
last sweep; the step spreads it as a seed and then runs that last sweep.

Device buffers for training data are torch CUDA tensors (torch supplies
device memory and streams only).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib as L

N_IN, N_H, N_OUT = 8, 64, 2
N_PARAMS = 4866
FEATURE_NAMES = ["slip_t", "slip_n", "dFprev_t", "dFprev_n", "stretch", "curvature",
                 "utarget_t", "utarget_n"]


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def he_init(seed: int) -> np.ndarray:
    """He-normal weights, zero biases (simple_nn.cpp:19-43)."""
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0.0, np.sqrt(2.0 / N_IN), N_H * N_IN), np.zeros(N_H),
             rng.normal(0.0, np.sqrt(2.0 / N_H), N_H * N_H), np.zeros(N_H),
             rng.normal(0.0, np.sqrt(2.0 / N_H), N_OUT * N_H), np.zeros(N_OUT)]
    return np.concatenate(parts).astype(np.float32)


class MDFNetwork:
    """The per-marker network on one GPU."""

    def __init__(self, device: int = 0, seed: int = 1):
        self._lib = L.lib()
        h = C.c_void_p()
        L.check(self._lib.sfg_mlp_create(int(device), C.byref(h)))
        self._h = h
        self.device = int(device)
        self.in_mean = np.zeros(N_IN, np.float32)
        self.in_std = np.ones(N_IN, np.float32)
        self.out_mean = np.zeros(N_OUT, np.float32)
        self.out_std = np.ones(N_OUT, np.float32)
        self.set_params(he_init(seed))

    # ---- state
    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            self._lib.sfg_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != N_PARAMS:
            raise ValueError(f"expected {N_PARAMS} parameters, got {p.size}")
        L.check(self._lib.sfg_mlp_set_params(self._h, _fptr(p)))

    def params(self) -> np.ndarray:
        out = np.zeros(N_PARAMS, np.float32)
        L.check(self._lib.sfg_mlp_get_params(self._h, _fptr(out)))
        return out

    def set_normalization(self, in_mean, in_std, out_mean, out_std) -> None:
        self.in_mean = np.ascontiguousarray(in_mean, np.float32)
        self.in_std = np.ascontiguousarray(in_std, np.float32)
        self.out_mean = np.ascontiguousarray(out_mean, np.float32)
        self.out_std = np.ascontiguousarray(out_std, np.float32)
        L.check(self._lib.sfg_mlp_set_normalization(
            self._h, _fptr(self.in_mean), _fptr(self.in_std), _fptr(self.out_mean),
            _fptr(self.out_std)))

    def fit_normalization(self, X: np.ndarray, Y: np.ndarray, floor: float = 1e-12) -> None:
        """Mean / standard deviation of the training data
        (simple_nn.cpp:156-165, computeNormalization)."""
        X = np.asarray(X, np.float64)
        Y = np.asarray(Y, np.float64)
        self.set_normalization(X.mean(0), np.maximum(X.std(0), floor), Y.mean(0),
                               np.maximum(Y.std(0), floor))

    def save(self, path: str) -> None:
        np.savez(path, params=self.params(), in_mean=self.in_mean, in_std=self.in_std,
                 out_mean=self.out_mean, out_std=self.out_std)

    @classmethod
    def load(cls, path: str, device: int = 0) -> "MDFNetwork":
        d = np.load(path)
        net = cls(device)
        net.set_params(d["params"])
        net.set_normalization(d["in_mean"], d["in_std"], d["out_mean"], d["out_std"])
        return net

    # ---- compute (torch CUDA tensors or numpy arrays)
    def _dev(self, a, cols):
        import torch
        t = torch.as_tensor(a, dtype=torch.float32, device=f"cuda:{self.device}")
        t = t.reshape(-1, cols).contiguous()
        return t

    def _stream(self):
        import torch
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def forward(self, X):
        """Network outputs (de-normalised) for raw features X [n x 8]."""
        import torch
        x = self._dev(X, N_IN)
        y = torch.empty((x.shape[0], N_OUT), dtype=torch.float32, device=x.device)
        L.check(self._lib.sfg_mlp_forward(self._h, C.c_void_p(x.data_ptr()), int(x.shape[0]),
                                          C.c_void_p(y.data_ptr()), self._stream()))
        return y

    def gradients(self, X, T):
        """(gradient [4866], loss) of mean((y - t)^2) with normalised targets."""
        x = self._dev(X, N_IN)
        t = self._dev(T, N_OUT)
        g = np.zeros(N_PARAMS, np.float32)
        loss = C.c_float()
        L.check(self._lib.sfg_mlp_gradients(self._h, C.c_void_p(x.data_ptr()),
                                            C.c_void_p(t.data_ptr()), int(x.shape[0]),
                                            _fptr(g), C.byref(loss), self._stream()))
        return g, float(loss.value)

    def train(self, X, T, epochs: int = 1, batch: int = 8192, lr: float = 1e-3,
              seed: int = 0) -> np.ndarray:
        """Adam over `epochs` shuffled passes (seeded); returns batch losses."""
        import torch
        x = self._dev(X, N_IN)
        t = self._dev(T, N_OUT)
        n = x.shape[0]
        if n < batch:
            raise ValueError(f"{n} samples is fewer than one batch of {batch}")
        gen = torch.Generator(device=x.device)
        gen.manual_seed(int(seed))
        losses = []
        for _ in range(int(epochs)):
            perm = torch.randperm(n, device=x.device, generator=gen)
            xs = x[perm].contiguous()
            ts = t[perm].contiguous()
            nb = n // batch
            out = np.zeros(nb, np.float32)
            L.check(self._lib.sfg_mlp_train(self._h, C.c_void_p(xs.data_ptr()),
                                            C.c_void_p(ts.data_ptr()), int(n), int(batch),
                                            float(lr), _fptr(out), self._stream()))
            losses.append(out)
        return np.concatenate(losses) if losses else np.zeros(0, np.float32)

    def steps(self) -> int:
        s = C.c_int()
        L.check(self._lib.sfg_mlp_step_count(self._h, C.byref(s)))
        return int(s.value)


# --------------------------------------------------------------- training data

def harvest(ens, records: int = 1, every: int = 1, warmup: int = 0, at=None):
    """Runs an initialized ensemble with the plain forcing sweeps and returns
    (features, labels) of all valid markers: at the given step numbers `at`
    (1-based, increasing), or at `records` steps spaced by `every` after
    `warmup` steps."""
    ens.setLearnedMDF(None)
    if at is None:
        at = [warmup + every * (i + 1) for i in range(int(records))]
    ens.setHarvest(False)
    feats, labs = [], []
    done = 0
    try:
        for s_at in at:
            if s_at - 1 > done:
                ens.run(s_at - 1 - done)
            ens.setHarvest(True)
            ens.run(1)
            done = s_at
            f, l, v = ens.harvest()
            v &= np.isfinite(f).all(1) & np.isfinite(l).all(1)
            feats.append(f[v])
            labs.append(l[v])
            ens.setHarvest(False)
    finally:
        ens.setHarvest(False)
    return np.concatenate(feats), np.concatenate(labs)


def _geometric_steps(first: int, last: int, n: int):
    """n distinct step numbers from first to last, spaced geometrically."""
    v = np.unique(np.round(np.geomspace(first, last, n)).astype(int))
    while len(v) < n:
        v = np.unique(np.concatenate([v, v[-1:] + np.arange(1, n - len(v) + 1)]))
    return [int(x) for x in v[:n]]


def training_set(samples: int = 2_000_000, device: int = 0, precision: str = "fp32",
                 c1_fraction: float = 0.1):
    """Training data from plain runs of the single 400 x 80 channel with 30
    capsules and of the 256-channel ensemble (synthetic, seeded placement):
    records at steps spaced geometrically from the first step (the start-up
    transient) to step 4000 (single channel) or 1500 (ensemble; beyond that
    a few of its channels approach the divergence the plain method shows
    there).  Returns (X, Y) with at most `samples` rows."""
    from . import workloads as W
    c1 = W.build(W.plan_c1(precision), precision, device)
    rec1 = max(1, int(samples * c1_fraction) // max(c1.num_markers(), 1))
    X1, Y1 = harvest(c1, at=_geometric_steps(1, 4000, rec1))
    c1.close()
    c3 = W.build(W.plan_c3(precision), precision, device)
    rec3 = max(1, int(np.ceil((samples - X1.shape[0]) / max(c3.num_markers(), 1))))
    X3, Y3 = harvest(c3, at=_geometric_steps(1, 1500, rec3))
    c3.close()
    X = np.concatenate([X1, X3])[:samples]
    Y = np.concatenate([Y1, Y3])[:samples]
    return X, Y


# inputs that change sign with the slip field (slip and previous correction)
ODD_INPUTS = (0, 1, 2, 3)


def mirror(X, Y=None):
    """P x: the inputs with the slip and the previous correction negated (and
    -y for the labels).  The step evaluates the odd part (N(x) - N(Px)) / 2."""
    Xm = np.array(X, dtype=np.float32, copy=True)
    Xm[:, list(ODD_INPUTS)] *= -1.0
    return Xm if Y is None else (Xm, -np.asarray(Y, dtype=np.float32))


def predict(net: "MDFNetwork", X) -> np.ndarray:
    """The step's predictor on host data: (N(x) - N(Px)) / 2."""
    a = net.forward(X).cpu().numpy()
    b = net.forward(mirror(X)).cpu().numpy()
    return 0.5 * (a - b)


def train_network(X, Y, device: int = 0, epochs: int = 8, batch: int = 8192, lr: float = 1e-3,
                  seed: int = 1):
    """Trains a fresh network with Adam on the tensor cores on the samples and
    their mirror images (P x, -y), so that the network is close to odd and
    its odd part, which the step evaluates, keeps what it learned; fits the
    normalisation to the mirrored set.  Returns (network, batch losses)."""
    Xm, Ym = mirror(X, Y)
    XA = np.concatenate([np.asarray(X, np.float32), Xm])
    YA = np.concatenate([np.asarray(Y, np.float32), Ym])
    net = MDFNetwork(device, seed=seed)
    net.fit_normalization(XA, YA)
    losses = net.train(XA, YA, epochs=epochs, batch=batch, lr=lr, seed=seed)
    return net, losses
