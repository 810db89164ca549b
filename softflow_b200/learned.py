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
stretch, curvature, u_target (t, n).  Output: the total multi-direct forcing
correction of the step (t, n), i.e. the sum of the correction sweeps.

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
