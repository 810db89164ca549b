"""Standalone deterministic spread (sfg_spread_forces) against the oracle,
and the momentum-conservation checks of the reference's
tests/verification/test_ibm_momentum_conservation.cpp (relative residual of
sum F - sum_k f_k ds_k below 1e-12)."""
import ctypes as C

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _ring_system(nx, ny, rings, force_fn, periodic=True):
    """Oracle channel holding the given rings (cx, cy, r, n); markers get
    forces from force_fn(positions) -> [M][2]."""
    o = O.OracleSim(O.ChannelSpec(nx=nx, ny=ny), "sfo")
    for (cx, cy, r, n) in rings:
        o.add_capsule(cx, cy, r, n, O.Membrane())
    o.initialize()
    pos = o.positions()
    frc = np.asarray(force_fn(pos), dtype=np.float64)
    o.set_markers(force=frc)
    return o, pos, frc


def _gpu_spread(nx, ny, offsets, pos, frc, F0=None):
    import torch
    from softflow_b200 import _lib as L
    lib = L.lib()
    dev = torch.device("cuda:0")
    d_off = torch.tensor(np.asarray(offsets, dtype=np.int32), device=dev)
    d_pos = torch.tensor(pos.ravel(), dtype=torch.float64, device=dev)
    d_frc = torch.tensor(frc.ravel(), dtype=torch.float64, device=dev)
    if F0 is None:
        d_Fx = torch.zeros(ny * nx, dtype=torch.float64, device=dev)
        d_Fy = torch.zeros(ny * nx, dtype=torch.float64, device=dev)
    else:
        d_Fx = torch.tensor(F0[0].ravel(), dtype=torch.float64, device=dev)
        d_Fy = torch.tensor(F0[1].ravel(), dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    L.check(lib.sfg_spread_forces(nx, ny, len(offsets) - 1, d_off.data_ptr(), d_pos.data_ptr(), d_frc.data_ptr(),
               d_Fx.data_ptr(), d_Fy.data_ptr(), int(offsets[-1]), C.c_void_p(s)))
    torch.cuda.synchronize()
    return d_Fx.cpu().numpy().reshape(ny, nx), d_Fy.cpu().numpy().reshape(ny, nx)


def test_spread_bit_exact_with_oracle(sfg, oracle_mod):
    rng = np.random.default_rng(3)
    rings = [(1.5, 20.3, 5.0, 32), (40.2, 11.7, 3.0, 24), (44.9, 17.2, 3.0, 24),
             (62.1, 28.0, 6.0, 48), (20.0, 2.5, 3.0, 24)]
    o, pos, frc = _ring_system(64, 32, rings, lambda p: rng.normal(0, 1e-3, p.shape))
    Fx, Fy = o.spread()
    gx, gy = _gpu_spread(64, 32, o.offsets(), pos, frc)
    assert np.array_equal(gx, Fx) and np.array_equal(gy, Fy)


def test_spread_adds_to_existing_field(sfg, oracle_mod):
    rng = np.random.default_rng(5)
    o, pos, frc = _ring_system(48, 24, [(20.5, 12.2, 4.0, 0)], lambda p: rng.normal(0, 1, p.shape))
    Fx, Fy = o.spread()
    F0 = (rng.normal(0, 1, (24, 48)), rng.normal(0, 1, (24, 48)))
    gx, gy = _gpu_spread(48, 24, o.offsets(), pos, frc, F0)
    np.testing.assert_array_equal(gx, F0[0] + Fx)
    np.testing.assert_array_equal(gy, F0[1] + Fy)


def _residual(F, pos, frc_per_node, nx):
    # sum_k f ds_k with minimum-image arc lengths
    P = pos.reshape(-1, 2)
    n = len(P)
    ds = np.zeros(n)
    for k in range(n):
        a, b = P[k] - P[k - 1], P[(k + 1) % n] - P[k]
        for d in (a, b):
            if d[0] > 0.5 * nx:
                d[0] -= nx
            if d[0] < -0.5 * nx:
                d[0] += nx
        ds[k] = 0.5 * (np.hypot(*a) + np.hypot(*b))
    ex = frc_per_node[0] * ds.sum()
    ey = frc_per_node[1] * ds.sum()
    got_x, got_y = F[0].sum(), F[1].sum()
    return (abs(got_x - ex) + abs(got_y - ey)) / (abs(ex) + abs(ey))


@pytest.mark.parametrize("nx,ny,center,R,Nn,f", [
    (128, 64, (64.0, 32.0), 12.0, 64, (0.001, -0.0007)),
    (256, 128, (128.0, 64.0), 16.0, 32, (0.002, 0.001)),
    (256, 128, (128.0, 64.0), 16.0, 256, (0.002, 0.001)),
    (64, 64, (2.0, 32.0), 5.0, 48, (0.0015, 0.0005)),   # straddles the seam
])
def test_spread_momentum_conservation(sfg, oracle_mod, nx, ny, center, R, Nn, f):
    o, pos, frc = _ring_system(nx, ny, [(center[0], center[1], R, Nn)],
                               lambda p: np.tile(np.array(f), (len(p), 1)))
    F = _gpu_spread(nx, ny, o.offsets(), pos, frc)
    assert _residual(F, pos, f, nx) < 1e-12
