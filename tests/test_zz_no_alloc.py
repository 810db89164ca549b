"""sfg_spread_forces_noalloc: the spread for callers that cannot allocate
device memory during a call (a host engine owning the memory pool, or a loop
that must not stall on cudaMalloc / cudaFree).  It reuses one fixed device
array for its scratch, so this file runs last: the checks below call it twice
in a row with different inputs (stale contents of the shared array must not
leak into the second result) and compare each result with the allocating
entry point, bit for bit, the tolerance of the other spread tests."""
import ctypes as C

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _inputs(nx, ny, rings, seed):
    rng = np.random.default_rng(seed)
    o = O.OracleSim(O.ChannelSpec(nx=nx, ny=ny), "sfo")
    for (cx, cy, r, n) in rings:
        o.add_capsule(cx, cy, r, n, O.Membrane())
    o.initialize()
    pos = o.positions()
    return o.offsets().astype(np.int32), pos, rng.normal(0.0, 1e-3, pos.shape)


def _call(name, nx, ny, off, pos, frc):
    import torch
    from softflow_b200 import _lib as L
    lib = L.lib()
    dev = torch.device("cuda:0")
    d_off = torch.tensor(off, device=dev)
    d_pos = torch.tensor(pos.ravel(), dtype=torch.float64, device=dev)
    d_frc = torch.tensor(frc.ravel(), dtype=torch.float64, device=dev)
    d_Fx = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
    d_Fy = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = getattr(lib, name)(nx, ny, len(off) - 1, d_off.data_ptr(), d_pos.data_ptr(),
                            d_frc.data_ptr(), d_Fx.data_ptr(), d_Fy.data_ptr(), int(off[-1]),
                            stream)
    L.check(rc)
    torch.cuda.synchronize()
    return d_Fx.cpu().numpy(), d_Fy.cpu().numpy()


RINGS_A = [(1.5, 20.3, 5.0, 32), (40.2, 11.7, 3.0, 24), (44.9, 17.2, 3.0, 24),
           (80.1, 30.0, 6.0, 48)]


def test_noalloc_matches_allocating_spread_twice(sfg, oracle_mod):
    """Calls in a row on the shared array: a first case, a smaller one, a
    larger one, then the first case's size again with other forces right
    after the larger call, so the tile counts and list entries the larger
    call left in the array lie inside what the last call reads."""
    cases = [
        (96, 48, RINGS_A, 11),
        (64, 32, [(30.5, 15.5, 4.0, 0), (3.0, 9.0, 3.0, 24)], 12),
        (160, 64, [(10.5, 12.3, 6.0, 48), (60.2, 40.7, 5.0, 32), (96.0, 20.0, 4.0, 0),
                   (130.3, 50.1, 3.0, 24), (158.9, 31.7, 5.0, 32)], 14),
        (96, 48, RINGS_A, 13),
    ]
    for nx, ny, rings, seed in cases:
        off, pos, frc = _inputs(nx, ny, rings, seed)
        ax, ay = _call("sfg_spread_forces", nx, ny, off, pos, frc)
        bx, by = _call("sfg_spread_forces_noalloc", nx, ny, off, pos, frc)
        assert np.array_equal(ax, bx) and np.array_equal(ay, by)
        assert np.abs(ax).max() > 0.0


def test_noalloc_rejects_oversized_calls(sfg, oracle_mod):
    from softflow_b200 import _lib as L
    lib = L.lib()
    rc = lib.sfg_spread_forces_noalloc(8192, 8192, 1, 1, 1, 1, 1, 1, 100, None)
    assert rc == 4
    assert "force tiles" in lib.sfg_last_error().decode()
    rc = lib.sfg_spread_forces_noalloc(64, 32, 1, 1, 1, 1, 1, 1, 40000, None)
    assert rc == 4
    assert "marker" in lib.sfg_last_error().decode()
