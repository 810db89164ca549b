"""Fluid boundaries beyond the periodic channel with resting walls, on the
GPU against the oracle (oracle/sfo.c, pinned bit for bit to the reference's
LBMSolver in tests/test_oracle_golden.py) and against the reference's own
outputs (tests/golden):

* Zou-He velocity inlet (parabolic profile) / pressure outlet channels, the
  reference's default BoundaryType::INLET_OUTLET (zou_he_boundary.cpp);
* closed boxes (SOLID columns) with a moving lid (moving_wall.cpp);
* plane Couette flow with a capsule (periodic x, walls moving apart);
* FP64 bit for bit; FP32 / FP16S within the precision tolerances of the
  other parity tests; steady Couette flow against the linear profile.
"""
import os

import numpy as np
import pytest

from cases import CASES, build_gpu, build_oracle, gpu_params, rel_l2

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

BOUNDARY = [("zouhe_bgk", 300), ("zouhe_mrt", 300), ("zouhe_reg", 300), ("cavity", 400),
            ("shear_capsule", 60), ("pillars_bb", 300), ("pillars_ibb", 300),
            ("pillars_zouhe", 300)]


def _open_mask(case, o=None):
    """Non-SOLID cells (CellType as LBMSolver::initialize sets it); with
    pillars, the cells where the oracle's density is not zeroed."""
    if case.get("pillars"):
        return o.rho() != 0.0
    sp = case["spec"]
    nx, ny = sp["nx"], sp["ny"]
    m = np.ones((ny, nx), dtype=bool)
    if not sp.get("periodic_y"):
        m[0, :] = m[ny - 1, :] = False
    if sp.get("boundary_type") == 2:
        m[:, 0] = m[:, nx - 1] = False
        if sp.get("periodic_y"):
            m[0, :] = m[ny - 1, :] = True
    return m


@pytest.mark.parametrize("name,steps", BOUNDARY)
def test_fp64_boundaries_bit_exact(sfg, oracle_mod, name, steps):
    case = CASES[name]
    o = build_oracle(case)
    o.step(steps)
    sim = build_gpu(case, "fp64")
    sim.run(steps)
    fld = sim.field()
    m = _open_mask(case, o)
    f = fld.distributions()
    assert np.array_equal(f[:, m], o.f()[:, m])
    rho, ux, uy, _, _ = fld.macroscopic()
    assert np.array_equal(rho, o.rho()) and np.array_equal(ux, o.ux())
    assert np.array_equal(uy, o.uy())
    if case["capsules"]:
        assert np.array_equal(sim.capsules().positions(), o.positions())
    assert sim.lastCappedNodes() == o.last_capped()
    assert np.abs(ux).max() > 1e-3          # the boundaries drive a flow


@pytest.mark.parametrize("name", ["zouhe_bgk", "zouhe_reg", "cavity", "shear_capsule",
                                  "pillars_ibb", "pillars_zouhe"])
def test_fp64_boundaries_match_reference_golden(sfg, name):
    """Against the reference's own outputs (tests/golden/make_golden.py)."""
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    case = CASES[name]
    sim = build_gpu(case, "fp64")
    sim.run(int(g["steps"]))
    fld = sim.field()
    assert np.array_equal(fld.velocity_x(), g["ux"]) and np.array_equal(fld.velocity_y(), g["uy"])
    assert np.array_equal(fld.density(), g["rho"])
    if "pos" in g:
        assert np.array_equal(sim.capsules().positions(), g["pos"])


@pytest.mark.parametrize("precision,tol", [("fp32", 1e-4), ("fp16s", 1e-3)])
@pytest.mark.parametrize("name,steps", [("zouhe_bgk", 300), ("zouhe_mrt", 300),
                                        ("cavity", 400), ("shear_capsule", 60),
                                        ("pillars_ibb", 300)])
def test_reduced_precision_boundaries(sfg, oracle_mod, precision, tol, name, steps):
    case = CASES[name]
    o = build_oracle(case)
    o.step(steps)
    sim = build_gpu(case, precision)
    sim.run(steps)
    fld = sim.field()
    m = _open_mask(case, o)
    ex = rel_l2(fld.velocity_x()[m], o.ux()[m])
    ey = rel_l2(fld.velocity_y()[m], o.uy()[m])
    print(f"{name} {precision}: rel L2 ux {ex:.3e}, uy {ey:.3e}")
    assert ex < tol and ey < 10 * tol


def test_couette_steady_profile(sfg):
    """Plane Couette flow between halfway walls at y = 0.5 and ny - 1.5
    moving at -U and +U: the steady profile is linear."""
    import softflow_b200 as S
    case = dict(CASES["shear_capsule"])
    case = dict(case, capsules=[])
    p = gpu_params(case, "fp64")
    p.nx, p.ny = 8, 34
    sim = S.Simulation(p)
    sim.initialize()
    nu = (p.fluid.tau - 0.5) / 3.0
    H = p.ny - 2
    sim.run(int(6.0 * H * H / nu))
    ux = sim.field().velocity_x()[1:p.ny - 1, 4]
    y = np.arange(1, p.ny - 1)
    Ub, Ut = p.fluid.bottom_wall_velocity, p.fluid.top_wall_velocity
    ua = Ub + (Ut - Ub) * (y - 0.5) / H
    err = float(np.abs(ux - ua).max() / abs(Ut - Ub))
    print(f"Couette: max |u - u_linear| / dU = {err:.3e}")
    assert err < 1e-6


def test_boundary_channel_restrictions(sfg):
    import softflow_b200 as S
    p = gpu_params(CASES["zouhe_bgk"], "fp32")
    sim = S.Simulation(p)
    sim.addCapsule((30.0, 10.0), 3.0, 24)
    with pytest.raises(S.SoftFlowGpuError, match="periodic in x"):
        sim.initialize()
    q = gpu_params(CASES["cavity"], "fp32")
    q.scalar.enabled = True
    with pytest.raises(S.SoftFlowGpuError, match="scalar"):
        S.Simulation(q).initialize()


def test_body_force_on_fluid_cells_only(sfg, oracle_mod):
    """The body force (and its cap) reaches FLUID cells only: the INLET /
    OUTLET columns get none (simulation.cpp:556-560)."""
    case = dict(CASES["zouhe_bgk"])
    case["spec"] = dict(case["spec"], body_fx=0.02)
    o = build_oracle(case)
    o.step(5)
    sim = build_gpu(case, "fp64")
    sim.run(5)
    sp = case["spec"]
    assert sim.lastCappedNodes() == o.last_capped() == (sp["nx"] - 2) * (sp["ny"] - 2)
    assert sim.thermo(0)["capped_nodes"] == o.last_capped()
    assert np.array_equal(sim.field().velocity_x(), o.ux())
