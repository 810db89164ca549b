"""Verification checks of the GPU path against analytic solutions and the
FP64 oracle, and independence of results from the launch shapes.

* configuration 0 (400 x 80 regularized channel, tau 0.8, fx 3e-5) against
  the analytic start-up flow of plane Poiseuille (the steady parabola minus
  the odd sine modes decaying as exp(-nu (n pi / H)^2 t)); the reference's
  own Poiseuille checks (tests/verification/test_poiseuille.cpp:29-79,
  test_poiseuille_collision_operators.cpp:40-132: profile L2 < 1-2 %, flow
  rate within 2 %) on the GPU for every collision model and precision;
* capsule centroid and perimeter drift of configuration 1 in FP32 and FP16S
  against the FP64 oracle after 200 steps;
* the autotuner's launch shapes do not change any result.
"""
import math

import numpy as np
import pytest

from cases import CASES, build_gpu, build_oracle

pytestmark = pytest.mark.gpu


def _startup(H, nu, fx, t, yp, modes=401):
    """Start-up Poiseuille flow from rest under a body force: walls at
    y' = 0 and H (halfway bounce-back at y = 0.5 and ny - 1.5)."""
    u = fx / (2.0 * nu) * yp * (H - yp)
    for n in range(1, modes + 1, 2):
        k = n * math.pi / H
        u -= 4.0 * fx * H * H / (nu * math.pi ** 3 * n ** 3) * np.sin(k * yp) * math.exp(-nu * k * k * t)
    return u


def _channel(nx, ny, coll, tau, fx, precision):
    import softflow_b200 as S
    p = S.SimulationParams(nx=nx, ny=ny, precision=precision)
    p.fluid.boundary_type = S.BoundaryType.PERIODIC
    p.fluid.collision_model = coll
    p.fluid.tau = tau
    p.fluid.body_force_x = fx
    sim = S.Simulation(p)
    sim.initialize()
    return sim


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp16s"])
def test_config0_startup_profile(sfg, precision):
    import softflow_b200 as S
    nx, ny, tau, fx, steps = 400, 80, 0.8, 3e-5, 20000
    sim = _channel(nx, ny, S.CollisionModel.REGULARIZED, tau, fx, precision)
    sim.run(steps)
    nu = (tau - 0.5) / 3.0
    H = ny - 2
    yp = np.arange(1, ny - 1) - 0.5
    ua = _startup(H, nu, fx, steps, yp)
    u = sim.field().velocity_x()[1:ny - 1]
    prof = u.mean(axis=1)
    err = float(np.linalg.norm(prof - ua) / np.linalg.norm(ua))
    print(f"config 0 {precision}: profile vs start-up series rel L2 {err:.3e}")
    # the start-up series is the incompressible continuum solution (measured:
    # 4e-5 FP64, 2e-5 FP32, 5e-5 FP16S; the lattice's own error is O(1/H^2))
    assert err < 5e-4, err
    # translation invariance along x (FP16S: per-column stochastic rounding)
    spread = float((u.max(axis=1) - u.min(axis=1)).max() / u.max())
    assert spread < {"fp64": 1e-10, "fp32": 1e-4, "fp16s": 5e-3}[precision], spread


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp16s"])
@pytest.mark.parametrize("coll_name,tau", [("BGK", 0.8), ("MRT", 0.8), ("REGULARIZED", 0.8),
                                           ("BGK", 1.2), ("REGULARIZED", 1.2)])
def test_poiseuille_steady(sfg, precision, coll_name, tau):
    """test_poiseuille_collision_operators.cpp:40-132 on the GPU: 8 x 34,
    fx 1e-6, 5 H^2 / nu steps; L2 of the profile < 2 %, flow rate within 2 %."""
    import softflow_b200 as S
    coll = getattr(S.CollisionModel, coll_name)
    nx, ny, fx = 8, 34, 1e-6
    nu = (tau - 0.5) / 3.0
    steps = int(5.0 * 32 * 32 / nu)
    sim = _channel(nx, ny, coll, tau, fx, precision)
    sim.run(steps)
    H = ny - 2
    ux = sim.field().velocity_x()
    u = ux[1:H + 1, nx // 2]
    yp = np.arange(H) + 0.5
    ua = fx / (2.0 * nu) * yp * (H - yp)
    l2 = float(np.linalg.norm(u - ua) / np.linalg.norm(ua))
    q = float(u.sum() / (fx * H ** 3 / (12.0 * nu)))
    # FP16 storage keeps (f - w) * 2^12 in binary16: at u ~ 1e-3 its
    # resolution bounds the profile error, not the method
    tol = 0.02 if precision != "fp16s" else 0.05
    print(f"{coll_name} tau {tau} {precision}: L2 {l2:.3e}, Q/Q_an {q:.5f}")
    assert l2 < tol and abs(q - 1.0) < tol, (l2, q)


@pytest.mark.parametrize("precision,tol_c,tol_p", [("fp32", 1e-5, 1e-8), ("fp16s", 1e-3, 2e-5)])
def test_capsule_centroid_perimeter_drift(sfg, oracle_mod, precision, tol_c, tol_p):
    case = CASES["c1"]
    o = build_oracle(case)
    o.step(200)
    sim = build_gpu(case, precision)
    sim.run(200)
    caps = sim.capsules()
    n = caps.numCapsules()
    dc = max(float(np.hypot(*(np.array(caps[i].centroid()) - np.array(o.capsule_centroid(i)))))
             for i in range(n))
    dp = max(abs(caps[i].perimeter() / o.capsule_perimeter(i) - 1.0) for i in range(n))
    print(f"{precision}: centroid drift {dc:.3e} lu, perimeter {dp:.3e}")
    assert dc < tol_c, dc
    assert dp < tol_p, dp


@pytest.mark.parametrize("learned", [False, True])
def test_autotuned_launch_shapes_keep_results(sfg, learned):
    """Every kernel's arithmetic and order per cell and per marker are
    independent of grid and block sizes, so the tuned context and an
    untuned one advanced by the same steps agree bit for bit."""
    from softflow_b200 import workloads as W
    a = W.build(W.plan_c1("fp32"), "fp32")
    b = W.build(W.plan_c1("fp32"), "fp32")
    if learned:
        from softflow_b200.learned import MDFNetwork
        net = MDFNetwork(0, seed=5)
        net.set_normalization(np.zeros(8), np.full(8, 1e-3), np.zeros(2), np.full(2, 1e-3))
        a.setLearnedMDF(net, threshold=1.0)
        b.setLearnedMDF(net, threshold=1.0)
    cfg = a.autotune(steps_per_trial=2)
    assert cfg["steps_run"] > 0
    assert cfg["lattice_ctas_per_sm"] >= 1 and cfg["spread_ctas_per_sm"] >= 1
    assert cfg["marker_block"] in (64, 128, 256)
    b.run(cfg["steps_run"])
    a.run(7)
    b.run(7)
    assert np.array_equal(a.field().distributions(), b.field().distributions())
    assert np.array_equal(a.capsules().positions(), b.capsules().positions())


def _feq(rho, ux, uy):
    """Second-order equilibrium of reference lattice.h:35-39, [9][ny][nx]."""
    W = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
    CX = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])
    CY = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])
    cs2 = 1.0 / 3.0
    out = np.empty((9,) + rho.shape)
    uu = ux * ux + uy * uy
    for q in range(9):
        eu = CX[q] * ux + CY[q] * uy
        out[q] = W[q] * rho * (1.0 + eu / cs2 + eu * eu / (2 * cs2 * cs2) - uu / (2 * cs2))
    return out


@pytest.mark.parametrize("precision,tol", [("fp64", 0.02), ("fp32", 0.02), ("fp16s", 0.03)])
def test_taylor_green_decay(sfg, precision, tol):
    """test_taylor_green.cpp:36-104: a 64 x 64 doubly periodic Taylor-Green
    vortex (U0 0.04, BGK tau 0.8) loses kinetic energy as exp(-2 nu k^2 t):
    after one e-fold of the amplitude E(t)/E(0) is exp(-2) within 2 %."""
    import softflow_b200 as S
    nx = ny = 64
    p = S.SimulationParams(nx=nx, ny=ny, precision=precision)
    p.fluid.boundary_type = S.BoundaryType.PERIODIC
    p.fluid.periodic_y = True
    p.fluid.collision_model = S.CollisionModel.BGK
    p.fluid.tau = 0.8
    p.enable_stability_checks = False
    sim = S.Simulation(p)
    sim.initialize()
    U0, kx, ky = 0.04, 2 * math.pi / nx, 2 * math.pi / ny
    y, x = np.mgrid[0:ny, 0:nx].astype(float)
    ux = -U0 * np.cos(kx * x) * np.sin(ky * y)
    uy = U0 * np.sin(kx * x) * np.cos(ky * y)
    rho = 1.0 - (U0 * U0 / (4.0 / 3.0)) * (np.cos(2 * kx * x) + np.cos(2 * ky * y))
    sim.field().set_distributions(_feq(rho, ux, uy))
    E0 = 0.5 * float((ux * ux + uy * uy).sum())
    nu = (p.fluid.tau - 0.5) / 3.0
    n = int(1.0 / (nu * (kx * kx + ky * ky)))
    sim.run(n)
    f = sim.field()
    Et = 0.5 * float((f.velocity_x() ** 2 + f.velocity_y() ** 2).sum())
    err = abs(Et / E0 - math.exp(-2.0)) / math.exp(-2.0)
    print(f"Taylor-Green {precision}: E(t)/E(0) {Et / E0:.6f}, rel err {err:.3e}")
    assert err < tol


def test_tank_treading_frequency(sfg):
    """test_capsule_shear.cpp:15-150: a Skalak capsule (R 5) in plane Couette
    flow (walls at +-0.02, 80 x 64, regularized tau 0.8) tank-treads at
    f = gamma_dot / (4 pi) (Keller-Skalak, 2D) within 10 %: zero crossings of
    node 0's height above the centroid over the second half of the record."""
    import softflow_b200 as S
    p = S.SimulationParams(nx=80, ny=64, precision="fp32")
    p.fluid.boundary_type = S.BoundaryType.PERIODIC
    p.fluid.collision_model = S.CollisionModel.REGULARIZED
    p.fluid.tau = 0.8
    Uw = 0.02
    p.fluid.top_wall_velocity, p.fluid.bottom_wall_velocity = Uw, -Uw
    p.enable_stability_checks = False
    mp = S.MembraneParams(model=S.MembraneModel.SKALAK, G_s=0.002, C_skalak=10.0,
                          k_bend=0.001, k_area=0.02, k_perimeter=0.005, gamma_visc=0.0,
                          eta_membrane=0.0)
    sim = S.Simulation(p)
    R = 5.0
    sim.addCapsule((p.nx / 2.0, p.ny / 2.0), R, max(12, math.ceil(2 * math.pi * R / 0.75)), mp)
    sim.initialize()
    H = p.ny - 2
    gdot = 2.0 * Uw / H
    sim.run(8000)
    ry = []
    f_meas = None
    caps = sim.capsules()
    for s in range(0, 200000, 50):
        sim.run(50)
        pos = caps.positions()
        ry.append(float(pos[0, 1] - pos[:, 1].mean()))
        if len(ry) > 200:
            i0 = len(ry) // 2
            tail = np.array(ry[i0:])
            crossings = int(np.sum((tail[:-1] < 0) & (tail[1:] >= 0)) +
                            np.sum((tail[:-1] > 0) & (tail[1:] <= 0)))
            if crossings >= 6:
                T = (len(ry) - i0) * 50 / (crossings / 2.0)
                f_meas = 1.0 / T
                break
    assert f_meas is not None, "fewer than three tank-treading periods"
    f_exp = gdot / (4.0 * math.pi)
    rel = abs(f_meas - f_exp) / f_exp
    print(f"tank-treading: f {f_meas:.4e}, Keller-Skalak {f_exp:.4e}, rel {rel:.3f}")
    assert rel < 0.10


@pytest.mark.parametrize("k_a,k_d,Gmax", [(0.0, 0.0, 1.0), (0.02, 0.005, 0.1)])
def test_chemistry_mass_balance(sfg, oracle_mod, k_a, k_d, Gmax):
    """test_chemistry_mass_balance.cpp: a capsule at rest in a doubly
    periodic box leaches from a finite reservoir (and adsorbs): reservoir +
    sum C + sum Gamma ds over 200 steps.  Leaching alone conserves it to
    1e-10 relative.  With adsorption the scalar step's undershoots (C < 0
    near the capsule, tau_s 0.53) meet the chemistry's clamp of negative
    concentrations, so the reference itself loses 1.4e-6 here (its own
    sources, run on the same full steps); the GPU budget equals the
    oracle's to rounding."""
    import softflow_b200 as S
    nx, ny = 128, 96
    p = S.SimulationParams(nx=nx, ny=ny, precision="fp64")
    p.fluid.boundary_type = S.BoundaryType.PERIODIC
    p.fluid.periodic_y = True
    p.fluid.collision_model = S.CollisionModel.BGK
    p.fluid.tau = 0.6
    p.enable_stability_checks = False
    p.scalar.enabled = True
    p.scalar.diffusivity = [0.01]
    p.scalar.periodic_y = True
    p.scalar.k_leach, p.scalar.C_eq, p.scalar.M_p_initial = [0.01], [0.05], [5.0]
    p.scalar.k_adsorb, p.scalar.k_desorb, p.scalar.Gamma_max = [k_a], [k_d], [Gmax]
    sim = S.Simulation(p)
    sim.addCapsule((nx / 2.0, ny / 2.0), 32.0 / (2 * math.pi), 32, S.MembraneParams())
    sim.initialize()

    def total():
        rel, ab, mp, gam = sim.chemistryState()
        pos = sim.capsules().positions()
        d_next = np.roll(pos, -1, axis=0) - pos
        d_prev = pos - np.roll(pos, 1, axis=0)
        ds = 0.5 * (np.hypot(*d_next.T) + np.hypot(*d_prev.T))
        return (float(mp[mp >= 0].sum()) + float(sim.advectionDiffusion().concentration().sum())
                + float((gam * ds).sum()))

    import oracle as O
    o = O.OracleSim(O.ChannelSpec(nx=nx, ny=ny, collision=O.BGK, tau=0.6, periodic_y=1,
                                  scalar_enabled=1, scalar_D=0.01, scalar_periodic_y=1))
    o.add_capsule(nx / 2.0, ny / 2.0, 32.0 / (2 * math.pi), 32, O.Membrane(), 0)
    o.set_chemistry(k_leach=[0.01], C_eq=[0.05], M_p_initial=[5.0], k_adsorb=[k_a],
                    k_desorb=[k_d], Gamma_max=[Gmax])
    o.initialize()

    def o_total():
        rel, ab, mp, gam = o.chemistry_state()
        pos = o.positions()
        d_next = np.roll(pos, -1, axis=0) - pos
        d_prev = pos - np.roll(pos, 1, axis=0)
        ds = 0.5 * (np.hypot(*d_next.T) + np.hypot(*d_prev.T))
        return (float(mp[mp >= 0].sum()) + float(o.concentration().sum())
                + float((gam * ds).sum()))

    t0 = total()
    assert abs(t0 - 5.0) < 1e-12
    worst = worst_o = 0.0
    for _ in range(20):
        sim.run(10)
        o.step(10)
        worst = max(worst, abs(total() - t0) / t0)
        worst_o = max(worst_o, abs(o_total() - 5.0) / 5.0)
    rel, ab, mp, gam = sim.chemistryState()
    print(f"chemistry budget: worst rel err {worst:.3e} (oracle {worst_o:.3e}), Mp {mp[0]:.4f}")
    assert mp[0] < 5.0 - 1e-6
    if k_a == 0.0:
        assert worst < 1e-10
    else:
        assert gam.max() > 0
        assert abs(worst - worst_o) <= 1e-12
