"""Device-side thermo (sfg_thermo) and the multi-step run with per-interval
thermo (sfg_run) against the oracle's restatements of the reference's
reductions (oracle/stats.py; Capsule geometry in oracle/sfo.c):

* max speed, extremes of rho, counts and capsule sums exact; the cell sums
  (mean rho, mean |u|, kinetic energy, total scalar) within rounding of the
  reference's serial order;
* capsule centroid / area / perimeter / deformation exact in FP64 on the
  same marker positions, inclination within the ulps of atan2;
* sfg_run calls back on schedule, stops on request and leaves the state of
  plain steps; the stability check runs at the reference's steps.
"""
import numpy as np
import pytest

from cases import CASES, build_gpu, build_oracle

pytestmark = pytest.mark.gpu


def _solid(sim):
    from oracle import stats as OS
    p = sim.params()
    return OS.solid_mask(p.nx, p.ny, p.fluid.periodic_y)


def _check_cells(t, rho, ux, uy, solid, C=None):
    from oracle import stats as OS
    ref = OS.global_stats(rho, ux, uy, solid, [], C)
    assert t["max_speed"] == OS.max_speed(ux, uy, solid)
    assert t["min_rho"] == ref["min_rho"] and t["max_rho"] == ref["max_rho"]
    assert t["fluid_cells"] == ref["fluid_cells"]
    for k, r in (("mean_rho", "mean_rho"), ("mean_velocity", "mean_velocity"),
                 ("kinetic_energy", "total_kinetic_energy")):
        # fixed tree order on the device, row-major serial in the reference
        assert abs(t[k] - ref[r]) <= 1e-12 * abs(ref[r]), (k, t[k], ref[r])
    if C is not None:
        assert abs(t["total_scalar"] - ref["total_dissolved_mass"]) <= \
            1e-11 * abs(ref["total_dissolved_mass"])
    assert t["first_nonfinite"] == -1


def test_thermo_fp64_lattice_equals_oracle_run(sfg, oracle_mod):
    """FP64 lattice runs are bit-exact, so the device max speed equals the
    reference's getMaxSpeed of the oracle's own fields."""
    from oracle import stats as OS
    case = CASES["reg_small"]
    o = build_oracle(case)
    o.step(200)
    sim = build_gpu(case, "fp64")
    sim.run(200)
    t = sim.thermo(0)
    _check_cells(t, o.rho(), o.ux(), o.uy(), _solid(sim))
    assert sim.getMaxSpeed() == OS.max_speed(o.ux(), o.uy(), _solid(sim))


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp16s"])
def test_thermo_cells_match_exported_fields(sfg, precision):
    """The reductions see exactly the rho and u that sfg_get_macroscopic
    exports (the reference's computeMacroscopic state)."""
    case = CASES["mini_c2"]
    sim = build_gpu(case, precision)
    sim.run(30)
    t = sim.thermo(0)
    f = sim.field()
    C = sim.advectionDiffusion().concentration()
    _check_cells(t, f.density(), f.velocity_x(), f.velocity_y(), _solid(sim), C)
    assert t["capped_nodes"] == sim.lastCappedNodes()
    assert t["num_capsules"] == sim.capsules().numCapsules()


@pytest.mark.parametrize("name", ["c1", "mini_c2", "seam_single"])
def test_capsule_geometry_equals_oracle(sfg, oracle_mod, name):
    """Geometry of the GPU's own marker positions, computed by the device
    and by the restatement: FP64 bit for bit (inclination: atan2 ulps)."""
    case = CASES[name]
    sim = build_gpu(case, "fp64")
    sim.run(40)
    caps = sim.capsules()
    pos = caps.positions()
    o = build_oracle(case)
    o.set_markers(pos=pos)
    n = caps.numCapsules()
    for c in range(n):
        cv = caps[c]
        assert cv.centroid() == o.capsule_centroid(c)
        assert cv.area() == o.capsule_area(c)
        assert cv.perimeter() == o.capsule_perimeter(c)
        assert cv.deformationIndex() == o.capsule_deformation(c)
        assert abs(cv.inclinationAngle() - o.capsule_inclination(c)) <= 4e-16 * np.pi
    D = [o.capsule_deformation(c) for c in range(n)]
    t = sim.thermo(0)
    assert t["max_deformation"] == max(D)
    s = 0.0
    for d in D:
        s += d
    assert t["mean_deformation"] == s / n


def test_thermo_first_nonfinite_cell(sfg):
    """checkStability's first non-finite cell in row-major order."""
    case = CASES["bgk_small"]
    sim = build_gpu(case, "fp64")
    sim.run(3)
    fld = sim.field()
    f = fld.distributions()
    nx = f.shape[2]
    f[4, 7, 3] = np.nan
    f[2, 5, 9] = np.inf
    fld.set_distributions(f)
    assert sim.thermo(0)["first_nonfinite"] == 5 * nx + 9
    msg = sim.checkStability(0)
    assert msg["nonfinite"] == (9, 5)


def test_run_thermo_schedule_and_stop(sfg):
    case = CASES["seam_single"]
    a = build_gpu(case, "fp32")
    b = build_gpu(case, "fp32")
    seen = []

    def cb(step, recs, caps):
        seen.append((step, recs[0]["max_speed"], caps.shape))
        return False
    assert a.run(20, thermo_every=7, callback=cb) == 20
    assert [s for s, _, _ in seen] == [7, 14, 20]
    assert all(shape == (1, 6) for _, _, shape in seen)
    b.run(20)
    assert np.array_equal(a.field().distributions(), b.field().distributions())
    assert np.array_equal(a.capsules().positions(), b.capsules().positions())
    assert seen[-1][1] == b.getMaxSpeed()

    stops = []

    def stop_at_14(step, recs, caps):
        stops.append(step)
        return step >= 14
    c = build_gpu(case, "fp32")
    assert c.run(100, thermo_every=7, callback=stop_at_14) == 14
    assert stops == [7, 14] and c.currentStep() == 14


def test_stability_check_schedule(sfg, capsys):
    """Simulation::step checks after the steps whose count before the step
    is a multiple of stability_check_interval (simulation.cpp:729-733)."""
    from cases import gpu_params
    import softflow_b200 as S
    p = gpu_params(CASES["bgk_small"], "fp32")
    p.max_velocity = 1e-12
    p.stability_check_interval = 5
    sim = S.Simulation(p)
    sim.initialize()
    sim.run(12)
    err = capsys.readouterr().err
    steps = [int(line.split("at step ")[1].split()[0])
             for line in err.splitlines() if "high velocity" in line]
    assert steps == [0, 5, 10]


def test_async_marker_readback(sfg):
    """sfg_get_all_markers_async: every step's snapshot, landed through the
    copy stream while later steps run, equals the synchronous read."""
    import ctypes as C
    import torch
    from softflow_b200 import _lib as L
    case = CASES["c1"]
    a = build_gpu(case, "fp32")
    b = build_gpu(case, "fp32")
    M = a.capsules().totalNodes()
    bufs = [(torch.zeros(2 * M, dtype=torch.float64).pin_memory(),
             torch.zeros(2 * M, dtype=torch.float64).pin_memory()) for _ in range(2)]
    ca, cb = a.context(), b.context()
    got = []
    for s in range(6):
        L.check(ca._lib.sfg_step(ca._h, 1))
        if s >= 1:
            L.check(ca._lib.sfg_wait_markers(ca._h, (s - 1) % 2))
            got.append(bufs[(s - 1) % 2][0].numpy().copy())
        p, v = bufs[s % 2]
        L.check(ca._lib.sfg_get_all_markers_async(ca._h, s % 2, L.dptr(p.numpy()),
                                                  L.dptr(v.numpy())))
    L.check(ca._lib.sfg_wait_markers(ca._h, 5 % 2))
    got.append(bufs[5 % 2][0].numpy().copy())
    for s in range(6):
        b.run(1)
        pos = np.zeros(2 * M)
        L.check(cb._lib.sfg_get_all_markers(cb._h, L.dptr(pos), None))
        assert np.array_equal(got[s], pos), s
