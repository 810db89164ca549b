"""Accuracy of the reduced-precision forms at the configurations' own sizes
and run lengths.

The bound of the chosen form is 1e-3 relative L2 of velocity against FP64.
Every case below states its measured error in the test output (-s).

* Configuration 1 (400 x 80, 30 Skalak capsules, 5 MDF sweeps): the full
  10,000 steps against the oracle, FP32 and FP16S. Checks velocity
  relative L2, the largest centroid drift relative to the distance the
  capsules travel in the run (position is the time integral of velocity,
  so it carries the velocity bound), and perimeter drift (relative).
* Configuration 0 (400 x 80 regularized channel): the full 20,000 steps
  against the oracle in FP16S.
* A 16-channel sample of the ensemble (its first 16 channels), 1,000 steps,
  FP16S with the learned and with the plain forcing. It is compared with an
  FP64 run of the same kernels and the same network, pooled and per
  channel. Each channel of the FP16S ensemble must equal, bit for bit, the
  same channel run alone.
* Configuration 2 at full size (4096 x 1024 MRT, 1,000 WLC + Helfrich and
  1,000 Skalak capsules, the scalar Gaussian). FP64 is checked against the
  oracle over 20 steps: contact pairs per marker and capped cells exact,
  fields within 1e-9 (the device atan2 / pow differ from glibc by ulps).
  FP32 and FP16S are checked against the FP64 kernels over 500 steps for
  u, rho, C, centroid and perimeter.
"""
import numpy as np
import pytest

from cases import CASES, build_gpu, build_oracle, fluid_rows, rel_l2

pytestmark = pytest.mark.gpu

VEL_TOL = {"fp32": 1e-4, "fp16s": 1e-3}


# ------------------------------------------------------------ helpers ----
def _velocity(field, rows):
    return np.stack([field.velocity_x()[rows], field.velocity_y()[rows]])


def _geometry_gpu(sim):
    st = sim.context().thermo()[1]
    return st[:, 0:2].copy(), st[:, 3].copy()


def _geometry_oracle(o):
    n = o.num_capsules
    cen = np.array([o.capsule_centroid(i) for i in range(n)])
    per = np.array([o.capsule_perimeter(i) for i in range(n)])
    return cen, per


def _min_image_dx(a, b, L):
    d = a - b
    d[:, 0] -= L * np.round(d[:, 0] / L)
    return d


# --------------------------------------------------- configuration 1 ----
@pytest.fixture(scope="module")
def c1_oracle_10k(oracle_mod):
    o = build_oracle(CASES["c1"])
    o.step(10_000)
    return o


@pytest.mark.parametrize("precision", ["fp32", "fp16s"])
def test_c1_full_run_against_oracle(sfg, c1_oracle_10k, precision):
    case = CASES["c1"]
    o = c1_oracle_10k
    sim = build_gpu(case, precision)
    sim.run(10_000)
    rows = fluid_rows(case)
    e = rel_l2(_velocity(sim.field(), rows), np.stack([o.ux()[rows], o.uy()[rows]]))
    cg, pg = _geometry_gpu(sim)
    co, po = _geometry_oracle(o)
    dc = float(np.max(np.linalg.norm(_min_image_dx(cg, co, 400.0), axis=1)))
    dp = float(np.max(np.abs(pg - po) / po))
    # distance travelled: the capsules' mean speed (their markers' mean
    # velocity, oracle) times the run length
    v = o.velocities().reshape(o.num_capsules, -1, 2).mean(axis=1)
    travel = float(np.mean(np.linalg.norm(v, axis=1))) * 10_000
    print(f"c1 {precision} 10000 steps: velocity rel L2 {e:.3e}, centroid drift {dc:.3e} lu "
          f"({dc / travel:.2e} of {travel:.0f} lu travelled), perimeter drift {dp:.3e}")
    assert e < VEL_TOL[precision]
    assert dc / travel < VEL_TOL[precision]
    assert dp < {"fp32": 1e-5, "fp16s": 1e-4}[precision]
    assert sim.lastCappedNodes() == o.last_capped()


def test_c0_full_run_fp16s_against_oracle(sfg, oracle_mod):
    case = CASES["c0"]
    o = build_oracle(case)
    o.step(20_000)
    sim = build_gpu(case, "fp16s")
    sim.run(20_000)
    rows = fluid_rows(case)
    e = rel_l2(_velocity(sim.field(), rows), np.stack([o.ux()[rows], o.uy()[rows]]))
    dr = float(np.max(np.abs(sim.field().density()[rows] - o.rho()[rows])))
    print(f"c0 fp16s 20000 steps: velocity rel L2 {e:.3e}, max |rho - rho_oracle| {dr:.2e}")
    assert e < VEL_TOL["fp16s"]


# ------------------------------------------- ensemble sample (c3) ------
N_SAMPLE = 16
SAMPLE_STEPS = 1000


def _sample(precision):
    from softflow_b200 import workloads as W
    return W.plan_c3(precision)[:N_SAMPLE]


@pytest.fixture(scope="module")
def mdf_net(sfg):
    """The headline network: trained on plain runs of configuration 1 and
    of the ensemble, 2M samples, 8 epochs (the bench's recipe)."""
    from softflow_b200.learned import training_set, train_network
    X, Y = training_set(2_000_000)
    net, losses = train_network(X, Y, epochs=8, seed=1)
    assert losses[-1] < 0.05 * losses[0]
    return net


def _run_sample(precision, net, steps, channels=None):
    from softflow_b200 import workloads as W
    plans = _sample(precision)
    if channels is not None:
        plans = [plans[i] for i in channels]
    ens = W.build(plans, precision)
    if net is not None:
        ens.setLearnedMDF(net, threshold=1e-4)
    ens.run(steps)
    return ens, plans


def _pooled_and_per_channel(a, b, plans):
    num = den = 0.0
    per = []
    for i, pl in enumerate(plans):
        rows = slice(1, pl.params.ny - 1)
        ua, ub = _velocity(a.field(i), rows), _velocity(b.field(i), rows)
        d2 = float(np.sum((ua - ub) ** 2))
        n2 = float(np.sum(ub ** 2))
        num += d2
        den += n2
        per.append(np.sqrt(d2 / n2))
    return np.sqrt(num / den), np.array(per)


@pytest.mark.parametrize("form", ["learned", "plain"])
def test_ensemble_sample_fp16s_against_fp64(sfg, mdf_net, form):
    net = mdf_net if form == "learned" else None
    ref, plans = _run_sample("fp64", net, SAMPLE_STEPS)
    got, _ = _run_sample("fp16s", net, SAMPLE_STEPS)
    pooled, per = _pooled_and_per_channel(got, ref, plans)
    fb = [got.mdfStats(i)["fallbacks"] for i in range(len(plans))] if net else []
    print(f"ensemble sample ({N_SAMPLE} channels, {SAMPLE_STEPS} steps) fp16s {form} vs fp64: "
          f"pooled {pooled:.3e}, worst channel {per.max():.3e} (channel {int(per.argmax())}), "
          f"fallback steps {sum(fb)}")
    assert pooled <= 1e-3
    assert per.max() <= 1e-3
    for i in range(len(plans)):
        assert np.isfinite(got.field(i).velocity_x()).all()
    got.close()
    ref.close()


def test_ensemble_sample_channels_equal_solo_runs(sfg, mdf_net):
    """FP16S with the learned forcing: every channel of the 16-channel
    ensemble equals the same channel run in a context of its own, bit for
    bit (the per-cell dither of the FP16 stores is keyed by the cell's
    index within its channel and the step)."""
    ens, plans = _run_sample("fp16s", mdf_net, SAMPLE_STEPS)
    for i in range(len(plans)):
        solo, _ = _run_sample("fp16s", mdf_net, SAMPLE_STEPS, channels=[i])
        assert np.array_equal(ens.field(i).distributions(), solo.field(0).distributions()), i
        assert np.array_equal(ens.capsules(i).positions(), solo.capsules(0).positions()), i
        assert ens.mdfStats(i)["fallbacks"] == solo.mdfStats(0)["fallbacks"], i
        solo.close()
    ens.close()


# --------------------------------------------------- configuration 2 ----
C2_STEPS_ORACLE = 20
C2_STEPS = 500


def _c2(precision):
    from softflow_b200 import workloads as W
    plans = W.plan_c2(precision)
    return W.build(plans, precision), plans


def test_c2_full_size_fp64_against_oracle(sfg, oracle_mod):
    """MRT at 4096 x 1024 with 2,000 capsules (1,170 x 291 contact cells)
    and the scalar, against the oracle step for step."""
    from oracle.plans import sims_from_plans
    sim, plans = _c2("fp64")
    o = sims_from_plans(plans)[0]
    assert np.array_equal(sim.capsules().positions(), o.positions())
    o.step(1)
    sim.run(1)
    counts, _ = o.contact_pairs()
    assert np.array_equal(sim.capsules().contact_counts(), counts)
    o.step(C2_STEPS_ORACLE - 1)
    sim.run(C2_STEPS_ORACLE - 1)
    rows = slice(1, 1023)
    fld = sim.field()
    errs = {k: rel_l2(getattr(fld, n)()[rows], getattr(o, k)()[rows])
            for k, n in (("ux", "velocity_x"), ("uy", "velocity_y"), ("rho", "density"))}
    C = sim.advectionDiffusion().concentration()
    errs["C"] = rel_l2(C, o.concentration())
    dx = float(np.max(np.abs(sim.capsules().positions() - o.positions())))
    print(f"c2 fp64 {C2_STEPS_ORACLE} steps vs oracle: " +
          ", ".join(f"{k} {v:.2e}" for k, v in errs.items()) + f", max |dX| {dx:.2e}")
    for k, v in errs.items():
        assert v < 1e-9, k
    assert dx < 1e-9
    assert sim.lastCappedNodes() == o.last_capped()


@pytest.fixture(scope="module")
def c2_fp64(sfg):
    sim, _ = _c2("fp64")
    sim.run(C2_STEPS)
    return dict(u=_velocity(sim.field(), slice(1, 1023)),
                rho=sim.field().density()[1:1023],
                C=sim.advectionDiffusion().concentration(),
                geom=_geometry_gpu(sim))


@pytest.mark.parametrize("precision", ["fp32", "fp16s"])
def test_c2_full_size_precision_study(sfg, c2_fp64, precision):
    sim, _ = _c2(precision)
    sim.run(C2_STEPS)
    rows = slice(1, 1023)
    eu = rel_l2(_velocity(sim.field(), rows), c2_fp64["u"])
    er = float(np.max(np.abs(sim.field().density()[rows] - c2_fp64["rho"])))
    eC = rel_l2(sim.advectionDiffusion().concentration(), c2_fp64["C"])
    cg, pg = _geometry_gpu(sim)
    co, po = c2_fp64["geom"]
    dc = float(np.max(np.linalg.norm(_min_image_dx(cg, co, 4096.0), axis=1)))
    dp = float(np.max(np.abs(pg - po) / po))
    print(f"c2 {precision} {C2_STEPS} steps vs fp64 kernels: velocity {eu:.3e}, "
          f"max |d rho| {er:.2e}, C {eC:.3e}, centroid drift {dc:.3e} lu, "
          f"perimeter drift {dp:.3e}")
    assert eu < VEL_TOL[precision]
    assert eC < {"fp32": 1e-5, "fp16s": 1e-4}[precision]
    assert dc < {"fp32": 1e-4, "fp16s": 1e-3}[precision]
    assert dp < {"fp32": 1e-6, "fp16s": 1e-5}[precision]
