"""Learned multi-direct forcing inside the step.

* threshold 0: every learned channel falls back to the plain sweeps, so the
  results equal the plain form bit for bit (the fallback restarts from the
  membrane-force spread of the same step);
* harvested features agree with the marker state (frame, stretch,
  curvature and target velocity against oracle/mlp.features; the previous
  correction input equals the last step's label);
* a network trained on harvested data reproduces the plain correction far
  better than no seed, and its no-slip residual matches the plain
  iteration's to the network's accuracy (within 5 %: a single channel, and
  the median over 16 ensemble channels from the same states).
"""
import numpy as np
import pytest

from oracle import mlp as Q

pytestmark = pytest.mark.gpu


def _c1(precision, K=5):
    from softflow_b200 import workloads as W
    plans = W.plan_c1(precision)
    plans[0].params.ibm_iterations = K
    return W.build(plans, precision)


def _random_net(seed=3):
    from softflow_b200.learned import MDFNetwork
    net = MDFNetwork(0, seed=seed)
    net.set_normalization(np.zeros(8), np.full(8, 1e-3), np.zeros(2), np.full(2, 1e-3))
    return net


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_zero_threshold_falls_back_to_plain_exactly(sfg, precision):
    plain = _c1(precision)
    plain.run(30)
    learned = _c1(precision)
    learned.setLearnedMDF(_random_net(), threshold=0.0)
    learned.run(30)
    assert np.array_equal(learned.field().distributions(), plain.field().distributions())
    assert np.array_equal(learned.capsules().positions(), plain.capsules().positions())
    st = learned.mdfStats(0)
    assert st["learned_steps"] == 30 and st["fallbacks"] == 30
    assert st["resid_plain"] == plain.mdfStats(0)["resid_plain"] > 0.0


def test_disable_restores_plain(sfg):
    b = _c1("fp32")
    b.setLearnedMDF(_random_net(), threshold=1.0)
    b.run(3)
    st = b.mdfStats(0)
    assert st["learned_steps"] == 3 and st["fallbacks"] == 0 and st["resid_plain"] == 0.0
    b.setLearnedMDF(None)
    b.run(5)
    st = b.mdfStats(0)
    assert st["learned_steps"] == 3 and st["resid_plain"] > 0.0


def test_harvest_features_consistent(sfg):
    ens = _c1("fp64")
    ens.run(5)
    pos0 = ens.capsules().positions().reshape(-1, 2)
    vel0 = ens.capsules().velocities().reshape(-1, 2)
    ens.setHarvest(True)
    ens.run(1)
    f1, l1, v1 = ens.harvest()
    assert v1.all()
    n = 24
    M = pos0.shape[0]
    idx = np.arange(M)
    first = (idx // n) * n
    prv = first + (idx - first - 1) % n
    nxt = first + (idx - first + 1) % n
    rest = np.full(M, 2 * 3.0 * np.sin(np.pi / n))   # chord of a 24-gon of radius 3
    z = np.zeros((M, 2))
    Fo, t, nn = Q.features(pos0, pos0[nxt], pos0[prv], rest, rest, z, vel0, z, 400.0)
    assert np.allclose(f1[:, 4], Fo[:, 4], rtol=0, atol=1e-5)
    assert np.allclose(f1[:, 5], Fo[:, 5], rtol=0, atol=1e-4)
    assert np.allclose(f1[:, 6:8], Fo[:, 6:8], rtol=0, atol=1e-7)
    # the next step's previous-correction input is this step's label
    lab_g = l1[:, :1] * t + l1[:, 1:] * nn
    pos1 = ens.capsules().positions().reshape(-1, 2)
    vel1 = ens.capsules().velocities().reshape(-1, 2)
    ens.run(1)
    f2, _, _ = ens.harvest()
    _, t2, n2 = Q.features(pos1, pos1[nxt], pos1[prv], rest, rest, z, vel1, z, 400.0)
    prev_g = f2[:, 2:3] * t2 + f2[:, 3:4] * n2
    assert np.allclose(prev_g, lab_g, rtol=1e-4, atol=1e-9)
    ens.setHarvest(False)


def test_trained_network_reproduces_plain_iteration(sfg):
    """Train on the single channel's own plain runs (5 sweeps).  From one
    state, one step in three forms: plain (4 correction sweeps), learned
    (network seed for the first 3, then the last sweep) and the same
    pipeline without the network (zero seed, then one sweep).  The learned seed is close to the
    plain correction before the last sweep and far closer than the zero
    seed, and the learned no-slip residual is no worse than the plain
    form's."""
    from softflow_b200.learned import MDFNetwork, harvest, train_network
    src = _c1("fp32")
    X, Y = harvest(src, records=300, every=5, warmup=20)
    net, losses = train_network(X, Y, epochs=20, batch=8192, lr=1e-3, seed=1)
    assert losses[-1] < 0.05 * losses[0]
    zero = MDFNetwork(0)
    zero.set_params(np.zeros(4866, np.float32))
    out = {}
    for name, model in (("plain", None), ("learned", net), ("zero", zero)):
        e = _c1("fp32")
        e.run(200)
        if model is not None:
            e.setLearnedMDF(model, threshold=1e9)   # never fall back
        e.setHarvest(True)
        e.run(1)
        _, lab, val = e.harvest()
        assert val.all()
        st = e.mdfStats(0)
        out[name] = (lab, st["resid_plain"] if model is None else st["resid_learned"])
    lp = out["plain"][0]
    err = {k: float(np.linalg.norm(out[k][0] - lp) / np.linalg.norm(lp)) for k in ("learned", "zero")}
    print(f"correction error vs plain: learned {err['learned']:.3f}, zero seed {err['zero']:.3f}; "
          f"residual plain {out['plain'][1]:.3e} learned {out['learned'][1]:.3e} "
          f"zero seed {out['zero'][1]:.3e}")
    assert err["learned"] < 0.5 * err["zero"]
    # the seed reproduces the plain correction to the network's accuracy
    # (2.4 % relative here), which adds about that much to the residual
    assert out["learned"][1] <= 1.05 * out["plain"][1]


def test_gate_residual_no_worse_than_plain_on_ensemble_sample(sfg):
    """The first 16 channels of the ensemble (FP16S), two identical plain
    runs of 200 steps (deterministic: the same state), then one step each:
    plain (4 correction sweeps) and learned (the network trained on plain
    runs, 2M samples).  Per channel, the learned form's gate residual
    against the plain iteration's residual at its last sweep: the medians
    agree to the network's accuracy (measured: 1.5 % above).  Lengthening
    the seed by the residual-minimising step lowers the one-step residual
    eightfold but destabilises the coupling within a few hundred steps
    (measured at 1.05 to 1.4 times the seed), so the seed is taken as
    predicted."""
    from softflow_b200 import workloads as W
    from softflow_b200.learned import train_network, training_set
    X, Y = training_set(2_000_000)
    net, _ = train_network(X, Y, epochs=8, seed=1)
    plans = W.plan_c3("fp16s")[:16]
    a = W.build(plans, "fp16s")
    b = W.build(W.plan_c3("fp16s")[:16], "fp16s")
    a.run(200)
    b.run(200)
    assert np.array_equal(a.field(3).distributions(), b.field(3).distributions())
    b.setLearnedMDF(net, threshold=1e9)      # never fall back: the learned sweep's own residual
    a.run(1)
    b.run(1)
    rp = np.array([a.mdfStats(i)["resid_plain"] for i in range(len(plans))])
    rl = np.array([b.mdfStats(i)["resid_learned"] for i in range(len(plans))])
    print(f"gate residual median: learned {np.median(rl):.3e}, plain {np.median(rp):.3e}; "
          f"learned <= plain on {int(np.sum(rl <= rp))} of {len(plans)} channels")
    assert np.all(rp > 0) and np.all(np.isfinite(rl))
    assert np.median(rl) <= 1.05 * np.median(rp)
