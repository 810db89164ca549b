"""Capsule chemistry of the scalar on the GPU (chemistry.cu) against the
oracle (oracle/sfo.c, pinned bit for bit to the reference's
AdvectionDiffusion::applySourceSink / applyChemistry in
tests/test_oracle_golden.py) and against the reference's own outputs:

* constant release / absorption at the nearest node;
* Fick leaching from finite reservoirs, Langmuir adsorption, constant
  release of a second capsule type, Peskin-weighted exchange;
* two capsules whose stencils overlap, so the order of the reference's
  serial loop matters (waves on the GPU);
* FP64 bit for bit (concentration, scalar populations, per-capsule and
  per-node chemistry state, flow and markers); FP32 arithmetic within a
  relative L2 of 1e-4 on the concentration.
"""
import os

import numpy as np
import pytest

from cases import CASES, build_gpu, build_oracle, rel_l2

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name,steps", [("chem_source", 60), ("chem_physics", 60)])
def test_fp64_chemistry_bit_exact(sfg, oracle_mod, name, steps):
    case = CASES[name]
    o = build_oracle(case)
    o.step(steps)
    sim = build_gpu(case, "fp64")
    sim.run(steps)
    ad = sim.advectionDiffusion()
    assert np.array_equal(ad.concentration(), o.concentration())
    g = ad.populations()                                  # [9][ny][nx]
    og = o.g().reshape(-1, 9).T.reshape(g.shape)          # cell-major in the oracle
    ny = case["spec"]["ny"]
    assert np.array_equal(g[:, 1:ny - 1], og[:, 1:ny - 1])
    for mine, ref in zip(sim.chemistryState(), o.chemistry_state()):
        assert np.array_equal(mine, ref)
    assert np.array_equal(sim.field().velocity_x(), o.ux())
    assert np.array_equal(sim.capsules().positions(), o.positions())
    rel, ab, mp, gam = sim.chemistryState()
    assert (rel > 0).any() and (ab > 0).any()
    assert sim.thermo(0)["total_scalar"] == pytest.approx(float(o.concentration().sum()),
                                                         rel=1e-12)


@pytest.mark.parametrize("name", ["chem_source", "chem_physics"])
def test_fp64_chemistry_matches_reference_golden(sfg, name):
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    sim = build_gpu(CASES[name], "fp64")
    sim.run(int(g["steps"]))
    assert np.array_equal(sim.advectionDiffusion().concentration(), g["C"])
    for k, v in zip(("released", "absorbed", "Mp", "gamma"), sim.chemistryState()):
        assert np.array_equal(v, g[k]), k
    assert np.array_equal(sim.capsules().positions(), g["pos"])


@pytest.mark.parametrize("precision", ["fp32", "fp16s"])
def test_reduced_precision_chemistry(sfg, oracle_mod, precision):
    case = CASES["chem_physics"]
    o = build_oracle(case)
    o.step(60)
    sim = build_gpu(case, precision)
    sim.run(60)
    ec = rel_l2(sim.advectionDiffusion().concentration(), o.concentration())
    rel, ab, mp, gam = sim.chemistryState()
    orel, oab, omp, ogam = o.chemistry_state()
    eg = float(np.abs(gam - ogam).max() / max(np.abs(ogam).max(), 1e-30))
    print(f"{precision}: C rel L2 {ec:.3e}, gamma max rel {eg:.3e}")
    tol = 1e-4 if precision == "fp32" else 5e-3
    assert ec < tol and eg < 10 * tol
    assert np.allclose(rel, orel, rtol=10 * tol, atol=1e-12)


def test_chemistry_checkpoint_keeps_scalar(sfg, tmp_path):
    """The concentration the chemistry stored survives a host read and a
    checkpoint round trip (the stored values, not sum g)."""
    case = CASES["chem_source"]
    a = build_gpu(case, "fp64")
    a.run(10)
    C1 = a.advectionDiffusion().concentration()
    assert np.array_equal(C1, a.advectionDiffusion().concentration())
    assert float(C1.sum()) == pytest.approx(a.thermo(0)["total_scalar"], rel=1e-12)
