"""The vectorised lattice kernels against each other.

In FP16-shifted storage the eight-cells-per-lane kernel (256-cell runs) and
the four-cells-per-lane kernel (128-cell runs) compute the same FP32 values
and differ only in the random bits of the stochastic rounding. From the
same state, after one step, every stored population of one is therefore
within one binary16 step of the other's. A misplaced load or store (a
shifted plane, a run edge, a wall row, a periodic seam, a force-tile cell)
would show up as a difference of the populations' own size.
"""
import contextlib
import io

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SCALE = 4096.0          # binary16 h = (f - w) * 2^12
W9 = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)


def _build(plans, precision, variant):
    from softflow_b200.engine import Ensemble
    ens = Ensemble(precision=precision, device=0, lattice_variant=variant)
    for i, pl in enumerate(plans):
        pl.params.precision = precision
        ens.add_channel(pl.params)
        for (count, x0, y0, x1, y1, r, nodes, mp, seed) in pl.placements:
            with contextlib.redirect_stdout(io.StringIO()):
                ens.addCapsuleRandom(i, count, x0, y0, x1, y1, r, r, nodes, mp, seed=seed,
                                     min_gap=pl.min_gap, check_walls=True)
    ens.initialize()
    return ens


def _h(f):
    return ((f - W9[:, None, None]) * SCALE).astype(np.float64)


@pytest.mark.parametrize("sample", ["ensemble", "c0"])
def test_fp16s_eight_and_four_cell_forms_agree_to_one_step(sfg, sample):
    from softflow_b200 import workloads as W
    plans = W.plan_c3("fp16s")[:12] if sample == "ensemble" else W.plan_c0("fp16s")
    src = _build(plans, "fp16s", 0)
    src.run(150)                       # a developed flow with capsule forces
    state = [(src.field(i).distributions(), src.capsules(i).positions(),
              src.capsules(i).velocities()) for i in range(len(plans))]
    src.close()
    runs = {}
    for variant in (0, 2):
        e = _build(plans, "fp16s", variant)
        for i, (f, pos, vel) in enumerate(state):
            e.field(i).set_distributions(f)
            if len(pos):
                e.capsules(i).set_state(pos, vel)
        e.run(1)
        runs[variant] = [e.field(i).distributions() for i in range(len(plans))]
        e.close()
    differ = total = 0
    for i, pl in enumerate(plans):
        rows = slice(1, pl.params.ny - 1)
        a, b = _h(runs[0][i][:, rows]), _h(runs[2][i][:, rows])
        assert np.isfinite(a).all() and np.isfinite(b).all()
        big = np.maximum(np.abs(a), np.abs(b)).astype(np.float16)
        step = np.spacing(big).astype(np.float64)
        d = np.abs(a - b)
        assert np.all(d <= step * (1 + 1e-9)), (i, float(np.max(d / np.maximum(step, 1e-30))))
        differ += int(np.count_nonzero(d))
        total += d.size
    # both forms round stochastically: a good share of the values differ
    assert 0.1 < differ / total < 0.9, differ / total
