"""The C restatement (oracle/sfo.c) against the reference engine: bit for bit
against the committed golden fixtures (outputs of the reference's own
sources, tests/golden/make_golden.py) and, where the reference build is
present, against a live run of it."""
import os

import numpy as np
import pytest

import oracle as O
from cases import CASES, build_oracle, fluid_rows

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ["bgk_small", "mrt_small", "reg_small", "mini_c2", "contact_brute", "seam_single", "c1"]


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference_golden(oracle_mod, name):
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    case = CASES[name]
    o = build_oracle(case)
    o.step(int(g["steps"]))
    for k in ("ux", "uy", "rho"):
        assert np.array_equal(getattr(o, k)(), g[k]), k
    assert o.last_capped() == int(g["capped"])
    if "f" in g:
        assert np.array_equal(o.f()[:, fluid_rows(case)], g["f"])
    if "pos" in g:
        assert np.array_equal(o.positions(), g["pos"])
        assert np.array_equal(o.velocities(), g["vel"])
        assert np.array_equal(o.forces(), g["force"])
    if "C" in g:
        assert np.array_equal(o.concentration(), g["C"])


@pytest.mark.skipif(not O.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("name,steps", [("c1_plain", 25), ("mini_c2", 25), ("diffusion", 200)])
def test_oracle_matches_live_reference(oracle_mod, name, steps):
    case = dict(CASES[name])
    if name == "diffusion":
        case["conc"] = lambda nx, ny: np.exp(-((np.arange(nx)[None, :] - nx / 2.0) ** 2) /
                                             (2 * 64.0)) * np.ones((ny, 1))
    a = build_oracle(case, "sfo")
    b = build_oracle(case, "ref")
    a.step(steps)
    b.step(steps)
    for k in ("ux", "uy", "rho", "positions", "velocities", "forces"):
        assert np.array_equal(getattr(a, k)(), getattr(b, k)()), k
    if case["conc"] is not None:
        assert np.array_equal(a.concentration(), b.concentration())


def test_peskin_table_matches_reference(oracle_mod):
    if not O.ref_available():
        pytest.skip("reference build absent")
    for r in np.linspace(-2.5, 2.5, 1001):
        assert O.phi(float(r), "sfo") == O.phi(float(r), "ref")
