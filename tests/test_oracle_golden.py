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
NAMES = ["bgk_small", "mrt_small", "reg_small", "mini_c2", "contact_brute", "seam_single", "c1",
         "zouhe_bgk", "zouhe_reg", "cavity", "shear_capsule", "pillars_ibb", "pillars_zouhe",
         "chem_source", "chem_physics", "pillars_capsules", "pillars_capsules_mdf"]


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
    if "released" in g:
        for k, v in zip(("released", "absorbed", "Mp", "gamma"), o.chemistry_state()):
            assert np.array_equal(v, g[k]), k


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


@pytest.mark.parametrize("name", [n for n in NAMES if CASES[n]["capsules"]])
def test_oracle_capsule_geometry_matches_reference_golden(oracle_mod, name):
    """Capsule::centroid / area / perimeter / deformationIndex /
    inclinationAngle (capsule.cpp:159-266) of the restatement against the
    reference's values in the fixtures, bit for bit."""
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    o = build_oracle(CASES[name])
    o.step(int(g["steps"]))
    geom = np.array([[*o.capsule_centroid(c), o.capsule_area(c), o.capsule_perimeter(c),
                      o.capsule_deformation(c), o.capsule_inclination(c)]
                     for c in range(o.num_capsules)])
    assert np.array_equal(geom, g["geom"])
    assert (g["geom"][:, 4] > 0).any()      # the capsules have deformed


def test_oracle_stats_restatement():
    """The serial reductions of oracle/stats.py on a small field with SOLID
    rows, a NaN cell and known extremes."""
    from oracle import stats as OS
    ny, nx = 5, 4
    rng = np.random.default_rng(3)
    rho = 1.0 + 0.01 * rng.standard_normal((ny, nx))
    ux = 0.02 * rng.standard_normal((ny, nx))
    uy = 0.02 * rng.standard_normal((ny, nx))
    solid = OS.solid_mask(nx, ny, False)
    rho[solid] = ux[solid] = uy[solid] = 0.0
    st = OS.global_stats(rho, ux, uy, solid, [0.1, 0.3])
    f = ~solid
    assert st["fluid_cells"] == f.sum()
    assert st["max_velocity"] == OS.max_speed(ux, uy, solid)
    assert np.isclose(st["max_velocity"], np.sqrt((ux[f] ** 2 + uy[f] ** 2).max()), rtol=0, atol=0)
    assert np.isclose(st["mean_rho"], rho[f].mean(), rtol=1e-14)
    assert st["min_rho"] == rho[f].min() and st["max_rho"] == rho[f].max()
    assert np.isclose(st["total_kinetic_energy"], (0.5 * rho * (ux ** 2 + uy ** 2))[f].sum(),
                      rtol=1e-14)
    assert st["mean_deformation"] == 0.2 and st["max_deformation"] == 0.3
    assert OS.first_nonfinite(rho, ux, uy, solid) == -1
    ux[3, 1] = np.nan
    ux[2, 2] = np.inf
    assert OS.first_nonfinite(rho, ux, uy, solid) == 2 * nx + 2


BOUNDARY_CASES = [("zouhe_bgk", 300), ("zouhe_mrt", 300), ("zouhe_reg", 300), ("cavity", 400),
                  ("shear_capsule", 60)]


@pytest.mark.skipif(not O.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("name,steps", BOUNDARY_CASES)
def test_oracle_boundaries_match_live_reference(oracle_mod, name, steps):
    """Zou-He inlet / outlet (zou_he_boundary.cpp), closed box, moving walls
    (moving_wall.cpp): the restatement against the reference's own
    LBMSolver, bit for bit."""
    case = CASES[name]
    a = build_oracle(case, "sfo")
    b = build_oracle(case, "ref")
    a.step(steps)
    b.step(steps)
    for k in ("f", "ux", "uy", "rho", "positions", "velocities"):
        assert np.array_equal(getattr(a, k)(), getattr(b, k)()), k


@pytest.mark.skipif(not O.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("name,steps", [("pillars_bb", 300), ("pillars_ibb", 300),
                                        ("pillars_zouhe", 300)])
def test_oracle_pillars_match_live_reference(oracle_mod, name, steps):
    """ChannelBuilder pillars (channel_builder.cpp) with halfway and
    interpolated bounce-back (interpolated_bounce_back.cpp): bit for bit."""
    case = CASES[name]
    a = build_oracle(case, "sfo")
    b = build_oracle(case, "ref")
    a.step(steps)
    b.step(steps)
    for k in ("f", "ux", "uy", "rho"):
        assert np.array_equal(getattr(a, k)(), getattr(b, k)()), k


@pytest.mark.skipif(not O.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("name,steps", [("pillars_capsules", 200),
                                        ("pillars_capsules_mdf", 200)])
def test_oracle_capsules_among_pillars_match_live_reference(oracle_mod, name, steps):
    """Capsules among pillars: placement that rejects the pillars
    (simulation.cpp:256-261) and the obstacle repulsion
    (repulsion.cpp:180-235, after the pair contact), bit for bit."""
    case = CASES[name]
    a = build_oracle(case, "sfo")
    b = build_oracle(case, "ref")
    a.step(steps)
    b.step(steps)
    for k in ("f", "ux", "uy", "rho", "positions", "velocities", "forces"):
        assert np.array_equal(getattr(a, k)(), getattr(b, k)()), k


@pytest.mark.skipif(not O.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("name,steps", [("chem_source", 60), ("chem_physics", 60)])
def test_oracle_chemistry_matches_live_reference(oracle_mod, name, steps):
    """Capsule chemistry of the scalar (applySourceSink / applyChemistry,
    advection_diffusion.cpp:225-437): concentration, scalar populations and
    the per-capsule / per-node chemistry state, bit for bit."""
    case = CASES[name]
    a = build_oracle(case, "sfo")
    b = build_oracle(case, "ref")
    a.step(steps)
    b.step(steps)
    for k in ("concentration", "g", "ux", "positions"):
        assert np.array_equal(getattr(a, k)(), getattr(b, k)()), k
    for x, y in zip(a.chemistry_state(), b.chemistry_state()):
        assert np.array_equal(x, y)
    rel, ab, mp, gam = a.chemistry_state()
    assert (rel > 0).any() and (ab > 0).any()
