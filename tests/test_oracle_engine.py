"""The orchestration restatement against the reference's own engine.

oracle/ref_driver.cpp calls the reference's physics classes in the order of
Simulation::step and restates Simulation::addCapsuleRandom;
oracle/ref_engine.cpp calls softflow::Simulation itself (engine/simulation.cpp
compiled unmodified with the rest of the reference sources).  Built with the
same deterministic flags, the two agree bit for bit: placement, populations,
macroscopic fields and forces, marker positions, velocities and forces, and
the scalar, on channels with capsules and MDF, contact, WLC + Helfrich,
pillars, chemistry, Zou-He and moving walls.  That pins the seeded
placement, the body force and force cap, the move and the y-clamp of every
GPU parity test to the reference's own Simulation::step.
"""
import os

import numpy as np
import pytest

import oracle as O
from cases import CASES, build_oracle

pytestmark = pytest.mark.skipif(not os.path.exists(O.ENGINE_LIB),
                                reason="reference engine library not built")

FIELDS = ("f", "ux", "uy", "rho", "Fx", "Fy", "positions", "velocities", "forces")


@pytest.mark.parametrize("name,steps", [("c1", 40), ("mini_c2", 40), ("contact_brute", 60),
                                        ("seam_single", 60), ("pillars_capsules", 60),
                                        ("pillars_capsules_mdf", 40), ("chem_physics", 40),
                                        ("chem_source", 40), ("zouhe_bgk", 100),
                                        ("cavity", 100), ("shear_capsule", 40),
                                        ("pillars_ibb", 80), ("c0", 100)])
def test_restated_step_equals_reference_engine(oracle_mod, name, steps):
    a = build_oracle(CASES[name], impl="ref")
    b = build_oracle(CASES[name], impl="engine")
    assert np.array_equal(a.positions(), b.positions())
    a.step(steps)
    b.step(steps)
    for k in FIELDS:
        assert np.array_equal(getattr(a, k)(), getattr(b, k)()), k
    if CASES[name]["conc"] is not None:
        assert np.array_equal(a.concentration(), b.concentration())
