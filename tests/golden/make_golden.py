"""Generates the golden fixtures from the reference engine's own sources.

Runs in the build container, where the reference tree is present and
oracle/Makefile has compiled it into oracle/_ref/libsfref.so (deterministic
build, one OpenMP thread).  Writes tests/golden/*.npz.  The fixtures are
outputs of the reference itself on seeded inputs; the tests compare the CPU
restatement (oracle/sfo.c) and the GPU path against them.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from cases import CASES, build_oracle, fluid_rows  # noqa: E402

RUNS = [("bgk_small", 300), ("mrt_small", 300), ("reg_small", 300), ("mini_c2", 30),
        ("contact_brute", 60), ("seam_single", 40), ("c1", 10)]


def main():
    oracle.build(ref=True)
    for name, steps in RUNS:
        case = CASES[name]
        o = build_oracle(case, impl="ref")
        o.step(steps)
        rows = fluid_rows(case)
        out = dict(steps=steps, ux=o.ux(), uy=o.uy(), rho=o.rho(), capped=o.last_capped())
        if not case["capsules"]:
            out.update(f=o.f()[:, rows])
        else:
            out.update(pos=o.positions(), vel=o.velocities(), force=o.forces())
            # Capsule::centroid / area / perimeter / deformationIndex /
            # inclinationAngle of the reference (capsule.cpp:159-266)
            n = o.num_capsules
            out.update(geom=np.array([[*o.capsule_centroid(c), o.capsule_area(c),
                                       o.capsule_perimeter(c), o.capsule_deformation(c),
                                       o.capsule_inclination(c)] for c in range(n)]))
        if case["conc"] is not None:
            out.update(C=o.concentration())
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
