"""Generates the golden fixtures from the reference engine's own sources.

Runs in the build container, where the reference tree is present and
oracle/Makefile has compiled it into oracle/_ref/libsfref.so (deterministic
build, one OpenMP thread).  Writes tests/golden/*.npz.  The fixtures are
outputs of the reference itself on seeded inputs; the tests compare the CPU
restatement (oracle/sfo.c) and the GPU path against them.

    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py NAME ...   # the named cases only
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from cases import CASES, build_oracle, diffusion_conc, fluid_rows  # noqa: E402

# Output files of the reference's own writers (VTKWriter, GlobalStatsWriter)
# on states the GPU path reproduces bit for bit in FP64.
OUTPUT_RUNS = [("bgk_small", 300), ("seam_single", 40), ("diffusion", 200)]

RUNS = [("bgk_small", 300), ("mrt_small", 300), ("reg_small", 300), ("mini_c2", 30),
        ("contact_brute", 60), ("seam_single", 40), ("c1", 10),
        ("zouhe_bgk", 300), ("zouhe_reg", 300), ("cavity", 400), ("shear_capsule", 60),
        ("pillars_ibb", 300), ("pillars_zouhe", 300), ("chem_source", 60),
        ("chem_physics", 60), ("pillars_capsules", 200), ("pillars_capsules_mdf", 200)]


def main(only=None):
    oracle.build(ref=True)
    for name, steps in RUNS:
        if only and name not in only:
            continue
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
        if case.get("chem"):
            rel, ab, mp, gam = o.chemistry_state()
            out.update(released=rel, absorbed=ab, Mp=mp, gamma=gam, g=o.g())
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path))


def outputs():
    """tests/golden/output/<case>_<steps>.npz: the bytes of every file the
    reference's writers produce for the state after <steps> steps (XML and
    legacy VTK, one global_stats.csv row at time = steps)."""
    import tempfile
    oracle.build(ref=True)
    os.makedirs(os.path.join(HERE, "output"), exist_ok=True)
    for name, steps in OUTPUT_RUNS:
        case = dict(CASES[name])
        if name == "diffusion":
            case["conc"] = diffusion_conc
        o = build_oracle(case, impl="ref")
        o.step(steps)
        files = {}
        with tempfile.TemporaryDirectory() as td:
            for legacy in (False, True):
                d = os.path.join(td, "legacy" if legacy else "xml")
                o.write_vtk(d, steps, legacy)
            o.write_global_stats(os.path.join(td, "stats"), steps, float(steps))
            for root, _, fns in os.walk(td):
                for fn in fns:
                    full = os.path.join(root, fn)
                    rel = os.path.relpath(full, td)
                    with open(full, "rb") as fh:
                        files[rel] = np.frombuffer(fh.read(), dtype=np.uint8)
        path = os.path.join(HERE, "output", f"{name}_{steps}.npz")
        np.savez_compressed(path, **{k.replace("/", "|"): v for k, v in files.items()})
        print(path, os.path.getsize(path), sorted(files))


if __name__ == "__main__":
    main(sys.argv[1:])
    if len(sys.argv) == 1:
        outputs()
