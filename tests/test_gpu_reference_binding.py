"""The reference's own Python module as the drop-in: python/bindings.cpp and
every engine source compiled unmodified into oracle/_ref/pybind/softflow_core,
with Simulation's step and run routed through libsoftflow_b200.so when the
environment variable SOFTFLOW_GPU names a precision (oracle/engine_gpu_hook.cpp,
linker symbol wrapping; oracle/Makefile target `binding`).

A user script drives the module exactly as it drives the CPU build: the
SimulationParams / MembraneParams objects, Simulation.addCapsuleRandom /
initialize, then Simulation.run (the reference's Simulation::run, GIL
released) or one Simulation.step per step from Python (the loop of
pysoftflow's SoftFlowSimulation.run, setup.py:1957-1959).  The same script
runs once on the CPU path and once on the GPU path; the fields and markers
the module exposes (LatticeField views, Capsule node positions) agree: FP64
within 1e-9 relative (the device pow of the contact law differs from glibc's
by ulps), FP16-shifted storage within the chosen form's 1e-3.
"""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
PYBIND = os.path.join(HERE, "..", "oracle", "_ref", "pybind")


@pytest.fixture(scope="module")
def core(sfg):
    if not os.path.isdir(PYBIND) or not any(f.startswith("softflow_core") for f in os.listdir(PYBIND)):
        pytest.skip("the reference's module with the GPU hook is not built")
    sys.path.insert(0, PYBIND)
    import softflow_core
    return softflow_core


def _script(sc, steps, per_step):
    """A Poiseuille channel with 30 Skalak capsules (configuration 1)."""
    p = sc.SimulationParams()
    p.nx, p.ny = 400, 80
    p.ibm_iterations = 5
    p.output_dir = "/tmp/softflow_binding_test"
    p.output_interval = 0
    p.stats_dump_every = 0
    p.probe_dump_every = 0
    p.fluid.tau = 0.8
    p.fluid.body_force_x = 3e-5
    p.fluid.boundary_type = sc.BoundaryType.PERIODIC
    p.fluid.collision_model = sc.CollisionModel.REGULARIZED
    mp = sc.MembraneParams()
    mp.model = sc.MembraneModel.SKALAK
    mp.G_s = 0.06
    mp.C_skalak = 10.0
    mp.k_bend = 0.0
    sim = sc.Simulation(p)
    sim.addCapsuleRandom(30, 20, 10, 380, 70, 3.0, 3.0, 24, mp, 0, 42, 1.0, 0)
    sim.initialize()
    if per_step:
        for _ in range(steps):
            sim.step()
    else:
        sim.run(steps)
    fld = sim.field()
    caps = sim.capsules()
    pos = np.array([[caps[c].nodePosition(i).x, caps[c].nodePosition(i).y]
                    for c in range(caps.numCapsules()) for i in range(caps[c].numNodes())])
    u = np.stack([np.array(fld.velocity_x()), np.array(fld.velocity_y())])[:, 1:-1]
    return dict(u=u, rho=np.array(fld.density())[1:-1], pos=pos, step=sim.currentStep(),
                umax=sim.getMaxSpeed())


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("per_step", [False, True])
def test_reference_module_gpu_path_fp64(core, monkeypatch, per_step):
    steps = 40
    monkeypatch.delenv("SOFTFLOW_GPU", raising=False)
    cpu = _script(core, steps, per_step)
    monkeypatch.setenv("SOFTFLOW_GPU", "fp64")
    gpu = _script(core, steps, per_step)
    e = _rel(gpu["u"], cpu["u"])
    dx = float(np.max(np.abs(gpu["pos"] - cpu["pos"])))
    print(f"reference module, {'step()' if per_step else 'run()'} x {steps}: GPU fp64 vs CPU "
          f"velocity rel L2 {e:.2e}, max |dX| {dx:.2e}")
    assert gpu["step"] == cpu["step"] == steps
    assert e < 1e-9 and _rel(gpu["rho"], cpu["rho"]) < 1e-12
    assert dx < 1e-9
    assert abs(gpu["umax"] - cpu["umax"]) < 1e-9 * cpu["umax"]


def test_reference_module_gpu_path_fp16s(core, monkeypatch):
    steps = 400
    monkeypatch.delenv("SOFTFLOW_GPU", raising=False)
    cpu = _script(core, steps, False)
    monkeypatch.setenv("SOFTFLOW_GPU", "fp16s")
    gpu = _script(core, steps, False)
    e = _rel(gpu["u"], cpu["u"])
    print(f"reference module, run() x {steps}: GPU fp16s vs CPU velocity rel L2 {e:.2e}")
    assert gpu["step"] == steps
    assert e < 1e-3
