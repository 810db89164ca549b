"""Output and restart through the device state:

* VTK files (XML and legacy) and the global-statistics row byte for byte
  against the reference's own writers on the same FP64 states
  (tests/golden/output, made by tests/golden/make_golden.py);
* the SFCK version-4 checkpoint: layout, a restart that continues a pure
  fluid run bit for bit, a checkpoint assembled from the oracle's state
  continued on the GPU, and a capsule restart;
* Simulation.run's output schedule (simulation.cpp:729-787).
"""
import os
import struct

import numpy as np
import pytest

from cases import CASES, build_gpu, build_oracle, diffusion_conc, gpu_params

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "output")


def _case(name):
    case = dict(CASES[name])
    if name == "diffusion":
        case["conc"] = diffusion_conc
    return case


@pytest.mark.parametrize("name,steps", [("bgk_small", 300), ("seam_single", 40),
                                        ("diffusion", 200)])
def test_vtk_and_stats_match_reference_writers(sfg, tmp_path, name, steps):
    from softflow_b200 import output as O
    g = np.load(os.path.join(GOLDEN, f"{name}_{steps}.npz"))
    ref = {k.replace("|", "/"): bytes(g[k]) for k in g.files}
    sim = build_gpu(_case(name), "fp64")
    sim.run(steps)
    for legacy in (False, True):
        w = O.VTKWriter(str(tmp_path / ("legacy" if legacy else "xml")), legacy=legacy)
        w.writeFluidField(sim, steps)
        w.writeCapsules(sim, steps)
    st = O.GlobalStatsWriter(str(tmp_path / "stats"))
    st.writeTimestep(sim, steps, float(steps))
    st.close()
    mine = {}
    for root, _, fns in os.walk(tmp_path):
        for fn in fns:
            full = os.path.join(root, fn)
            with open(full, "rb") as fh:
                mine[os.path.relpath(full, tmp_path)] = fh.read()
    assert sorted(mine) == sorted(ref)
    for k in ref:
        assert mine[k] == ref[k], k


def _read_sfck(path):
    with open(path, "rb") as fh:
        b = fh.read()
    assert b[:4] == b"SFCK"
    version, step, nx, ny, ncaps = struct.unpack_from("=iiiii", b, 4)
    off = 24
    N = nx * ny
    f = np.frombuffer(b, np.float64, 9 * N, off).reshape(9, ny, nx)
    off += 72 * N
    rho, ux, uy = (np.frombuffer(b, np.float64, N, off + 8 * N * i).reshape(ny, nx)
                   for i in range(3))
    off += 24 * N
    flags = np.frombuffer(b, np.int32, N, off).reshape(ny, nx)
    off += 4 * N
    caps = []
    for _ in range(ncaps):
        cid, tid, nn = struct.unpack_from("=iii", b, off)
        off += 12
        pos = np.frombuffer(b, np.float64, 2 * nn, off).reshape(nn, 2)
        vel = np.frombuffer(b, np.float64, 2 * nn, off + 16 * nn).reshape(nn, 2)
        off += 32 * nn
        area, perim, pnx = struct.unpack_from("=ddi", b, off)
        off += 20
        caps.append((cid, tid, pos, vel, area, perim, pnx))
    (nbonds,) = struct.unpack_from("=i", b, off)
    off += 4
    (has_scalar,) = struct.unpack_from("=i", b, off)
    off += 4
    extra = None
    if has_scalar:
        (ns,) = struct.unpack_from("=i", b, off)
        off += 4
        g = np.frombuffer(b, np.float64, 9 * N, off).reshape(N, 9)
        C = np.frombuffer(b, np.float64, N, off + 72 * N)
        off += 80 * N
        n_tr, = struct.unpack_from("=i", b, off)
        n_mp, = struct.unpack_from("=i", b, off + 4)
        n_g, = struct.unpack_from("=i", b, off + 8)
        off += 12
        extra = (ns, g, C, n_tr, n_mp, n_g)
    assert off == len(b)
    return dict(version=version, step=step, nx=nx, ny=ny, f=f, rho=rho, ux=ux, uy=uy,
                flags=flags, caps=caps, nbonds=nbonds, scalar=extra)


def test_checkpoint_layout(sfg, tmp_path):
    sim = build_gpu(_case("mini_c2"), "fp64")
    sim.run(12)
    path = sim.saveCheckpoint(str(tmp_path / "c.sfck"))
    d = _read_sfck(path)
    assert (d["version"], d["step"], d["nx"], d["ny"]) == (4, 12, 128, 64)
    fld = sim.field()
    assert np.array_equal(d["f"], fld.distributions())
    assert np.array_equal(d["ux"], fld.velocity_x())
    assert (d["flags"][0] == 1).all() and (d["flags"][-1] == 1).all()
    assert (d["flags"][1:-1] == 0).all()
    caps = sim.capsules()
    pos = caps.positions()
    for c, (cid, tid, p, v, area, perim, pnx) in enumerate(d["caps"]):
        o = caps._offsets[c]
        assert cid == c and pnx == 128
        assert np.array_equal(p, pos[o:o + len(p)])
        assert area == caps[c].area() and perim == caps[c].perimeter()
    ns, g, C, n_tr, n_mp, n_g = d["scalar"]
    ad = sim.advectionDiffusion()
    assert ns == 1 and (n_tr, n_mp, n_g) == (0, 0, 0)
    assert np.array_equal(g.T.reshape(9, 64, 128), ad.populations())
    assert np.array_equal(C.reshape(64, 128), ad.concentration())


@pytest.mark.parametrize("name", ["bgk_small", "diffusion"])
def test_checkpoint_restart_continues_fluid_run_exactly(sfg, tmp_path, name):
    """Without capsules the previous step's force is the body force, so a
    restart continues the run bit for bit (the reference restores u with
    that force in it)."""
    case = _case(name)
    a = build_gpu(case, "fp64")
    a.run(60)
    path = a.saveCheckpoint(str(tmp_path / "a.sfck"))
    a.run(40)
    b = build_gpu(case, "fp64")
    assert b.loadCheckpoint(path) == 60
    assert np.array_equal(b.field().velocity_x(), _read_sfck(path)["ux"])
    b.run(40)
    assert b.currentStep() == 100
    assert np.array_equal(a.field().distributions(), b.field().distributions())
    if case["conc"] is not None:
        assert np.array_equal(a.advectionDiffusion().concentration(),
                              b.advectionDiffusion().concentration())


def test_checkpoint_from_oracle_state(sfg, oracle_mod, tmp_path):
    """A checkpoint assembled in the reference layout from the oracle's
    state after 50 steps, continued on the GPU, equals the oracle's run."""
    case = CASES["reg_small"]
    o = build_oracle(case)
    o.step(50)
    nx, ny = case["spec"]["nx"], case["spec"]["ny"]
    flags = np.zeros((ny, nx), np.int32)
    flags[0] = flags[-1] = 1
    path = str(tmp_path / "o.sfck")
    with open(path, "wb") as fh:
        fh.write(b"SFCK" + struct.pack("=iiiii", 4, 50, nx, ny, 0))
        for a in (o.f(), o.rho(), o.ux(), o.uy()):
            fh.write(np.ascontiguousarray(a, np.float64).tobytes())
        fh.write(flags.tobytes())
        fh.write(struct.pack("=ii", 0, 0))
    sim = build_gpu(case, "fp64")
    sim.loadCheckpoint(path)
    sim.run(30)
    o.step(30)
    rows = slice(1, ny - 1)
    assert np.array_equal(sim.field().distributions()[:, rows], o.f()[:, rows])
    assert np.array_equal(sim.field().velocity_x(), o.ux())


def test_checkpoint_restart_with_capsules(sfg, tmp_path):
    """Capsules: positions and velocities restored exactly; the first step
    after the restart lacks the previous step's capsule force in u and the
    membrane's viscous memory (as the reference's restart does for the
    latter), so the runs part by a small amount."""
    case = _case("seam_single")
    a = build_gpu(case, "fp64")
    a.run(30)
    path = a.saveCheckpoint(str(tmp_path / "s.sfck"))
    pos0 = a.capsules().positions()
    a.run(20)
    b = build_gpu(case, "fp64")
    b.loadCheckpoint(path)
    assert np.array_equal(b.capsules().positions(), pos0)
    b.run(20)
    dp = np.abs(a.capsules().positions() - b.capsules().positions()).max()
    du = np.abs(a.field().velocity_x() - b.field().velocity_x()).max()
    print(f"capsule restart after 20 steps: max |dX| {dp:.3e} lu, max |du| {du:.3e}")
    assert dp < 1e-3 and du < 1e-4


def test_checkpoint_rejects_mismatch(sfg, tmp_path):
    from softflow_b200.output import CheckpointError
    a = build_gpu(_case("bgk_small"), "fp64")
    a.run(3)
    path = a.saveCheckpoint(str(tmp_path / "x.sfck"))
    b = build_gpu(_case("reg_small"), "fp64")   # 64 x 20 as well: accepted
    b.loadCheckpoint(path)
    c = build_gpu(_case("seam_single"), "fp64")
    with pytest.raises(CheckpointError, match="domain mismatch"):
        c.loadCheckpoint(path)
    with pytest.raises(CheckpointError, match="not stepped"):
        a.loadCheckpoint(path)


def test_run_output_schedule(sfg, tmp_path):
    """Simulation::step writes after the steps whose count before the step
    is a multiple of the interval; the checkpoint skips step 0; run() ends
    with the PVD collections."""
    import softflow_b200 as S
    p = gpu_params(_case("seam_single"), "fp32")
    p.output_dir = str(tmp_path)
    p.output_interval = 10
    p.stats_dump_every = 10
    p.checkpoint_interval = 10
    p.probes = [(5, 5, "a")]
    p.probe_dump_every = 7
    sim = S.Simulation(p)
    S.Ensemble.addCapsule(sim, 0, (20.0, 15.0), 4.0, 24)
    sim.initialize()
    sim.run(25)
    names = sorted(os.listdir(tmp_path))
    assert [n for n in names if n.startswith("checkpoint")] == ["checkpoint_10.sfck",
                                                               "checkpoint_20.sfck"]
    assert sorted(os.listdir(tmp_path / "fluid")) == ["fluid.pvd", "fluid_000000.vti",
                                                      "fluid_000010.vti", "fluid_000020.vti"]
    assert len(os.listdir(tmp_path / "particles")) == 4
    rows = open(tmp_path / "global_stats.csv").read().splitlines()
    assert [r.split(",")[0] for r in rows[1:]] == ["0", "10", "20"]
    probes = open(tmp_path / "fluid_probes.csv").read().splitlines()
    assert [r.split(",")[0] for r in probes[1:]] == ["0", "7", "14", "21"]
    csv = open(tmp_path / "particle_data.csv").read().splitlines()
    assert csv[0] == "timestep,time,capsule_id,type,cx,cy,vx,vy" and len(csv) == 4
    # stamped with the count before the step, as the reference stamps it
    assert _read_sfck(tmp_path / "checkpoint_20.sfck")["step"] == 20


@pytest.mark.parametrize("precision", ["fp64", "fp16s"])
def test_set_all_populations_equals_per_channel(sfg, precision):
    """sfg_set_all_populations (every channel's FP64 populations back to
    back, copies overlapped with the import) leaves the same device state as
    one sfg_set_populations per channel."""
    from softflow_b200 import _lib as L
    from softflow_b200 import workloads as W
    plans = W.plan_c3(precision, n_channels=5)
    a = W.build(plans, precision)
    b = W.build(W.plan_c3(precision, n_channels=5), precision)
    a.run(3)
    rng = np.random.default_rng(4)
    fs = []
    for i in range(len(plans)):
        f = a.field(i).distributions()
        fs.append(f + 1e-4 * rng.standard_normal(f.shape))
    flat = np.concatenate([f.ravel() for f in fs])
    ctx = b.context()
    L.check(ctx._lib.sfg_set_all_populations(ctx._h, L.dptr(flat)))
    for i, f in enumerate(fs):
        L.check(a.context()._lib.sfg_set_populations(a.context()._h, i, L.dptr(f.ravel().copy())))
    for i in range(len(plans)):
        assert np.array_equal(a.field(i).distributions(), b.field(i).distributions())
