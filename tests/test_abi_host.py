"""C-ABI checks that need no GPU: the library loads, exports every entry
point the header declares, rejects bad arguments, and its host-side setup
helpers (capsule rest geometry, seeded placement) reproduce the reference's
results bit for bit (compared with the CPU oracle)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "softflow_gpu.h")


def _declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(sfg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(sfg):
    lib = sfg.load_library()
    names = _declared()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_bad_arguments_are_rejected(sfg):
    lib = sfg.load_library()
    ctx = C.c_void_p()
    assert lib.sfg_create(0, 7, C.byref(ctx)) == 1          # SFG_ERR_ARG: unknown precision
    assert b"precision" in lib.sfg_last_error()
    assert lib.sfg_step(None, 1) == 1
    assert lib.sfg_set_all_populations(None, None) == 1
    assert b"null context" in lib.sfg_last_error()


@pytest.mark.parametrize("model,helfrich,r,n", [(O.SKALAK, 0, 3.0, 24), (O.WLC, 1, 6.0, 48),
                                                (O.HOOKEAN, 0, 5.3, 0), (O.WLC, 0, 2.1, 17)])
def test_circle_capsule_geometry_matches_reference(sfg, oracle_mod, model, helfrich, r, n):
    import softflow_b200 as S
    mp = S.MembraneParams(model=S.MembraneModel(model), use_helfrich_bending=bool(helfrich))
    rest, pos, rl, ra, rd = S.build_circle_capsule((17.25, 11.5), r, n, mp)
    o = O.OracleSim(O.ChannelSpec(nx=64, ny=32), "sfo")
    o.add_capsule(17.25, 11.5, r, n, O.Membrane(model=model, use_helfrich=helfrich))
    o.initialize()
    assert np.array_equal(pos.reshape(-1, 2), o.positions())
    assert rest.num_nodes == o.num_markers


def test_seeded_placement_matches_reference(sfg, oracle_mod):
    import softflow_b200 as S
    from cases import CASES, add_case_capsules, build_oracle, gpu_params
    for name in ("c1", "mini_c2"):
        case = CASES[name]
        e = S.Ensemble("fp32")
        e.add_channel(gpu_params(case, "fp32"))
        add_case_capsules(e, 0, case)
        pos = np.concatenate([c.pos for c in e._chans[0].caps]).reshape(-1, 2)
        assert np.array_equal(pos, build_oracle(case).positions())


def test_seeded_placement_among_pillars_matches_reference(sfg, oracle_mod):
    """Random placement with a channel builder rejects candidates within
    r + gap of a pillar (simulation.cpp:256-261): the placed capsules are the
    oracle's (itself checked against the reference in test_oracle_golden)."""
    import softflow_b200 as S
    from cases import CASES, add_case_capsules, build_oracle, gpu_params
    case = CASES["pillars_capsules"]
    sp = case["spec"]
    e = S.Ensemble("fp32")
    e.add_channel(gpu_params(case, "fp32"))
    b = S.ChannelBuilder(sp["nx"], sp["ny"])
    for ob in case["pillars"]:
        if ob[0] == "circle":
            b.addCirclePillar(*ob[1:])
        else:
            b.addRectPillar(*ob[1:])
    e.setChannelBuilder(0, b)
    add_case_capsules(e, 0, case)
    pos = np.concatenate([c.pos for c in e._chans[0].caps]).reshape(-1, 2)
    assert len(e._chans[0].caps) == 5
    assert np.array_equal(pos, build_oracle(case).positions())


def test_workload_generators_are_deterministic(sfg):
    from softflow_b200 import workloads as W
    a, b = W.plan_c3(), W.plan_c3()
    assert len(a) == 256
    assert [(p.params.nx, p.params.ny, p.params.fluid.tau, p.placements[0][0]) for p in a] == \
           [(p.params.nx, p.params.ny, p.params.fluid.tau, p.placements[0][0]) for p in b]
    for p in a:
        assert 200 <= p.params.nx <= 800 and p.params.nx % 8 == 0
        assert 40 <= p.params.ny <= 160 and p.params.ny % 8 == 0
        assert 5 <= p.placements[0][0] <= 60
        assert 0.6 <= p.params.fluid.tau <= 1.0
        assert 1e-5 <= p.params.fluid.body_force_x <= 5e-5
        assert 0.01 <= p.placements[0][7].G_s <= 0.1
