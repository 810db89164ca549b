"""Shared test cases: the same channel set up on the CPU oracle and on the
GPU library.  A case is a dict:

    spec:     oracle.ChannelSpec keyword arguments
    capsules: list of ("add", cx, cy, r, nn, membrane_kwargs)
              or ("random", count, x0, y0, x1, y1, rmin, rmax, nn,
                  membrane_kwargs, seed, min_gap, check_walls)
    conc:     None or a function (nx, ny) -> initial concentration [ny][nx]
"""
from __future__ import annotations

import numpy as np

import oracle as O


def gaussian_conc(cx, cy, sigma):
    def f(nx, ny):
        y, x = np.mgrid[0:ny, 0:nx]
        return np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2.0 * sigma * sigma))
    return f


def diffusion_conc(nx, ny):
    """Initial concentration of the diffusion fixtures: a Gaussian in x."""
    return np.exp(-((np.arange(nx)[None, :] - nx / 2.0) ** 2) / (2 * 64.0)) * np.ones((ny, 1))


SKALAK_C1 = dict(model=O.SKALAK, G_s=0.06, C_skalak=10.0, k_bend=0.0)
WLC_HELF = dict(model=O.WLC, G_s=0.06, use_helfrich=1, k_bend=0.01)

CASES = {
    # config 0 geometry (400 x 80 regularized channel, fx = 3e-5)
    "c0": dict(spec=dict(nx=400, ny=80, collision=O.REGULARIZED, tau=0.8, body_fx=3e-5),
               capsules=[], conc=None),
    "bgk_small": dict(spec=dict(nx=64, ny=20, collision=O.BGK, tau=0.8, body_fx=3e-5),
                      capsules=[], conc=None),
    "mrt_small": dict(spec=dict(nx=64, ny=20, collision=O.MRT, tau=0.8, body_fx=3e-5),
                      capsules=[], conc=None),
    "reg_small": dict(spec=dict(nx=64, ny=20, collision=O.REGULARIZED, tau=1.2, body_fx=3e-5),
                      capsules=[], conc=None),
    # config 1: 30 Skalak capsules placed from seed 42, 5 MDF sweeps
    "c1": dict(spec=dict(nx=400, ny=80, collision=O.REGULARIZED, tau=0.8, body_fx=3e-5,
                         ibm_iterations=5),
               capsules=[("random", 30, 20, 10, 380, 70, 3.0, 3.0, 24, SKALAK_C1, 42, 1.0, True)],
               conc=None),
    "c1_plain": dict(spec=dict(nx=400, ny=80, collision=O.REGULARIZED, tau=0.8, body_fx=3e-5,
                               ibm_iterations=1),
                     capsules=[("random", 30, 20, 10, 380, 70, 3.0, 3.0, 24, SKALAK_C1, 42,
                                1.0, True)],
                     conc=None),
    # one capsule, no contact, across the periodic seam
    "seam_single": dict(spec=dict(nx=64, ny=32, collision=O.BGK, tau=0.8, body_fx=2e-5,
                                  ibm_iterations=3),
                        capsules=[("add", 1.5, 15.3, 5.0, 32,
                                   dict(model=O.NEO_HOOKEAN, G_s=0.05))],
                        conc=None),
    # a channel narrower than one 32-wide force tile: the stencil of a capsule
    # across the seam covers columns 8, 9, 0, 1 of the same tile
    "narrow_seam": dict(spec=dict(nx=10, ny=24, collision=O.BGK, tau=0.8, body_fx=2e-5,
                                  ibm_iterations=3),
                        capsules=[("add", 0.7, 11.6, 2.0, 12,
                                   dict(model=O.NEO_HOOKEAN, G_s=0.05))],
                        conc=None),
    # config 2 in miniature: MRT, WLC + Helfrich and Skalak, scalar transport
    "mini_c2": dict(spec=dict(nx=128, ny=64, collision=O.MRT, tau=0.8, body_fx=1e-5,
                              scalar_enabled=1, scalar_D=0.05),
                    capsules=[("random", 6, 0, 8, 128, 56, 6.0, 6.0, 48, WLC_HELF, 11, 1.0, True),
                              ("random", 6, 0, 8, 128, 56, 3.0, 3.0, 24, SKALAK_C1, 12, 1.0, True)],
                    conc=gaussian_conc(64.0, 31.5, 20.0)),
    # two capsules in contact, fewer than 100 markers (all-pairs contact),
    # with normal damping and Coulomb friction
    "contact_brute": dict(spec=dict(nx=40, ny=40, collision=O.BGK, tau=0.8, body_fx=1e-5,
                                    rep_damping_normal=0.1, rep_friction=0.2),
                          capsules=[("add", 10.0, 20.0, 4.0, 0, dict(model=O.HOOKEAN)),
                                    ("add", 19.5, 21.0, 4.0, 0, dict(model=O.NEO_HOOKEAN))],
                          conc=None),
    # Zou-He velocity inlet / pressure outlet channels (the reference's
    # default BoundaryType::INLET_OUTLET), no body force
    "zouhe_bgk": dict(spec=dict(nx=64, ny=20, collision=O.BGK, tau=0.8,
                                boundary_type=O.INLET_OUTLET, inlet_velocity=0.03,
                                outlet_density=1.0),
                      capsules=[], conc=None),
    "zouhe_mrt": dict(spec=dict(nx=48, ny=26, collision=O.MRT, tau=0.7,
                                boundary_type=O.INLET_OUTLET, inlet_velocity=0.02,
                                outlet_density=0.995, body_fx=1e-6),
                      capsules=[], conc=None),
    "zouhe_reg": dict(spec=dict(nx=40, ny=18, collision=O.REGULARIZED, tau=0.9,
                                boundary_type=O.INLET_OUTLET, inlet_velocity=0.04,
                                outlet_density=1.0, bottom_wall_velocity=0.01),
                      capsules=[], conc=None),
    # lid-driven cavity: closed box, moving top wall
    "cavity": dict(spec=dict(nx=32, ny=32, collision=O.BGK, tau=0.7,
                             boundary_type=O.CLOSED, top_wall_velocity=0.05),
                   capsules=[], conc=None),
    # pillars (ChannelBuilder): flow past a cylinder and a rectangle in a
    # periodic channel and in a Zou-He channel, halfway and interpolated
    # (Bouzidi) bounce-back
    "pillars_bb": dict(spec=dict(nx=80, ny=30, collision=O.BGK, tau=0.8, body_fx=2e-5),
                       capsules=[], conc=None,
                       pillars=[("circle", 20.3, 14.6, 5.2), ("rect", 50.0, 8.0, 58.5, 20.0)]),
    "pillars_ibb": dict(spec=dict(nx=80, ny=30, collision=O.REGULARIZED, tau=0.8, body_fx=2e-5,
                                  use_interpolated_bb=1),
                        capsules=[], conc=None,
                        pillars=[("circle", 20.3, 14.6, 5.2), ("rect", 50.0, 8.0, 58.5, 20.0)]),
    "pillars_zouhe": dict(spec=dict(nx=72, ny=28, collision=O.MRT, tau=0.7,
                                    boundary_type=O.INLET_OUTLET, inlet_velocity=0.03,
                                    use_interpolated_bb=1),
                          capsules=[], conc=None,
                          pillars=[("circle", 24.0, 13.3, 4.7), ("circle", 45.5, 9.0, 3.1)]),
    # capsules among pillars: one capsule inside the contact range of a
    # cylinder, one above a rectangle, three more placed at random with the
    # pillars rejected (simulation.cpp:256-261); obstacle repulsion with
    # normal damping and Coulomb friction (repulsion.cpp:180-235)
    "pillars_capsules": dict(spec=dict(nx=80, ny=30, collision=O.BGK, tau=0.8, body_fx=2e-5,
                                       rep_damping_normal=0.1, rep_friction=0.2),
                             pillars=[("circle", 40.0, 15.0, 5.0), ("rect", 55.0, 3.0, 62.0, 11.0)],
                             capsules=[("add", 30.5, 15.2, 4.0, 24, SKALAK_C1),
                                       ("add", 58.5, 16.0, 4.0, 24, SKALAK_C1),
                                       ("random", 3, 0, 5, 80, 25, 3.0, 3.0, 24, SKALAK_C1, 7,
                                        1.0, True)],
                             conc=None),
    # the same with interpolated bounce-back, regularized collision and
    # three direct-forcing sweeps
    "pillars_capsules_mdf": dict(spec=dict(nx=80, ny=30, collision=O.REGULARIZED, tau=0.8,
                                           body_fx=2e-5, use_interpolated_bb=1,
                                           ibm_iterations=3),
                                 pillars=[("circle", 40.0, 15.0, 5.0),
                                          ("rect", 55.0, 3.0, 62.0, 11.0)],
                                 capsules=[("add", 30.5, 15.2, 4.0, 24, SKALAK_C1),
                                           ("add", 58.5, 16.0, 4.0, 24, SKALAK_C1)],
                                 conc=None),
    # capsules that reach into both pillars at the start: the nodes inside
    # get the push-out branch of the obstacle repulsion
    "pillars_overlap": dict(spec=dict(nx=80, ny=30, collision=O.BGK, tau=0.8, body_fx=2e-5),
                            pillars=[("circle", 40.0, 15.0, 5.0), ("rect", 55.0, 3.0, 62.0, 11.0)],
                            capsules=[("add", 40.0, 22.5, 3.0, 20, SKALAK_C1),
                                      ("add", 58.5, 13.5, 3.0, 20, SKALAK_C1)],
                            conc=None),
    # plane Couette flow with a capsule (periodic x, walls moving apart)
    "shear_capsule": dict(spec=dict(nx=64, ny=34, collision=O.BGK, tau=0.8,
                                    top_wall_velocity=0.01, bottom_wall_velocity=-0.01,
                                    ibm_iterations=3),
                          capsules=[("add", 32.0, 17.0, 6.0, 36,
                                     dict(model=O.SKALAK, G_s=0.05, C_skalak=10.0))],
                          conc=None),
    # capsule chemistry of the scalar: constant release / absorption at the
    # nearest node, and Fick leaching from finite reservoirs with Langmuir
    # adsorption; capsules of two types, two of them close enough for their
    # stencils to overlap (the reference applies capsules in order); contact
    # strength 0 keeps the FP64 runs free of the device pow's last-ulp
    # differences
    "chem_source": dict(spec=dict(nx=96, ny=48, collision=O.BGK, tau=0.8, body_fx=1e-5,
                                  scalar_enabled=1, scalar_D=0.05, rep_epsilon=0.0),
                        capsules=[("add", 30.0, 20.0, 4.0, 24, SKALAK_C1, 0),
                                  ("add", 39.2, 21.0, 4.0, 24, SKALAK_C1, 1),
                                  ("add", 70.0, 30.0, 5.0, 32, SKALAK_C1, 0)],
                        conc=gaussian_conc(48.0, 24.0, 12.0),
                        chem=dict(release=[0.002, 0.0], absorb=[0.0, 0.001])),
    "chem_physics": dict(spec=dict(nx=96, ny=48, collision=O.BGK, tau=0.8, body_fx=1e-5,
                                   scalar_enabled=1, scalar_D=0.05, rep_epsilon=0.0),
                         capsules=[("add", 30.0, 20.0, 4.0, 24, SKALAK_C1, 0),
                                   ("add", 39.2, 21.0, 4.0, 24, SKALAK_C1, 1),
                                   ("add", 70.0, 30.0, 5.0, 32, SKALAK_C1, 0)],
                         conc=gaussian_conc(48.0, 24.0, 12.0),
                         chem=dict(k_leach=[0.05, 0.0], C_eq=[1.0, 0.0],
                                   M_p_initial=[0.02, 0.0], k_adsorb=[0.0, 0.02],
                                   k_desorb=[0.0, 0.001], Gamma_max=[1.0, 0.5],
                                   release=[0.0, 0.0005])),
    # pure diffusion (reference tests/verification/test_pure_diffusion.cpp)
    "diffusion": dict(spec=dict(nx=256, ny=8, collision=O.BGK, tau=0.6, periodic_y=1,
                                scalar_enabled=1, scalar_D=0.05, scalar_periodic_y=1),
                      capsules=[], conc=None),
}


def build_oracle(case, impl="sfo"):
    s = O.OracleSim(O.ChannelSpec(**case["spec"]), impl)
    for ob in case.get("pillars", []):
        if ob[0] == "circle":
            s.add_circle_pillar(*ob[1:])
        else:
            s.add_rect_pillar(*ob[1:])
    for c in case["capsules"]:
        if c[0] == "add":
            _, cx, cy, r, nn, mk = c[:6]
            s.add_capsule(cx, cy, r, nn, O.Membrane(**mk), c[6] if len(c) > 6 else 0)
        else:
            _, count, x0, y0, x1, y1, rmin, rmax, nn, mk, seed, gap, walls = c
            s.add_capsule_random(count, x0, y0, x1, y1, rmin, rmax, nn, O.Membrane(**mk),
                                 seed=seed, min_gap=gap, check_walls=walls)
    if case.get("chem"):
        s.set_chemistry(**case["chem"])
    s.initialize()
    if case["conc"] is not None:
        sp = case["spec"]
        s.set_concentration(case["conc"](sp["nx"], sp["ny"]))
    return s


def gpu_params(case, precision):
    import softflow_b200 as S
    sp = dict(O.ChannelSpec(**case["spec"]).__dict__)
    p = S.SimulationParams()
    p.nx, p.ny = sp["nx"], sp["ny"]
    p.dt = sp["dt"]
    p.ibm_iterations = sp["ibm_iterations"]
    p.max_lattice_force = sp["max_lattice_force"]
    p.fluid.boundary_type = S.BoundaryType(sp["boundary_type"])
    p.fluid.inlet_velocity, p.fluid.outlet_density = sp["inlet_velocity"], sp["outlet_density"]
    p.fluid.top_wall_velocity = sp["top_wall_velocity"]
    p.fluid.bottom_wall_velocity = sp["bottom_wall_velocity"]
    p.fluid.use_interpolated_bb = bool(sp["use_interpolated_bb"])
    p.fluid.tau, p.fluid.rho0 = sp["tau"], sp["rho0"]
    p.fluid.collision_model = S.CollisionModel(sp["collision"])
    p.fluid.mrt_se, p.fluid.mrt_s_eps, p.fluid.mrt_sq = sp["mrt_se"], sp["mrt_s_eps"], sp["mrt_sq"]
    p.fluid.body_force_x, p.fluid.body_force_y = sp["body_fx"], sp["body_fy"]
    p.fluid.periodic_y = bool(sp["periodic_y"])
    p.repulsion.epsilon, p.repulsion.sigma = sp["rep_epsilon"], sp["rep_sigma"]
    p.repulsion.r_cut, p.repulsion.power = sp["rep_r_cut"], sp["rep_power"]
    p.repulsion.damping_normal = sp["rep_damping_normal"]
    p.repulsion.friction_coeff = sp["rep_friction"]
    p.scalar.enabled = bool(sp["scalar_enabled"])
    p.scalar.diffusivity = [sp["scalar_D"]]
    p.scalar.periodic_y = bool(sp["scalar_periodic_y"])
    p.scalar.inlet_concentration = [sp["scalar_inlet"]]
    for k in ("k_leach", "C_eq", "M_p_initial", "k_adsorb", "k_desorb", "Gamma_max"):
        setattr(p.scalar, k, list((case.get("chem") or {}).get(k, [])))
    p.precision = precision
    return p


def gpu_membrane(mk):
    import softflow_b200 as S
    m = O.Membrane(**mk)
    return S.MembraneParams(
        model=S.MembraneModel(m.model), k_stretch=m.k_stretch, G_s=m.G_s, C_skalak=m.C_skalak,
        wlc_L_max_ratio=m.wlc_L_max_ratio, wlc_kBT_p=m.wlc_kBT_p, wlc_k_pow=m.wlc_k_pow,
        k_bend=m.k_bend, use_helfrich_bending=bool(m.use_helfrich), kappa_0=m.kappa_0,
        k_area=m.k_area, k_perimeter=m.k_perimeter, gamma_visc=m.gamma_visc,
        eta_membrane=m.eta_membrane)


def add_case_capsules(ens, chan, case):
    import softflow_b200 as S
    for c in case["capsules"]:
        if c[0] == "add":
            _, cx, cy, r, nn, mk = c[:6]
            S.Ensemble.addCapsule(ens, chan, (cx, cy), r, nn, gpu_membrane(mk),
                                  c[6] if len(c) > 6 else 0)
        else:
            _, count, x0, y0, x1, y1, rmin, rmax, nn, mk, seed, gap, walls = c
            S.Ensemble.addCapsuleRandom(ens, chan, count, x0, y0, x1, y1, rmin, rmax, nn,
                                        gpu_membrane(mk), seed=seed, min_gap=gap,
                                        check_walls=walls)


def build_gpu(case, precision="fp32"):
    import softflow_b200 as S
    sim = S.Simulation(gpu_params(case, precision))
    if case.get("pillars"):
        sp = case["spec"]
        b = S.ChannelBuilder(sp["nx"], sp["ny"])
        for ob in case["pillars"]:
            if ob[0] == "circle":
                b.addCirclePillar(*ob[1:])
            else:
                b.addRectPillar(*ob[1:])
        sim.setChannelBuilder(b)
    add_case_capsules(sim, 0, case)
    chem = case.get("chem") or {}
    for t, r in enumerate(chem.get("release", [])):
        sim.setScalarReleaseRate(t, r)
    for t, r in enumerate(chem.get("absorb", [])):
        sim.setScalarAbsorptionRate(t, r)
    sim.initialize()
    if case["conc"] is not None:
        sp = case["spec"]
        sim.advectionDiffusion().setConcentration(case["conc"](sp["nx"], sp["ny"]))
    return sim


def fluid_rows(case):
    sp = case["spec"]
    return slice(0, sp["ny"]) if sp.get("periodic_y") else slice(1, sp["ny"] - 1)


def rel_l2(a, b):
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return d / n if n > 0 else d
