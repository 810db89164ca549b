"""Oracle simulations built from the product's workload plans
(softflow_b200.workloads.ChannelPlan): the same channel parameters, seeded
placements and scalar initial condition, on the C restatement (impl "sfo")
or on the reference's own sources (impl "ref").  Test and baseline
infrastructure only."""
from __future__ import annotations

import contextlib
import io

import numpy as np

from . import ChannelSpec, Membrane, OracleSim


def spec_from_params(params) -> ChannelSpec:
    f = params.fluid
    return ChannelSpec(
        nx=params.nx, ny=params.ny, collision=int(f.collision_model), tau=f.tau, rho0=f.rho0,
        mrt_se=f.mrt_se, mrt_s_eps=f.mrt_s_eps, mrt_sq=f.mrt_sq, body_fx=f.body_force_x,
        body_fy=f.body_force_y, periodic_y=int(f.periodic_y),
        max_lattice_force=params.max_lattice_force, ibm_iterations=params.ibm_iterations,
        dt=params.dt, scalar_enabled=int(params.scalar.enabled),
        scalar_D=params.scalar.diffusivity[0] if params.scalar.diffusivity else 0.01)


def membrane_from_params(mp) -> Membrane:
    return Membrane(model=int(mp.model), k_stretch=mp.k_stretch, G_s=mp.G_s,
                    C_skalak=mp.C_skalak, wlc_L_max_ratio=mp.wlc_L_max_ratio,
                    wlc_kBT_p=mp.wlc_kBT_p, wlc_k_pow=mp.wlc_k_pow, k_bend=mp.k_bend,
                    use_helfrich=int(mp.use_helfrich_bending), kappa_0=mp.kappa_0,
                    k_area=mp.k_area, k_perimeter=mp.k_perimeter,
                    gamma_visc=mp.gamma_visc, eta_membrane=mp.eta_membrane)


def sims_from_plans(plans, impl: str = "sfo", threads: int = 1):
    """One initialized oracle simulation per plan (fast=True for the
    reference's Release build when impl is "ref")."""
    sims = []
    for pl in plans:
        s = OracleSim(spec_from_params(pl.params), impl, fast=(impl == "ref"), threads=threads)
        with contextlib.redirect_stdout(io.StringIO()):
            for (count, x0, y0, x1, y1, r, nodes, mp, seed) in pl.placements:
                s.add_capsule_random(count, x0, y0, x1, y1, r, r, nodes, membrane_from_params(mp),
                                     seed=seed, min_gap=pl.min_gap, check_walls=True)
        s.initialize()
        if pl.gaussian is not None:
            cx, cy, sg = pl.gaussian
            p = pl.params
            y, x = np.mgrid[0:p.ny, 0:p.nx]
            s.set_concentration(np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2.0 * sg * sg)))
        sims.append(s)
    return sims
