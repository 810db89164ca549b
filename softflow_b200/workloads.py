"""Standard workloads of the hot path (synthetic, seeded).

c0  400 x 80 regularized channel, tau 0.8, fx 3e-5, no capsules.
c1  c0 + 30 Skalak capsules (r 3, 24 markers, G_s 0.06, no bending) placed
    from seed 42 in x [20, 380], y [10, 70] with gap 1, 5 MDF sweeps.
c2  4096 x 1024 MRT channel, tau 0.8, fx 1e-5; 1000 WLC capsules with
    Helfrich bending (r 6, 48 markers) placed from seed 11, then 1000 Skalak
    capsules (r 3, 24 markers) from seed 12 (about 3.4 % area fraction);
    scalar with D 0.05 seeded as a unit Gaussian of sigma 20 at the centre.
c3  256 independent channels drawn from seed 7: nx in {200, 208, ..., 800},
    ny in {40, 48, ..., 160}, 5-60 Skalak capsules (r 3, 24 markers),
    G_s log-uniform in [0.01, 0.1], tau uniform in [0.6, 1.0], fx uniform in
    [1e-5, 5e-5]; regularized collision, 5 MDF sweeps.  Channel i places its
    capsules from seed fnv1a64(str(i)) & 0x7fffffff with centres in
    x [8, nx - 8], y [8, ny - 8] and surfaces at least 3.5 lu apart (the
    contact cut-off).

Centres are kept MARGIN = 8 lu from the walls and from the periodic seam
(configuration 1 keeps them 10 lu from the walls and 20 lu from the seam).
The reference placement tests overlap with the plain distance between
centres, without the periodic image, so capsules seeded at both ends of a
channel can overlap across the seam; capsules seeded against a wall have
nodes inside the y-clamp band.  With multi-direct forcing the reference
algorithm diverges within a few steps on channels seeded either way.

Membrane constants not fixed by the configuration use the reference Python
API defaults (C_skalak 10, k_area 0.5, k_perimeter 0.1, gamma 0.01,
eta 0.05; Helfrich k_bend 0.005).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Tuple

import numpy as np

from .engine import (BoundaryType, CollisionModel, Ensemble, MembraneModel, MembraneParams,
                     SimulationParams)


def fnv1a64(s: str, seed: int = 0) -> int:
    """FNV-1a 64-bit (the reference's seed derivation, simulation.cpp:284-291)."""
    h = (seed ^ 0xcbf29ce484222325) & 0xFFFFFFFFFFFFFFFF
    for ch in s.encode():
        h ^= ch
        h = (h * 0x100000001b3) & 0xFFFFFFFFFFFFFFFF
    return h if h else 0x9e3779b97f4a7c15


def skalak(G_s=0.06, k_bend=0.0) -> MembraneParams:
    return MembraneParams(model=MembraneModel.SKALAK, G_s=G_s, C_skalak=10.0, k_bend=k_bend)


def wlc_helfrich(G_s=0.06, k_bend=0.005) -> MembraneParams:
    return MembraneParams(model=MembraneModel.WLC, G_s=G_s, k_bend=k_bend,
                          use_helfrich_bending=True)


def channel_params(nx, ny, collision, tau, fx, ibm_iterations=1, precision="fp32",
                   scalar_D=None) -> SimulationParams:
    p = SimulationParams(nx=nx, ny=ny, ibm_iterations=ibm_iterations, precision=precision)
    p.fluid.boundary_type = BoundaryType.PERIODIC
    p.fluid.collision_model = collision
    p.fluid.tau = tau
    p.fluid.body_force_x = fx
    if scalar_D is not None:
        p.scalar.enabled = True
        p.scalar.diffusivity = [scalar_D]
    return p


@dataclass
class ChannelPlan:
    params: SimulationParams
    # (count, x0, y0, x1, y1, r, nodes, membrane, seed)
    placements: List[Tuple] = field(default_factory=list)
    min_gap: float = 1.0       # surface gap of the rejection test (lu)
    gaussian: Tuple = None     # (cx, cy, sigma) for the scalar


def plan_c0(precision="fp32") -> List[ChannelPlan]:
    return [ChannelPlan(channel_params(400, 80, CollisionModel.REGULARIZED, 0.8, 3e-5,
                                       1, precision))]


def plan_c1(precision="fp32") -> List[ChannelPlan]:
    p = channel_params(400, 80, CollisionModel.REGULARIZED, 0.8, 3e-5, 5, precision)
    return [ChannelPlan(p, [(30, 20, 10, 380, 70, 3.0, 24, skalak(), 42)])]


MARGIN = 8
# c3 rejects placements whose surfaces come closer than the contact cut-off
# (3.5 lu): capsules seeded 1 lu apart start inside each other's repulsion
# range, the spread contact forces exceed the 0.01 lattice-force cap, and
# with 5 MDF sweeps the flow diverges within a few hundred steps.
C3_MIN_GAP = 3.5


def plan_c2(precision="fp32") -> List[ChannelPlan]:
    p = channel_params(4096, 1024, CollisionModel.MRT, 0.8, 1e-5, 1, precision, scalar_D=0.05)
    m = MARGIN
    return [ChannelPlan(p, [(1000, m, m, 4096 - m, 1024 - m, 6.0, 48, wlc_helfrich(), 11),
                            (1000, m, m, 4096 - m, 1024 - m, 3.0, 24, skalak(), 12)],
                        gaussian=(2048.0, 511.5, 20.0))]


def plan_c2_lattice(precision="fp32") -> List[ChannelPlan]:
    """Configuration 2's fluid alone (4096 x 1024 MRT, tau 0.8, fx 1e-5, no
    capsules, no scalar): the plain stream-collide of the roofline target."""
    return [ChannelPlan(channel_params(4096, 1024, CollisionModel.MRT, 0.8, 1e-5, 1, precision))]


def plan_c3(precision="fp32", n_channels=256, ibm_iterations=5) -> List[ChannelPlan]:
    rng = np.random.default_rng(7)
    plans = []
    for i in range(n_channels):
        nx = int(rng.integers(25, 101)) * 8
        ny = int(rng.integers(5, 21)) * 8
        ncap = int(rng.integers(5, 61))
        G_s = float(10.0 ** rng.uniform(-2.0, -1.0))
        tau = float(rng.uniform(0.6, 1.0))
        fx = float(rng.uniform(1e-5, 5e-5))
        p = channel_params(nx, ny, CollisionModel.REGULARIZED, tau, fx, ibm_iterations, precision)
        seed = fnv1a64(str(i)) & 0x7FFFFFFF
        m = MARGIN
        plans.append(ChannelPlan(p, [(ncap, m, m, nx - m, ny - m, 3.0, 24, skalak(G_s), seed)],
                                 min_gap=C3_MIN_GAP))
    return plans


PLANS = {"c0": plan_c0, "c1": plan_c1, "c2": plan_c2, "c2_lattice": plan_c2_lattice,
         "c3": plan_c3}


def build(plans: List[ChannelPlan], precision: str = None, device: int = 0,
          verbose: bool = False) -> Ensemble:
    """Creates an initialized ensemble holding every planned channel."""
    prec = precision or plans[0].params.precision
    ens = Ensemble(precision=prec, device=device)
    import contextlib
    import io
    for i, pl in enumerate(plans):
        pl.params.precision = prec
        ens.add_channel(pl.params)
        for (count, x0, y0, x1, y1, r, nodes, mp, seed) in pl.placements:
            sink = contextlib.nullcontext() if verbose else contextlib.redirect_stdout(io.StringIO())
            with sink:
                ens.addCapsuleRandom(i, count, x0, y0, x1, y1, r, r, nodes, mp, seed=seed,
                                     min_gap=pl.min_gap, check_walls=True)
    ens.initialize()
    for i, pl in enumerate(plans):
        if pl.gaussian is not None:
            cx, cy, sg = pl.gaussian
            p = pl.params
            y, x = np.mgrid[0:p.ny, 0:p.nx]
            ens.advectionDiffusion(i).setConcentration(
                np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2.0 * sg * sg)))
    return ens


def totals(plans: List[ChannelPlan], ens: Ensemble = None):
    """(fluid cells, capsules, markers, scalar cells) over all channels."""
    cells = caps = markers = scal = 0
    for i, pl in enumerate(plans):
        p = pl.params
        rows = p.ny if p.fluid.periodic_y else p.ny - 2
        cells += p.nx * rows
        if p.scalar.enabled:
            scal += p.nx * rows
        if ens is not None:
            c = ens._chans[i].caps
            caps += len(c)
            markers += sum(r.rest.num_nodes for r in c)
    return cells, caps, markers, scal
