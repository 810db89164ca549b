"""Oracle restatements of the reference's reductions of the state (test
infrastructure; the product computes these on the device).

* max_speed: Simulation::getMaxSpeed (src/engine/simulation.cpp:892-907);
* global_stats: GlobalStatsWriter::writeTimestep
  (src/io/global_stats_writer.cpp:41-124), serial row-major sums;
* first_nonfinite: the scan order of Simulation::checkStability
  (src/engine/simulation.cpp:817-845).

Inputs are the reference's macroscopic fields [ny][nx] (rho = u = 0 on SOLID
cells) and a SOLID mask of the same shape.
"""
from __future__ import annotations

import math

import numpy as np


def solid_mask(nx: int, ny: int, periodic_y: bool) -> np.ndarray:
    m = np.zeros((ny, nx), dtype=bool)
    if not periodic_y:
        m[0, :] = True
        m[ny - 1, :] = True
    return m


def max_speed(ux: np.ndarray, uy: np.ndarray, solid: np.ndarray) -> float:
    """simulation.cpp:892-907: sqrt of the largest ux^2 + uy^2 (a NaN never
    replaces the running maximum)."""
    sp = ux * ux + uy * uy
    sp = sp[~solid]
    sp = sp[~np.isnan(sp)]
    m = float(sp.max()) if sp.size else 0.0
    return math.sqrt(max(m, 0.0))


def global_stats(rho, ux, uy, solid, deformations, C=None) -> dict:
    """global_stats_writer.cpp:52-103 with its serial accumulation order."""
    sum_rho = 0.0
    min_rho, max_rho = 1e30, -1e30
    max_v2 = sum_vel = ke = 0.0
    count = 0
    r = rho.ravel().tolist()
    vx = ux.ravel().tolist()
    vy = uy.ravel().tolist()
    sd = solid.ravel().tolist()
    for i in range(len(r)):
        if sd[i]:
            continue
        v2 = vx[i] * vx[i] + vy[i] * vy[i]
        sum_rho += r[i]
        if r[i] < min_rho:
            min_rho = r[i]
        if r[i] > max_rho:
            max_rho = r[i]
        if v2 > max_v2:
            max_v2 = v2
        sum_vel += math.sqrt(v2)
        ke += 0.5 * r[i] * v2
        count += 1
    mean_def = max_def = 0.0
    for D in deformations:
        mean_def += D
        if D > max_def:
            max_def = D
    if len(deformations):
        mean_def /= len(deformations)
    out = {"mean_rho": sum_rho / count if count else 0.0,
           "max_velocity": math.sqrt(max_v2),
           "mean_velocity": sum_vel / count if count else 0.0,
           "total_kinetic_energy": ke, "n_active_particles": len(deformations),
           "mean_deformation": mean_def, "max_deformation": max_def,
           "min_rho": min_rho, "max_rho": max_rho, "fluid_cells": count}
    if C is not None:
        tot = 0.0
        for v in C.ravel().tolist():
            tot += v
        out["total_dissolved_mass"] = tot
    return out


def first_nonfinite(rho, ux, uy, solid) -> int:
    """Row-major index of the first non-SOLID cell whose rho or u is not
    finite (simulation.cpp:829-845), or -1."""
    bad = ~(np.isfinite(rho) & np.isfinite(ux) & np.isfinite(uy)) & ~solid
    idx = np.flatnonzero(bad.ravel())
    return int(idx[0]) if idx.size else -1
