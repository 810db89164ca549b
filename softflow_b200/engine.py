"""Host mirror of the reference engine API on top of the C ABI.

Names, argument meanings and defaults follow the reference's pybind11
module ``softflow_core`` (python/bindings.cpp:128-307 for the parameter
structs, :846-981 for ``Simulation``), so a script written against the
reference's core API runs here unchanged for the hot-path features:

    p = SimulationParams(); p.nx, p.ny = 400, 80
    p.fluid.boundary_type = BoundaryType.PERIODIC
    p.fluid.collision_model = CollisionModel.REGULARIZED
    sim = Simulation(p)
    sim.addCapsuleRandom(30, 20, 10, 380, 70, 3, 3, 24, mp, seed=42)
    sim.initialize(); sim.run(1000)
    ux = sim.field().velocity_x()

``Ensemble`` runs many independent channels in one device context: every
step is one launch per kernel phase over all channels.

All numerical work of a step runs in libsoftflow_b200.so on the GPU.  The
host side only builds rest geometry at setup and moves data on request.
"""
from __future__ import annotations

import ctypes as C
import enum
import math
import os
import sys
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _lib as L

PI = 3.14159265358979323846


class CollisionModel(enum.IntEnum):
    BGK = 0
    MRT = 1
    REGULARIZED = 2


class MembraneModel(enum.IntEnum):
    HOOKEAN = 0
    NEO_HOOKEAN = 1
    SKALAK = 2
    WLC = 3


class BoundaryType(enum.IntEnum):
    INLET_OUTLET = 0
    PERIODIC = 1
    CLOSED = 2


class CapsuleShape(enum.IntEnum):
    CIRCLE = 0
    ELLIPSE = 1
    BICONCAVE = 2
    FIBER = 3


@dataclass
class FluidParams:
    """Reference FluidParams (parameters.h:41-79), hot-path fields."""
    tau: float = 0.8
    rho0: float = 1.0
    boundary_type: BoundaryType = BoundaryType.INLET_OUTLET
    body_force_x: float = 0.0
    body_force_y: float = 0.0
    collision_model: CollisionModel = CollisionModel.BGK
    use_mrt: bool = False
    mrt_se: float = 1.4
    mrt_s_eps: float = 1.4
    mrt_sq: float = 1.4
    periodic_y: bool = False
    inlet_velocity: float = 0.02
    outlet_density: float = 1.0
    top_wall_velocity: float = 0.0
    bottom_wall_velocity: float = 0.0
    use_interpolated_bb: bool = False


@dataclass
class MembraneParams:
    """Reference MembraneParams (parameters.h:82-136)."""
    model: MembraneModel = MembraneModel.HOOKEAN
    k_stretch: float = 0.1
    G_s: float = 0.1
    C_skalak: float = 1.0
    wlc_L_max_ratio: float = 2.2
    wlc_kBT_p: float = 0.0
    wlc_k_pow: float = 0.0
    k_bend: float = 0.005
    use_helfrich_bending: bool = False
    kappa_0: float = 0.0
    k_area: float = 0.5
    k_perimeter: float = 0.1
    gamma_visc: float = 0.01
    eta_membrane: float = 0.05
    shape: CapsuleShape = CapsuleShape.CIRCLE
    is_rigid: bool = False
    density: float = 1.0

    def to_c(self) -> L.MembraneParamsC:
        if self.shape != CapsuleShape.CIRCLE:
            raise NotImplementedError("only circular rest shapes are on this path")
        if self.is_rigid:
            raise NotImplementedError("rigid capsules are not on this path")
        return L.MembraneParamsC(
            model=int(self.model), k_stretch=self.k_stretch, G_s=self.G_s,
            C_skalak=self.C_skalak, wlc_L_max_ratio=self.wlc_L_max_ratio,
            wlc_kBT_p=self.wlc_kBT_p, wlc_k_pow=self.wlc_k_pow, k_bend=self.k_bend,
            use_helfrich=int(bool(self.use_helfrich_bending)), kappa_0=self.kappa_0,
            k_area=self.k_area, k_perimeter=self.k_perimeter, gamma_visc=self.gamma_visc,
            eta_membrane=self.eta_membrane)


@dataclass
class RepulsionParams:
    """Reference RepulsionParams (parameters.h:138-161)."""
    epsilon: float = 0.05
    sigma: float = 1.0
    r_cut: float = 3.5
    power: int = 4
    damping_normal: float = 0.0
    friction_coeff: float = 0.0


@dataclass
class ScalarParams:
    """Reference ScalarParams (parameters.h:177-205), one species."""
    enabled: bool = False
    n_species: int = 1
    diffusivity: List[float] = field(default_factory=lambda: [0.01])
    inlet_concentration: List[float] = field(default_factory=lambda: [0.0])
    periodic_y: bool = False
    # capsule chemistry kinetics per capsule type (parameters.h:214-228);
    # empty vectors select the constant release / absorption rates
    k_leach: List[float] = field(default_factory=list)
    C_eq: List[float] = field(default_factory=list)
    M_p_initial: List[float] = field(default_factory=list)
    k_adsorb: List[float] = field(default_factory=list)
    k_desorb: List[float] = field(default_factory=list)
    Gamma_max: List[float] = field(default_factory=list)


@dataclass
class SimulationParams:
    """Reference SimulationParams (parameters.h:279-342), hot-path fields,
    plus the device options ``precision`` ("fp64" | "fp32" | "fp16s") and
    ``device``."""
    nx: int = 200
    ny: int = 50
    dt: float = 1.0
    ibm_iterations: int = 1
    max_lattice_force: float = 0.01
    fluid: FluidParams = field(default_factory=FluidParams)
    membrane: MembraneParams = field(default_factory=MembraneParams)
    repulsion: RepulsionParams = field(default_factory=RepulsionParams)
    scalar: ScalarParams = field(default_factory=ScalarParams)
    # output (parameters.h:302-313).  output_dir None writes no files (the
    # reference's default is "output"); set it to get the reference's
    # per-step output schedule in run().
    output_dir: Optional[str] = None
    output_interval: int = 100
    vtk_dump_every: int = 0
    csv_dump_every: int = 0
    probe_dump_every: int = 10
    stats_dump_every: int = 100
    checkpoint_interval: int = 0
    vtk_format: str = "ascii"
    probes: List[tuple] = field(default_factory=list)
    # stability monitoring (parameters.h:315-319)
    enable_stability_checks: bool = True
    max_density_deviation: float = 0.1
    max_velocity: float = 0.1
    stability_check_interval: int = 1000
    precision: str = "fp32"
    device: int = 0

    def kinematicViscosity(self) -> float:
        return (self.fluid.tau - 0.5) / 3.0

    def to_c(self) -> L.ChannelParamsC:
        f = self.fluid
        coll = CollisionModel.MRT if f.use_mrt else CollisionModel(f.collision_model)
        if self.scalar.enabled and self.scalar.n_species != 1:
            raise NotImplementedError("one scalar species is supported")
        return L.ChannelParamsC(
            nx=self.nx, ny=self.ny, collision=int(coll), tau=f.tau, rho0=f.rho0,
            mrt_se=f.mrt_se, mrt_s_eps=f.mrt_s_eps, mrt_sq=f.mrt_sq,
            body_fx=f.body_force_x, body_fy=f.body_force_y, periodic_y=int(bool(f.periodic_y)),
            max_lattice_force=self.max_lattice_force, ibm_iterations=self.ibm_iterations,
            dt=self.dt, rep_epsilon=self.repulsion.epsilon, rep_sigma=self.repulsion.sigma,
            rep_r_cut=self.repulsion.r_cut, rep_power=self.repulsion.power,
            rep_damping_normal=self.repulsion.damping_normal,
            rep_friction=self.repulsion.friction_coeff,
            scalar_enabled=int(bool(self.scalar.enabled)),
            scalar_D=(self.scalar.diffusivity[0] if self.scalar.diffusivity else 0.01),
            scalar_periodic_y=int(bool(self.scalar.periodic_y)),
            scalar_inlet=(self.scalar.inlet_concentration[0]
                          if self.scalar.inlet_concentration else 0.0),
            boundary_type=int(f.boundary_type), inlet_velocity=f.inlet_velocity,
            outlet_density=f.outlet_density, top_wall_velocity=f.top_wall_velocity,
            bottom_wall_velocity=f.bottom_wall_velocity,
            use_interpolated_bb=int(bool(f.use_interpolated_bb)))


@dataclass
class _CapsuleRec:
    mp: MembraneParams
    rest: L.CapsuleRestC
    pos: np.ndarray
    rest_len: np.ndarray
    rest_ang: np.ndarray
    rest_ds: np.ndarray
    type_id: int


def build_circle_capsule(center, radius: float, num_nodes: int, mp: MembraneParams):
    """Rest geometry of a circular capsule (reference capsule.cpp:7-141)."""
    lib = L.lib()
    mpc = mp.to_c()
    rest = L.CapsuleRestC()
    L.check(lib.sfg_build_circle_capsule(float(center[0]), float(center[1]), float(radius),
                                         int(num_nodes), C.byref(mpc), C.byref(rest),
                                         None, None, None, None, 0))
    n = rest.num_nodes
    pos = np.zeros(2 * n)
    rl, ra, rd = np.zeros(n), np.zeros(n), np.zeros(n)
    L.check(lib.sfg_build_circle_capsule(float(center[0]), float(center[1]), float(radius),
                                         int(num_nodes), C.byref(mpc), C.byref(rest),
                                         L.dptr(pos), L.dptr(rl), L.dptr(ra), L.dptr(rd), n))
    return rest, pos, rl, ra, rd


def _centroid_periodic(pos: np.ndarray, nx: int):
    """Capsule::centroid with minimum image (capsule.cpp:159-173), evaluated
    sequentially in IEEE double like the reference."""
    p = pos.reshape(-1, 2)
    Lx = float(nx)
    rx, ry = float(p[0, 0]), float(p[0, 1])
    sx, sy = rx, ry
    for i in range(1, len(p)):
        dx = float(p[i, 0]) - rx
        dy = float(p[i, 1]) - ry
        if dx > 0.5 * Lx:
            dx -= Lx
        if dx < -0.5 * Lx:
            dx += Lx
        sx = sx + (rx + dx)
        sy = sy + (ry + dy)
    n = float(len(p))
    return sx / n, sy / n


class ChannelBuilder:
    """Channel geometry (reference ChannelBuilder, geometry/channel_builder.h:
    14-62; bindings.cpp:634-654): circular and rectangular pillars.  Walls
    and the boundary type come from the simulation parameters, as the
    reference's LBMSolver::initialize re-applies them."""

    def __init__(self, nx: int, ny: int):
        self.nx, self.ny = int(nx), int(ny)
        self.pillars: List[tuple] = []
        self._walls = False
        self._bt = BoundaryType.INLET_OUTLET

    def addWalls(self):
        self._walls = True
        return self

    def addCirclePillar(self, cx: float, cy: float, radius: float):
        self.pillars.append((0, float(cx), float(cy), float(radius), 0.0))
        return self

    def addRectPillar(self, x0: float, y0: float, x1: float, y1: float):
        self.pillars.append((1, float(x0), float(y0), float(x1), float(y1)))
        return self

    def setBoundaryType(self, bt):
        self._bt = BoundaryType(bt)
        return self

    def getBoundaryType(self):
        return self._bt

    def hasTopWall(self):
        return self._walls

    def hasBottomWall(self):
        return self._walls

    def getNx(self):
        return self.nx

    def getNy(self):
        return self.ny

    def wallBottom(self):
        return 0.0

    def wallTop(self):
        return float(self.ny - 1)


class _Channel:
    def __init__(self, params: SimulationParams):
        self.params = params
        self.cparams = params.to_c()
        self.caps: List[_CapsuleRec] = []
        self.pillars: List[tuple] = []
        self.walls_in_placement = False
        self.release_rates: List[float] = []
        self.absorption_rates: List[float] = []

    def chemistry(self) -> Optional[L.ChemistryC]:
        """sfg_chemistry of the channel, or None when no vector is set
        (Simulation::step then runs no chemistry, simulation.cpp:640-653)."""
        sc = self.params.scalar
        vecs = {"release": self.release_rates, "absorb": self.absorption_rates,
                "k_leach": sc.k_leach, "C_eq": sc.C_eq, "M_p_initial": sc.M_p_initial,
                "k_adsorb": sc.k_adsorb, "k_desorb": sc.k_desorb, "Gamma_max": sc.Gamma_max}
        if not any(len(v) for v in vecs.values()):
            return None
        counts = {"release": "n_release", "absorb": "n_absorb", "k_leach": "n_k_leach",
                  "C_eq": "n_C_eq", "M_p_initial": "n_M_p", "k_adsorb": "n_k_adsorb",
                  "k_desorb": "n_k_desorb", "Gamma_max": "n_Gamma_max"}
        c = L.ChemistryC()
        for k, v in vecs.items():
            if len(v) > 8:
                raise ValueError(f"at most 8 capsule types ({k})")
            setattr(c, counts[k], len(v))
            arr = getattr(c, k)
            for i, x in enumerate(v):
                arr[i] = float(x)
        return c

    def add_capsule(self, center, radius, num_nodes=0, mparams=None, type_id=0):
        mp = mparams if mparams is not None else self.params.membrane
        rest, pos, rl, ra, rd = build_circle_capsule(center, radius, num_nodes, mp)
        self.caps.append(_CapsuleRec(mp, rest, pos, rl, ra, rd, type_id))
        return len(self.caps) - 1

    def add_random(self, count, x0, y0, x1, y1, rmin, rmax, num_nodes, mparams, type_id, seed,
                   min_gap, max_attempts, check_walls):
        n_ex = len(self.caps)
        cen = np.zeros(2 * max(n_ex, 1))
        rad = np.zeros(max(n_ex, 1))
        for i, c in enumerate(self.caps):
            cx, cy = _centroid_periodic(c.pos, self.params.nx)
            cen[2 * i], cen[2 * i + 1] = cx, cy
            rad[i] = math.sqrt(c.rest.rest_area / PI)
        out_c = np.zeros(2 * max(count, 1))
        out_r = np.zeros(max(count, 1))
        placed, attempts = C.c_int(0), C.c_int(0)
        pl = np.array([x for o in self.pillars for x in o], dtype=np.float64)
        L.check(L.lib().sfg_place_random_pillars(
            int(count), float(x0), float(y0), float(x1), float(y1), float(rmin), float(rmax),
            int(num_nodes), int(seed), float(min_gap), int(max_attempts), int(bool(check_walls)),
            int(self.params.nx), int(self.params.ny), n_ex, L.dptr(cen), L.dptr(rad),
            int(count), L.dptr(out_c), L.dptr(out_r), C.byref(placed), C.byref(attempts),
            len(self.pillars), L.dptr(pl) if len(self.pillars) else None))
        for i in range(placed.value):
            self.add_capsule((out_c[2 * i], out_c[2 * i + 1]), out_r[i], num_nodes, mparams,
                             type_id)
        print(f"Placed {placed.value}/{count} capsules ({attempts.value} attempts)")
        return placed.value


class _Context:
    """One device context holding one or more channels."""

    def __init__(self, channels: Sequence[_Channel], precision: str, device: int,
                 lattice_variant: int = 0):
        if precision not in L.PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(L.PRECISIONS)}")
        lib = L.lib()
        self._lib = lib
        self.precision = precision
        self.num_channels = len(channels)
        self.num_capsules = sum(len(ch.caps) for ch in channels)
        self._version = 0
        self._thermo_cache = None
        h = C.c_void_p()
        L.check(lib.sfg_create(int(device), L.PRECISIONS[precision], C.byref(h)))
        self._h = h
        try:
            L.check(lib.sfg_set_lattice_variant(h, int(lattice_variant)))
            for ch in channels:
                idx = C.c_int()
                L.check(lib.sfg_add_channel(h, C.byref(ch.cparams), C.byref(idx)))
                for pl in ch.pillars:
                    L.check(lib.sfg_add_pillar(h, idx.value, *pl))
                for rec in ch.caps:
                    mpc = rec.mp.to_c()
                    L.check(lib.sfg_add_capsule(h, idx.value, C.byref(mpc), C.byref(rec.rest),
                                                L.dptr(rec.pos), L.dptr(rec.rest_len),
                                                L.dptr(rec.rest_ang), L.dptr(rec.rest_ds), None))
                for k, rec in enumerate(ch.caps):
                    if rec.type_id:
                        L.check(lib.sfg_set_capsule_type(h, idx.value, k, int(rec.type_id)))
                chem = ch.chemistry()
                if chem is not None:
                    self._chem_keep = getattr(self, "_chem_keep", []) + [chem]
                    L.check(lib.sfg_set_chemistry(h, idx.value, C.byref(chem)))
            L.check(lib.sfg_initialize(h))
        except Exception:
            lib.sfg_destroy(h)
            self._h = None
            raise

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sfg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int):
        L.check(self._lib.sfg_step(self._h, int(n)))
        self.touch()

    def touch(self):
        """Marks the device state as changed (drops cached reductions)."""
        self._version += 1
        self._thermo_cache = None

    def thermo(self):
        """Device-side reductions of the current state (sfg_thermo): a list
        of per-channel dicts and the [capsules][6] geometry array (centroid
        x, y, area, perimeter, deformation, inclination).  Cached until the
        state changes."""
        if self._thermo_cache is not None:
            return self._thermo_cache
        recs = (L.ThermoRecordC * max(self.num_channels, 1))()
        caps = np.zeros((max(self.num_capsules, 1), 6))
        L.check(self._lib.sfg_thermo(self._h, recs, L.dptr(caps)))
        out = [thermo_dict(recs[i]) for i in range(self.num_channels)]
        self._thermo_cache = (out, caps[:self.num_capsules])
        return self._thermo_cache

    def run(self, n: int, every: int, fn) -> int:
        """sfg_run: n steps; fn(step, records, caps) after every `every`
        steps and after the last; a true return stops the run."""
        def cb(step, recs, nch, caps, ncaps, user):
            try:
                r = [thermo_dict(recs[i]) for i in range(nch)]
                c = (np.ctypeslib.as_array(caps, shape=(ncaps, 6)).copy() if ncaps
                     else np.zeros((0, 6)))
                return 1 if fn(int(step), r, c) else 0
            except Exception as e:          # stop the run; re-raised below
                errors.append(e)
                return 1
        errors = []
        done = C.c_int(0)
        cfn = L.THERMO_FN(cb)
        try:
            L.check(self._lib.sfg_run(self._h, int(n), int(every), cfn, None, C.byref(done)))
        finally:
            self.touch()
        if errors:
            raise errors[0]
        return int(done.value)

    def synchronize(self) -> int:
        st = C.c_uint(0)
        L.check(self._lib.sfg_synchronize(self._h, C.byref(st)))
        return st.value

    def last_step_ms(self) -> float:
        ms = C.c_float()
        L.check(self._lib.sfg_last_step_ms(self._h, C.byref(ms)))
        return ms.value

    def launches_per_step(self) -> int:
        v = C.c_int()
        L.check(self._lib.sfg_launches_per_step(self._h, C.byref(v)))
        return v.value

    def set_profiling(self, on: bool):
        L.check(self._lib.sfg_set_profiling(self._h, int(bool(on))))

    def phase_times(self) -> dict:
        """Accumulated milliseconds per phase since the last reset."""
        arr = (C.c_float * len(L.PHASES))()
        L.check(self._lib.sfg_get_phase_times(self._h, arr, len(L.PHASES)))
        return {k: float(v) for k, v in zip(L.PHASES, arr)}

    def reset_phase_times(self):
        L.check(self._lib.sfg_reset_phase_times(self._h))

    def stream(self) -> int:
        s = C.c_void_p()
        L.check(self._lib.sfg_get_stream(self._h, C.byref(s)))
        return s.value or 0


def thermo_dict(r) -> dict:
    return {k: getattr(r, k) for k, _ in L.ThermoRecordC._fields_ if k != "reserved"}


class FieldView:
    """Lattice field of one channel (reference LatticeField views,
    bindings.cpp:313-383).  Arrays are copies taken at the call."""

    def __init__(self, ctx: _Context, chan: int, nx: int, ny: int):
        self._ctx, self._ch, self.nx, self.ny = ctx, chan, nx, ny

    def getNx(self):
        return self.nx

    def getNy(self):
        return self.ny

    def size(self):
        return self.nx * self.ny

    def _macro(self):
        N = self.nx * self.ny
        out = [np.zeros(N) for _ in range(5)]
        L.check(self._ctx._lib.sfg_get_macroscopic(self._ctx._h, self._ch,
                                                   *[L.dptr(a) for a in out]))
        return [a.reshape(self.ny, self.nx) for a in out]

    def macroscopic(self):
        """(rho, ux, uy, Fx, Fy), each [ny][nx]."""
        return tuple(self._macro())

    def density(self):
        return self._macro()[0]

    def velocity_x(self):
        return self._macro()[1]

    def velocity_y(self):
        return self._macro()[2]

    def force_x(self):
        return self._macro()[3]

    def force_y(self):
        return self._macro()[4]

    def distributions(self):
        """Populations [9][ny][nx] (reference layout f[q*N + y*nx + x])."""
        f = np.zeros(9 * self.nx * self.ny)
        L.check(self._ctx._lib.sfg_get_populations(self._ctx._h, self._ch, L.dptr(f)))
        return f.reshape(9, self.ny, self.nx)

    def set_distributions(self, f: np.ndarray):
        a = np.ascontiguousarray(f, dtype=np.float64).ravel()
        if a.size != 9 * self.nx * self.ny:
            raise ValueError("populations must have 9*ny*nx entries")
        L.check(self._ctx._lib.sfg_set_populations(self._ctx._h, self._ch, L.dptr(a)))
        self._ctx.touch()

    def getRho(self, x, y):
        return float(self.density()[y, x])

    def getUx(self, x, y):
        return float(self.velocity_x()[y, x])

    def getUy(self, x, y):
        return float(self.velocity_y()[y, x])


class CapsuleView:
    def __init__(self, system: "CapsuleSystemView", idx: int):
        self._s, self._i = system, idx

    def numNodes(self):
        return self._s._counts[self._i]

    def getTypeId(self):
        return self._s._types[self._i]

    getType = getTypeId

    def _slice(self, arr):
        o = self._s._offsets[self._i]
        return arr[o:o + self.numNodes()]

    def node_positions_array(self):
        return self._slice(self._s.positions()).copy()

    def nodePosition(self, k):
        return tuple(self._slice(self._s.positions())[k])

    def nodeVelocity(self, k):
        return tuple(self._slice(self._s.velocities())[k])

    def nodeForce(self, k):
        return tuple(self._slice(self._s.forces())[k])

    def _stats(self):
        return self._s._ctx.thermo()[1][self._s._cap_base + self._i]

    # Geometry reduced on the device (sfg_thermo), FP64 in the reference's
    # serial order: Capsule::centroid, area, perimeter, deformationIndex,
    # inclinationAngle (capsule.cpp:159-266).
    def centroid(self):
        st = self._stats()
        return (float(st[0]), float(st[1]))

    def area(self):
        return float(self._stats()[2])

    def perimeter(self):
        return float(self._stats()[3])

    def deformationIndex(self):
        return float(self._stats()[4])

    def inclinationAngle(self):
        return float(self._stats()[5])


class CapsuleSystemView:
    """Marker state of one channel (reference CapsuleSystem, capsule-major)."""

    def __init__(self, ctx: _Context, chan: int, recs: List[_CapsuleRec], nx: int,
                 cap_base: int = 0):
        self._ctx, self._ch, self._nx = ctx, chan, nx
        self._cap_base = cap_base
        self._counts = [r.rest.num_nodes for r in recs]
        self._types = [r.type_id for r in recs]
        self._offsets = np.concatenate([[0], np.cumsum(self._counts)]).astype(int)
        self.M = int(self._offsets[-1])

    def numCapsules(self):
        return len(self._counts)

    def totalNodes(self):
        return self.M

    def __len__(self):
        return self.numCapsules()

    def __getitem__(self, i):
        if i < 0 or i >= self.numCapsules():
            raise IndexError("Capsule index out of range")
        return CapsuleView(self, i)

    def _get(self):
        pos, vel, frc = np.zeros(2 * self.M), np.zeros(2 * self.M), np.zeros(2 * self.M)
        if self.M:
            L.check(self._ctx._lib.sfg_get_markers(self._ctx._h, self._ch, L.dptr(pos),
                                                   L.dptr(vel), L.dptr(frc)))
        return pos.reshape(-1, 2), vel.reshape(-1, 2), frc.reshape(-1, 2)

    def positions(self):
        return self._get()[0]

    def velocities(self):
        return self._get()[1]

    def forces(self):
        return self._get()[2]

    def set_state(self, pos: Optional[np.ndarray] = None, vel: Optional[np.ndarray] = None):
        p = None if pos is None else np.ascontiguousarray(pos, dtype=np.float64).ravel()
        v = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64).ravel()
        L.check(self._ctx._lib.sfg_set_markers(self._ctx._h, self._ch, L.dptr(p), L.dptr(v)))
        self._ctx.touch()

    def contact_counts(self):
        c = np.zeros(max(self.M, 1), dtype=np.int32)
        L.check(self._ctx._lib.sfg_get_contact_counts(self._ctx._h, self._ch, L.iptr(c)))
        return c[:self.M]


class ScalarView:
    """Advection-diffusion scalar of one channel (reference AdvectionDiffusion,
    bindings.cpp:422-455)."""

    def __init__(self, ctx: _Context, chan: int, nx: int, ny: int):
        self._ctx, self._ch, self.nx, self.ny = ctx, chan, nx, ny

    def _chem(self):
        lib, h = self._ctx._lib, self._ctx._h
        nc, nm = C.c_int(), C.c_int()
        L.check(lib.sfg_channel_counts(h, self._ch, C.byref(nc), C.byref(nm)))
        out = [np.zeros(max(nc.value, 1)) for _ in range(3)] + [np.zeros(max(nm.value, 1))]
        L.check(lib.sfg_get_chemistry_state(h, self._ch, *[L.dptr(a) for a in out]))
        nodes = (C.c_int * max(nc.value, 1))()
        L.check(lib.sfg_get_capsule_nodes(h, self._ch, nodes))
        return out, list(nodes)[:nc.value]

    # chemistry state (AdvectionDiffusion accessors, advection_diffusion.h:75-103)
    def getCapsuleReleased(self, capsule_id: int) -> float:
        return float(self._chem()[0][0][capsule_id])

    def getCapsuleAbsorbed(self, capsule_id: int) -> float:
        return float(self._chem()[0][1][capsule_id])

    def getCapsuleMp(self, capsule_id: int) -> float:
        return float(self._chem()[0][2][capsule_id])

    def getNodeGamma(self, capsule_id: int, node: int) -> float:
        (st, nodes) = self._chem()
        return float(st[3][sum(nodes[:capsule_id]) + node])

    def concentration(self, species: int = 0):
        Cf = np.zeros(self.nx * self.ny)
        L.check(self._ctx._lib.sfg_get_concentration(self._ctx._h, self._ch, L.dptr(Cf), None))
        return Cf.reshape(self.ny, self.nx)

    def populations(self):
        """Scalar populations [9][ny][nx]."""
        Cf = np.zeros(self.nx * self.ny)
        g = np.zeros(9 * self.nx * self.ny)
        L.check(self._ctx._lib.sfg_get_concentration(self._ctx._h, self._ch, L.dptr(Cf),
                                                     L.dptr(g)))
        return g.reshape(9, self.ny, self.nx)

    def setConcentration(self, Cfield: np.ndarray):
        """Sets C and the equilibrium populations g = w C."""
        a = np.ascontiguousarray(Cfield, dtype=np.float64).ravel()
        if a.size != self.nx * self.ny:
            raise ValueError("concentration must have ny*nx entries")
        L.check(self._ctx._lib.sfg_set_concentration(self._ctx._h, self._ch, L.dptr(a)))
        self._ctx.touch()

    def setRegion(self, x0, y0, x1, y1, concentration, species=0):
        Cf = self.concentration()
        Cf[max(0, y0):min(self.ny, y1), max(0, x0):min(self.nx, x1)] = concentration
        self.setConcentration(Cf)

    def setPoint(self, x, y, concentration, species=0):
        if 0 <= x < self.nx and 0 <= y < self.ny:
            Cf = self.concentration()
            Cf[y, x] = concentration
            self.setConcentration(Cf)


class Ensemble:
    """Many independent channels advanced together on one GPU.

    Build channels with ``add_channel(params)`` -> index, add capsules through
    ``addCapsule`` / ``addCapsuleRandom`` with that index, then
    ``initialize()`` and ``run(n)``.  Each channel's results equal the same
    channel run alone.
    """

    def __init__(self, precision: str = "fp32", device: int = 0, lattice_variant: int = 0):
        self.precision = precision
        self.device = device
        self.lattice_variant = lattice_variant
        self._chans: List[_Channel] = []
        self._ctx: Optional[_Context] = None
        self._steps = 0

    def add_channel(self, params: SimulationParams) -> int:
        if self._ctx is not None:
            raise RuntimeError("channels must be added before initialize()")
        self._chans.append(_Channel(params))
        return len(self._chans) - 1

    def addCapsule(self, chan, center, radius, num_nodes=0, mparams=None, type=0):
        self._pre_init()
        return self._chans[chan].add_capsule(center, radius, num_nodes, mparams, type)

    def addCapsuleRandom(self, chan, count, x0, y0, x1, y1, radius_min, radius_max,
                         num_nodes=0, mparams=None, type=0, seed=12345, min_gap=1.0,
                         max_attempts=0, check_walls=None):
        self._pre_init()
        ch = self._chans[chan]
        cw = ch.walls_in_placement if check_walls is None else check_walls
        return ch.add_random(count, x0, y0, x1, y1, radius_min, radius_max, num_nodes, mparams,
                             type, seed, min_gap, max_attempts, cw)

    def setChannelWalls(self, chan: int, enabled: bool = True):
        """Apply the channel-builder wall test in random placement
        (simulation.cpp:250-256), as the declarative Python API does."""
        self._chans[chan].walls_in_placement = bool(enabled)

    def setScalarReleaseRate(self, chan: int, capsule_type: int, rate: float):
        """Simulation::setScalarReleaseRate (simulation.cpp:929-935)."""
        self._pre_init()
        v = self._chans[chan].release_rates
        if capsule_type >= len(v):
            v.extend([0.0] * (capsule_type + 1 - len(v)))
        v[capsule_type] = float(rate)

    def setScalarAbsorptionRate(self, chan: int, capsule_type: int, rate: float):
        """Simulation::setScalarAbsorptionRate (simulation.cpp:936-942)."""
        self._pre_init()
        v = self._chans[chan].absorption_rates
        if capsule_type >= len(v):
            v.extend([0.0] * (capsule_type + 1 - len(v)))
        v[capsule_type] = float(rate)

    def chemistryState(self, chan: int = 0):
        """(released [capsules], absorbed [capsules], Mp [capsules],
        gamma [markers]) of a channel (AdvectionDiffusion's per-capsule and
        per-node chemistry state)."""
        ctx = self._need()
        n = len(self._chans[chan].caps)
        m = sum(r.rest.num_nodes for r in self._chans[chan].caps)
        out = [np.zeros(max(n, 1)), np.zeros(max(n, 1)), np.zeros(max(n, 1)),
               np.zeros(max(m, 1))]
        L.check(ctx._lib.sfg_get_chemistry_state(ctx._h, chan, *[L.dptr(a) for a in out]))
        return out[0][:n], out[1][:n], out[2][:n], out[3][:m]

    def setChannelBuilder(self, chan: int, builder: "ChannelBuilder"):
        """Simulation::setChannelBuilder (simulation.cpp:211-213): the
        builder's pillars become SOLID nodes of the channel (with Bouzidi
        links when fluid.use_interpolated_bb)."""
        self._pre_init()
        self._chans[chan].pillars = list(builder.pillars)
        # with a channel builder the random placement tests the walls and
        # the obstacles (simulation.cpp:250-262)
        self._chans[chan].walls_in_placement = True

    def _pre_init(self):
        if self._ctx is not None:
            raise RuntimeError("capsules must be added before initialize()")

    def initialize(self):
        if self._ctx is not None:
            raise RuntimeError("already initialized")
        self._ctx = _Context(self._chans, self.precision, self.device, self.lattice_variant)
        self._steps = 0

    def _need(self):
        if self._ctx is None:
            raise RuntimeError("call initialize() first")
        return self._ctx

    def step(self):
        self._need().step(1)
        self._steps += 1

    def run(self, num_steps: int, thermo_every: int = 0, callback=None) -> int:
        """Advances every channel by num_steps steps in C++ (sfg_run / sfg_step
        in CUDA graphs; no Python per step).

        callback(step, records, capsule_stats) -> bool, if given, is called
        after every thermo_every steps and after the last one with the
        device-reduced thermo (see thermo()); a true return stops the run.
        Without a callback, the stability check of Simulation::step
        (simulation.cpp:729-733) runs where the reference runs it: after the
        step whose count before the step is a multiple of
        stability_check_interval.  Returns the steps run."""
        ctx = self._need()
        num_steps = int(num_steps)
        if callback is not None:
            done = ctx.run(num_steps, int(thermo_every), callback)
            self._steps += done
            return done
        events = self._scheduled()
        done = 0
        while done < num_steps:
            # next step (counted before the step, as the reference's
            # step_count_) at which some per-step task runs
            s0 = self._steps
            nxt = None
            for iv, first, _ in events:
                k = max(s0, first)
                m = -(-k // iv) * iv
                nxt = m if nxt is None else min(nxt, m)
            n = num_steps - done if nxt is None else min(num_steps - done, nxt - s0 + 1)
            ctx.step(n)
            self._steps += n
            done += n
            if nxt is not None and self._steps - 1 == nxt:
                for iv, first, fn in events:
                    if nxt >= first and nxt % iv == 0:
                        fn(nxt)
        ctx.synchronize()
        self._finish_run()
        return done

    def _scheduled(self):
        """Per-step tasks of Simulation::step after the physics
        (simulation.cpp:729-787) as (interval, first step, fn(step))."""
        ev = []
        for k, c in enumerate(self._chans):
            iv = c.params.stability_check_interval
            if c.params.enable_stability_checks and iv > 0:
                ev.append((iv, 0, lambda s, k=k: self.checkStability(k, step=s)))
        return ev

    def _finish_run(self):
        pass

    def synchronize(self) -> int:
        return self._need().synchronize()

    def currentStep(self) -> int:
        return self._steps

    def num_channels(self) -> int:
        return len(self._chans)

    def field(self, chan: int = 0) -> FieldView:
        p = self._chans[chan].params
        return FieldView(self._need(), chan, p.nx, p.ny)

    def capsules(self, chan: int = 0) -> CapsuleSystemView:
        base = sum(len(c.caps) for c in self._chans[:chan])
        return CapsuleSystemView(self._need(), chan, self._chans[chan].caps,
                                 self._chans[chan].params.nx, base)

    def advectionDiffusion(self, chan: int = 0) -> Optional[ScalarView]:
        p = self._chans[chan].params
        if not p.scalar.enabled:
            return None
        return ScalarView(self._need(), chan, p.nx, p.ny)

    def lastCappedNodes(self, chan: int = 0) -> int:
        v = C.c_int()
        L.check(self._need()._lib.sfg_get_capped_count(self._ctx._h, chan, C.byref(v)))
        return v.value

    def thermo(self, chan: Optional[int] = None):
        """Device-side reductions of the state after the last step (one
        launch set for every channel, sfg_thermo): max_speed, mean_rho,
        mean_velocity, kinetic_energy, min_rho, max_rho, total_scalar,
        mean_deformation, max_deformation, fluid_cells, first_nonfinite,
        capped_nodes, num_capsules.  One dict for `chan`, else a list."""
        recs = self._need().thermo()[0]
        return recs if chan is None else recs[chan]

    def getMaxSpeed(self, chan: int = 0) -> float:
        """max |u| over non-SOLID cells (simulation.cpp:892-907), reduced on
        the device."""
        return float(self.thermo(chan)["max_speed"])

    def checkStability(self, chan: int = 0, step: Optional[int] = None) -> dict:
        """Simulation::checkStability (simulation.cpp:817-889) from the
        device reductions: warnings for a non-finite cell (the first in
        row-major order), a density deviation above max_density_deviation
        (the extreme rho), a speed above max_velocity, and the capped-cell
        notice, printed to stderr as the reference does.  Returns the
        findings."""
        p = self._chans[chan].params
        t = self.thermo(chan)
        step = self._steps if step is None else step
        nx = p.nx
        out = {"nonfinite": None, "worst_rho": None, "worst_velocity": None,
               "capped_nodes": int(t["capped_nodes"])}
        if t["first_nonfinite"] >= 0:
            i = int(t["first_nonfinite"])
            out["nonfinite"] = (i % nx, i // nx)
            print(f"*** STABILITY WARNING: NaN/Inf detected at step {step} at "
                  f"({i % nx},{i // nx})", file=sys.stderr)
        rho0 = p.fluid.rho0
        dev_lo = abs(t["min_rho"] - rho0) / rho0
        dev_hi = abs(t["max_rho"] - rho0) / rho0
        # the reference's scan stops at the first non-finite cell; the
        # whole-field extremes are only reported for a finite field
        finite = out["nonfinite"] is None
        if finite and max(dev_lo, dev_hi) > p.max_density_deviation:
            worst = t["min_rho"] if dev_lo > dev_hi else t["max_rho"]
            out["worst_rho"] = worst
            print(f"*** STABILITY WARNING: density deviation at step {step} \u2014 rho = "
                  f"{worst:g} (rho0 = {rho0:g}, deviation = "
                  f"{abs(worst - rho0) / rho0 * 100.0:g}%)", file=sys.stderr)
        if finite and t["max_speed"] > p.max_velocity:
            out["worst_velocity"] = t["max_speed"]
            print(f"*** STABILITY WARNING: high velocity at step {step} \u2014 |u| = "
                  f"{t['max_speed']:g} (limit = {p.max_velocity:g}, Ma = "
                  f"{t['max_speed'] / math.sqrt(1.0 / 3.0):g})", file=sys.stderr)
        if t["capped_nodes"] > 0:
            print(f"*** STABILITY NOTICE: max_lattice_force cap rescaled {t['capped_nodes']} "
                  f"fluid nodes at step {step} (cap = {p.max_lattice_force:g})", file=sys.stderr)
        return out

    def context(self) -> _Context:
        return self._need()

    # ---- launch shapes
    def autotune(self, steps_per_trial: int = 5) -> dict:
        """Times candidate launch shapes on real steps and keeps the fastest;
        the ensemble advances by the returned number of steps."""
        ctx = self._need()
        n = C.c_int()
        L.check(ctx._lib.sfg_autotune(ctx._h, int(steps_per_trial), C.byref(n)))
        ctx.touch()
        ctx.synchronize()
        self._steps += int(n.value)
        cfg = self.launchConfig()
        cfg["steps_run"] = int(n.value)
        return cfg

    def launchConfig(self) -> dict:
        ctx = self._need()
        v = [C.c_int() for _ in range(4)]
        L.check(ctx._lib.sfg_get_launch_config(ctx._h, *[C.byref(x) for x in v]))
        return dict(lattice_ctas_per_sm=v[0].value, spread_ctas_per_sm=v[1].value,
                    marker_block=v[2].value, learned_ctas_per_sm=v[3].value)

    # ---- learned multi-direct forcing
    def setLearnedMDF(self, net=None, threshold: float = 1e-4):
        """Use the network `net` (softflow_b200.learned.MDFNetwork) to seed
        the forcing correction, followed by one plain sweep, on every channel
        with ibm_iterations >= 3; a channel whose no-slip residual exceeds
        `threshold` (lu/step) redoes the plain sweeps.  net=None restores the
        plain sweeps everywhere."""
        ctx = self._need()
        L.check(ctx._lib.sfg_set_mdf_model(ctx._h, net.handle if net is not None else None,
                                           float(threshold)))
        self._learned_net = net     # keeps the trainer object alive

    def mdfStats(self, chan: int = 0) -> dict:
        """Last step's no-slip residuals (learned gate, plain iteration) and
        the cumulative learned / fallback step counts of a channel."""
        ctx = self._need()
        a, b = C.c_float(), C.c_float()
        ls, fb = C.c_longlong(), C.c_longlong()
        L.check(ctx._lib.sfg_get_mdf_stats(ctx._h, int(chan), C.byref(a), C.byref(b),
                                           C.byref(ls), C.byref(fb)))
        return dict(resid_learned=float(a.value), resid_plain=float(b.value),
                    learned_steps=int(ls.value), fallbacks=int(fb.value))

    def setHarvest(self, enabled: bool = True):
        ctx = self._need()
        L.check(ctx._lib.sfg_set_harvest(ctx._h, int(bool(enabled))))

    def num_markers(self) -> int:
        return sum(r.rest.num_nodes for ch in self._chans for r in ch.caps)

    def harvest(self):
        """(features [M, 8], labels [M, 2], valid [M] bool) of the last step."""
        ctx = self._need()
        M = self.num_markers()
        feat = np.zeros((M, 8), np.float32)
        lab = np.zeros((M, 2), np.float32)
        val = np.zeros(M, np.int32)
        L.check(ctx._lib.sfg_get_harvest(ctx._h, feat.ctypes.data_as(C.POINTER(C.c_float)),
                                         lab.ctypes.data_as(C.POINTER(C.c_float)),
                                         val.ctypes.data_as(C.POINTER(C.c_int))))
        return feat, lab, val.astype(bool)

    def close(self):
        if self._ctx is not None:
            self._ctx.close()
            self._ctx = None


class Simulation(Ensemble):
    """Single-channel engine with the reference ``Simulation`` API
    (bindings.cpp:846-981)."""

    def __init__(self, params: SimulationParams):
        super().__init__(params.precision, params.device)
        self.add_channel(params)
        self._params = params

    def params(self) -> SimulationParams:
        return self._params

    def addCapsule(self, center, radius, num_nodes=0, mparams=None, type=0):
        return super().addCapsule(0, center, radius, num_nodes, mparams, type)

    def addCapsuleRandom(self, count, x0, y0, x1, y1, radius_min, radius_max, num_nodes=0,
                         mparams=None, type=0, seed=12345, min_gap=1.0, max_attempts=0,
                         check_walls=None):
        return super().addCapsuleRandom(0, count, x0, y0, x1, y1, radius_min, radius_max,
                                        num_nodes, mparams, type, seed, min_gap, max_attempts,
                                        check_walls)

    def setChannelWalls(self, enabled: bool = True):
        super().setChannelWalls(0, enabled)

    def setChannelBuilder(self, builder: "ChannelBuilder"):
        super().setChannelBuilder(0, builder)

    def setScalarReleaseRate(self, capsule_type: int, rate: float):
        super().setScalarReleaseRate(0, capsule_type, rate)

    def setScalarAbsorptionRate(self, capsule_type: int, rate: float):
        super().setScalarAbsorptionRate(0, capsule_type, rate)

    def setStepCallback(self, fn):
        """fn(sim, step) after every step (Simulation::setStepCallback; step
        counted before the step, simulation.cpp:781-784).  Costs one host
        round trip per step."""
        self._step_callback = fn

    def _writers(self):
        from . import output as O
        if getattr(self, "_out", None) is None:
            p = self._params
            d = p.output_dir
            self._out = {"vtk": O.VTKWriter(d, legacy=(p.vtk_format == "legacy")),
                         "csv": O.CSVWriter(d), "probe": O.FluidProbeWriter(d),
                         "stats": O.GlobalStatsWriter(d)}
            for i, j, label in p.probes:
                self._out["probe"].addProbe(i, j, label)
        return self._out

    def _scheduled(self):
        ev = super()._scheduled()
        p = self._params
        if p.output_dir:
            w = self._writers()
            t = lambda s: s * p.dt  # noqa: E731
            vtk_iv = p.vtk_dump_every if p.vtk_dump_every > 0 else p.output_interval
            csv_iv = p.csv_dump_every if p.csv_dump_every > 0 else p.output_interval

            def vtk(s):
                w["vtk"].writeFluidField(self, s)
                w["vtk"].writeCapsules(self, s)
                w["vtk"].recordTimestep(s, t(s))
            if vtk_iv > 0:
                ev.append((vtk_iv, 0, vtk))
            if csv_iv > 0:
                ev.append((csv_iv, 0, lambda s: w["csv"].writeTimestep(self, s, t(s))))
            if p.probe_dump_every > 0 and p.probes:
                ev.append((p.probe_dump_every, 0,
                           lambda s: w["probe"].writeTimestep(self, s, t(s))))
            if p.stats_dump_every > 0:
                ev.append((p.stats_dump_every, 0,
                           lambda s: w["stats"].writeTimestep(self, s, t(s))))
            if p.checkpoint_interval > 0:
                from .output import Checkpoint

                def ckpt(s):
                    # named and stamped with the step count before the
                    # increment, as the reference does (simulation.cpp:
                    # 773-779); the file holds the state after the step
                    Checkpoint.save(self, os.path.join(p.output_dir, f"checkpoint_{s}.sfck"),
                                    step=s)
                ev.append((p.checkpoint_interval, 1, ckpt))
        cb = getattr(self, "_step_callback", None)
        if cb is not None:
            ev.append((1, 0, lambda s: cb(self, s)))
        return ev

    def _finish_run(self):
        """Simulation::finalize (simulation.cpp:802-817): PVD collections,
        writers closed."""
        out = getattr(self, "_out", None)
        if out is not None:
            out["vtk"].writePVDFiles()
            for k in ("csv", "probe", "stats"):
                out[k].close()
            self._out = None

    def saveCheckpoint(self, filename: str) -> str:
        from .output import Checkpoint
        return Checkpoint.save(self, filename)

    def loadCheckpoint(self, filename: str) -> int:
        from .output import Checkpoint
        return Checkpoint.load(self, filename)
