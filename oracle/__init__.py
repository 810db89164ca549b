"""CPU checkers for the SoftFlow hot path (test infrastructure only).

Two implementations share one ctypes wrapper:

* ``impl="sfo"`` -- ``oracle/sfo.c``, the C restatement of the reference
  algorithm (always buildable from this repository);
* ``impl="ref"`` -- the reference engine's own sources compiled by
  ``oracle/Makefile`` into ``oracle/_ref/libsfref.so`` (deterministic build)
  or ``libsfref_fast.so`` (the reference's Release flags, used only to time
  the CPU baseline).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package.  The product (``softflow_b200``) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field, fields

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SFO_LIB = os.path.join(HERE, "_build", "libsfo.so")
REF_LIB = os.path.join(HERE, "_ref", "libsfref.so")
REF_FAST_LIB = os.path.join(HERE, "_ref", "libsfref_fast.so")
# the reference's own softflow::Simulation (engine/simulation.cpp) behind the
# same C entry points (ref_engine.cpp)
ENGINE_LIB = os.path.join(HERE, "_ref", "libsfengine.so")

BGK, MRT, REGULARIZED = 0, 1, 2
HOOKEAN, NEO_HOOKEAN, SKALAK, WLC = 0, 1, 2, 3
INLET_OUTLET, PERIODIC, CLOSED = 0, 1, 2


class _Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("collision", C.c_int),
        ("tau", C.c_double), ("rho0", C.c_double),
        ("mrt_se", C.c_double), ("mrt_s_eps", C.c_double), ("mrt_sq", C.c_double),
        ("body_fx", C.c_double), ("body_fy", C.c_double),
        ("periodic_y", C.c_int), ("max_lattice_force", C.c_double),
        ("ibm_iterations", C.c_int), ("dt", C.c_double),
        ("rep_epsilon", C.c_double), ("rep_sigma", C.c_double), ("rep_r_cut", C.c_double),
        ("rep_power", C.c_int), ("rep_damping_normal", C.c_double), ("rep_friction", C.c_double),
        ("scalar_enabled", C.c_int), ("scalar_D", C.c_double),
        ("scalar_periodic_y", C.c_int), ("scalar_inlet", C.c_double),
        ("boundary_type", C.c_int), ("inlet_velocity", C.c_double),
        ("outlet_density", C.c_double), ("top_wall_velocity", C.c_double),
        ("bottom_wall_velocity", C.c_double), ("use_interpolated_bb", C.c_int),
    ]


class _Chemistry(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("n_release", "n_absorb", "n_k_leach", "n_C_eq", "n_M_p",
                                       "n_k_adsorb", "n_k_desorb", "n_Gamma_max")] + \
               [(n, C.c_double * 8) for n in ("release", "absorb", "k_leach", "C_eq",
                                              "M_p_initial", "k_adsorb", "k_desorb",
                                              "Gamma_max")]


def chemistry_struct(**vectors) -> _Chemistry:
    """Per capsule type vectors (lists) keyed release, absorb, k_leach, C_eq,
    M_p_initial, k_adsorb, k_desorb, Gamma_max; missing keys are empty."""
    counts = {"release": "n_release", "absorb": "n_absorb", "k_leach": "n_k_leach",
              "C_eq": "n_C_eq", "M_p_initial": "n_M_p", "k_adsorb": "n_k_adsorb",
              "k_desorb": "n_k_desorb", "Gamma_max": "n_Gamma_max"}
    c = _Chemistry()
    for k, v in vectors.items():
        setattr(c, counts[k], len(v))
        arr = getattr(c, k)
        for i, x in enumerate(v):
            arr[i] = float(x)
    return c


class _Membrane(C.Structure):
    _fields_ = [
        ("model", C.c_int), ("k_stretch", C.c_double), ("G_s", C.c_double),
        ("C_skalak", C.c_double), ("wlc_L_max_ratio", C.c_double),
        ("wlc_kBT_p", C.c_double), ("wlc_k_pow", C.c_double), ("k_bend", C.c_double),
        ("use_helfrich", C.c_int), ("kappa_0", C.c_double), ("k_area", C.c_double),
        ("k_perimeter", C.c_double), ("gamma_visc", C.c_double), ("eta_membrane", C.c_double),
    ]


@dataclass
class ChannelSpec:
    """Hot-path subset of the reference SimulationParams (parameters.h:41-342)."""
    nx: int = 200
    ny: int = 50
    collision: int = BGK
    tau: float = 0.8
    rho0: float = 1.0
    mrt_se: float = 1.4
    mrt_s_eps: float = 1.4
    mrt_sq: float = 1.4
    body_fx: float = 0.0
    body_fy: float = 0.0
    periodic_y: int = 0
    max_lattice_force: float = 0.01
    ibm_iterations: int = 1
    dt: float = 1.0
    rep_epsilon: float = 0.05
    rep_sigma: float = 1.0
    rep_r_cut: float = 3.5
    rep_power: int = 4
    rep_damping_normal: float = 0.0
    rep_friction: float = 0.0
    scalar_enabled: int = 0
    scalar_D: float = 0.01
    scalar_periodic_y: int = 0
    scalar_inlet: float = 0.0
    # BoundaryType (types.h:58-62): 0 INLET_OUTLET, 1 PERIODIC, 2 CLOSED
    boundary_type: int = 1
    inlet_velocity: float = 0.02
    outlet_density: float = 1.0
    top_wall_velocity: float = 0.0
    bottom_wall_velocity: float = 0.0
    use_interpolated_bb: int = 0

    def to_c(self) -> _Params:
        return _Params(**{f.name: getattr(self, f.name) for f in fields(self)})


@dataclass
class Membrane:
    """Reference MembraneParams defaults (parameters.h:82-136)."""
    model: int = HOOKEAN
    k_stretch: float = 0.1
    G_s: float = 0.1
    C_skalak: float = 1.0
    wlc_L_max_ratio: float = 2.2
    wlc_kBT_p: float = 0.0
    wlc_k_pow: float = 0.0
    k_bend: float = 0.005
    use_helfrich: int = 0
    kappa_0: float = 0.0
    k_area: float = 0.5
    k_perimeter: float = 0.1
    gamma_visc: float = 0.01
    eta_membrane: float = 0.05

    def to_c(self) -> _Membrane:
        return _Membrane(**{f.name: getattr(self, f.name) for f in fields(self)})


def build(ref="auto") -> None:
    """Build the C restatement, and the reference libraries: always when ref
    is True, never when False, and with "auto" when the Makefile finds the
    reference tree (REF_SRC, overridable from the environment)."""
    targets = {True: ["oracle", "ref"], False: ["oracle"]}.get(ref, ["auto"])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


_LIBS: dict = {}


def _load(path: str, prefix: str):
    key = (path, prefix)
    if key in _LIBS:
        return _LIBS[key]
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    lib = C.CDLL(path)
    d = C.POINTER(C.c_double)
    sig = {
        "create": (C.c_void_p, [C.POINTER(_Params)]),
        "destroy": (None, [C.c_void_p]),
        "add_capsule": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int,
                                  C.POINTER(_Membrane), C.c_int]),
        "add_capsule_random": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double,
                                         C.c_double, C.c_double, C.c_double, C.c_int,
                                         C.POINTER(_Membrane), C.c_int, C.c_int, C.c_double,
                                         C.c_int, C.c_int]),
        "initialize": (None, [C.c_void_p]),
        "add_circle_pillar": (None, [C.c_void_p, C.c_double, C.c_double, C.c_double]),
        "set_chemistry": (None, [C.c_void_p, C.POINTER(_Chemistry)]),
        "chemistry_state": (None, [C.c_void_p, d, d, d, d]),
        "add_rect_pillar": (None, [C.c_void_p, C.c_double, C.c_double, C.c_double,
                                   C.c_double]),
        "step": (None, [C.c_void_p, C.c_int]),
        "num_capsules": (C.c_int, [C.c_void_p]),
        "num_markers": (C.c_int, [C.c_void_p]),
        "capsule_offsets": (C.POINTER(C.c_int), [C.c_void_p]),
        "f": (d, [C.c_void_p]), "rho": (d, [C.c_void_p]), "ux": (d, [C.c_void_p]),
        "uy": (d, [C.c_void_p]), "Fx": (d, [C.c_void_p]), "Fy": (d, [C.c_void_p]),
        "pos": (d, [C.c_void_p]), "vel": (d, [C.c_void_p]), "force": (d, [C.c_void_p]),
        "g": (d, [C.c_void_p]), "C": (d, [C.c_void_p]),
        "last_capped": (C.c_int, [C.c_void_p]),
        "capsule_area": (C.c_double, [C.c_void_p, C.c_int]),
        "capsule_perimeter": (C.c_double, [C.c_void_p, C.c_int]),
        "capsule_deformation": (C.c_double, [C.c_void_p, C.c_int]),
        "capsule_inclination": (C.c_double, [C.c_void_p, C.c_int]),
        "capsule_centroid": (None, [C.c_void_p, C.c_int, d, d]),
        "set_concentration": (None, [C.c_void_p, d]),
        "phi": (C.c_double, [C.c_double]),
        "spread_forces": (None, [C.c_void_p]),
        "compute_membrane_forces": (None, [C.c_void_p]),
    }
    fns = {}
    for name, (res, args) in sig.items():
        fn = getattr(lib, prefix + name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
        fns[name] = fn
    if prefix == "sfe_":
        lib.sfe_set_threads.argtypes = [C.c_int]
        lib.sfe_set_threads.restype = None
        lib.sfe_get_threads.restype = C.c_int
        fns["set_threads"] = lib.sfe_set_threads
        fns["get_threads"] = lib.sfe_get_threads
    if prefix == "sfr_":
        lib.sfr_write_vtk.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int]
        lib.sfr_write_vtk.restype = None
        lib.sfr_write_global_stats.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_double]
        lib.sfr_write_global_stats.restype = None
        fns["write_vtk"] = lib.sfr_write_vtk
        fns["write_global_stats"] = lib.sfr_write_global_stats
        lib.sfr_set_threads.argtypes = [C.c_int]
        lib.sfr_set_threads.restype = None
        lib.sfr_get_threads.restype = C.c_int
        fns["set_threads"] = lib.sfr_set_threads
        fns["get_threads"] = lib.sfr_get_threads
    if prefix == "sfo_":
        for name in ("contact_pairs",):
            fn = getattr(lib, prefix + name)
            fn.restype = C.c_int
            fn.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int]
            fns[name] = fn
    _LIBS[key] = (lib, fns)
    return _LIBS[key]


class OracleSim:
    """One channel on a CPU checker, mirroring the reference Simulation
    (create -> add capsules -> initialize -> step)."""

    def __init__(self, spec: ChannelSpec, impl: str = "sfo", fast: bool = False,
                 threads: int = 1):
        if impl == "sfo":
            if not os.path.exists(SFO_LIB):
                build(False)
            self._lib, self._fn = _load(SFO_LIB, "sfo_")
        elif impl == "ref":
            self._lib, self._fn = _load(REF_FAST_LIB if fast else REF_LIB, "sfr_")
            # one thread: the reference spread is order-dependent with more
            self._fn["set_threads"](threads)
        elif impl == "engine":
            # the reference's own Simulation object (deterministic build)
            self._lib, self._fn = _load(ENGINE_LIB, "sfe_")
            self._fn["set_threads"](threads)
        else:
            raise ValueError(impl)
        self.impl = impl
        self.spec = spec
        self._p = spec.to_c()
        self._h = self._fn["create"](C.byref(self._p))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._fn["destroy"](h)
            self._h = None

    # setup ------------------------------------------------------------
    def add_capsule(self, cx, cy, r, nn, m: Membrane, type_: int = 0) -> int:
        mc = m.to_c()
        return self._fn["add_capsule"](self._h, cx, cy, r, nn, C.byref(mc), type_)

    def add_capsule_random(self, count, x0, y0, x1, y1, rmin, rmax, nn, m: Membrane,
                           type_=0, seed=12345, min_gap=1.0, max_attempts=0,
                           check_walls=True) -> int:
        mc = m.to_c()
        return self._fn["add_capsule_random"](self._h, count, x0, y0, x1, y1, rmin, rmax, nn,
                                              C.byref(mc), type_, seed, min_gap, max_attempts,
                                              int(check_walls))

    def set_chemistry(self, **vectors):
        self._chem = chemistry_struct(**vectors)
        self._fn["set_chemistry"](self._h, C.byref(self._chem))

    def chemistry_state(self):
        """(released [caps], absorbed [caps], Mp [caps], gamma [markers])."""
        n, M = self.num_capsules, self.num_markers
        out = [np.zeros(max(n, 1)), np.zeros(max(n, 1)), np.zeros(max(n, 1)),
               np.zeros(max(M, 1))]
        dp = C.POINTER(C.c_double)
        self._fn["chemistry_state"](self._h, *[a.ctypes.data_as(dp) for a in out])
        return out[0][:n], out[1][:n], out[2][:n], out[3][:M]

    def add_circle_pillar(self, cx, cy, r):
        self._fn["add_circle_pillar"](self._h, cx, cy, r)

    def add_rect_pillar(self, x0, y0, x1, y1):
        self._fn["add_rect_pillar"](self._h, x0, y0, x1, y1)

    def initialize(self):
        self._fn["initialize"](self._h)

    def set_concentration(self, Cfield: np.ndarray):
        a = np.ascontiguousarray(Cfield, dtype=np.float64).ravel()
        self._fn["set_concentration"](self._h, a.ctypes.data_as(C.POINTER(C.c_double)))

    def step(self, n: int = 1):
        self._fn["step"](self._h, int(n))

    def set_threads(self, n: int) -> None:
        """OpenMP threads of the reference build (a setting of its library,
        shared by every simulation on it); the C restatement is serial."""
        if self.impl in ("ref", "engine"):
            self._fn["set_threads"](int(n))

    # state views (copies) -------------------------------------------
    def _arr(self, name, n):
        if n == 0:
            return np.zeros(0)
        ptr = self._fn[name](self._h)
        if not ptr:
            return None
        return np.ctypeslib.as_array(ptr, shape=(n,)).copy()

    @property
    def num_markers(self):
        return self._fn["num_markers"](self._h)

    @property
    def num_capsules(self):
        return self._fn["num_capsules"](self._h)

    def offsets(self):
        nc = self.num_capsules
        ptr = self._fn["capsule_offsets"](self._h)
        return np.ctypeslib.as_array(ptr, shape=(nc + 1,)).copy()

    def f(self):
        nx, ny = self.spec.nx, self.spec.ny
        return self._arr("f", 9 * nx * ny).reshape(9, ny, nx)

    def rho(self):
        return self._arr("rho", self.spec.nx * self.spec.ny).reshape(self.spec.ny, self.spec.nx)

    def ux(self):
        return self._arr("ux", self.spec.nx * self.spec.ny).reshape(self.spec.ny, self.spec.nx)

    def uy(self):
        return self._arr("uy", self.spec.nx * self.spec.ny).reshape(self.spec.ny, self.spec.nx)

    def Fx(self):
        return self._arr("Fx", self.spec.nx * self.spec.ny).reshape(self.spec.ny, self.spec.nx)

    def Fy(self):
        return self._arr("Fy", self.spec.nx * self.spec.ny).reshape(self.spec.ny, self.spec.nx)

    def positions(self):
        return self._arr("pos", 2 * self.num_markers).reshape(-1, 2)

    def velocities(self):
        return self._arr("vel", 2 * self.num_markers).reshape(-1, 2)

    def forces(self):
        return self._arr("force", 2 * self.num_markers).reshape(-1, 2)

    def concentration(self):
        a = self._arr("C", self.spec.nx * self.spec.ny)
        return None if a is None else a.reshape(self.spec.ny, self.spec.nx)

    def g(self):
        """Scalar populations in the reference's AoS layout [ny*nx][9]."""
        a = self._arr("g", 9 * self.spec.nx * self.spec.ny)
        return None if a is None else a.reshape(self.spec.ny, self.spec.nx, 9)

    def last_capped(self) -> int:
        return self._fn["last_capped"](self._h)

    def capsule_area(self, c):
        return self._fn["capsule_area"](self._h, c)

    def capsule_perimeter(self, c):
        return self._fn["capsule_perimeter"](self._h, c)

    def capsule_deformation(self, c):
        return self._fn["capsule_deformation"](self._h, c)

    def capsule_inclination(self, c):
        return self._fn["capsule_inclination"](self._h, c)

    def capsule_centroid(self, c):
        x, y = C.c_double(), C.c_double()
        self._fn["capsule_centroid"](self._h, c, C.byref(x), C.byref(y))
        return x.value, y.value

    def write_vtk(self, directory: str, step: int, legacy: bool):
        """The reference's VTKWriter on the current state (reference build
        only)."""
        self._fn["write_vtk"](self._h, directory.encode(), int(step), int(bool(legacy)))

    def write_global_stats(self, directory: str, step: int, time: float):
        """One row of the reference's GlobalStatsWriter (reference build only)."""
        self._fn["write_global_stats"](self._h, directory.encode(), int(step), float(time))

    def _view(self, name, n):
        ptr = self._fn[name](self._h)
        return np.ctypeslib.as_array(ptr, shape=(n,))

    def set_markers(self, pos=None, vel=None, force=None):
        """Overwrite marker state in place ([M][2] arrays)."""
        M = self.num_markers
        for name, arr in (("pos", pos), ("vel", vel), ("force", force)):
            if arr is not None:
                self._view(name, 2 * M)[:] = np.asarray(arr, dtype=np.float64).ravel()

    def spread(self, clear=True):
        """ImmersedBoundary::spreadForces on the current marker forces; returns
        (Fx, Fy).  Only the C restatement exposes this."""
        N = self.spec.nx * self.spec.ny
        if clear:
            self._view("Fx", N)[:] = 0.0
            self._view("Fy", N)[:] = 0.0
        self._fn["spread_forces"](self._h)
        return self.Fx(), self.Fy()

    def compute_membrane(self):
        """Capsule::computeMembraneForces on the current state (forces cleared
        first); the result is in forces()."""
        M = self.num_markers
        self._view("force", 2 * M)[:] = 0.0
        self._fn["compute_membrane_forces"](self._h)

    def contact_pairs(self):
        """(counts per marker, flat neighbour list) of the last contact pass."""
        M = self.num_markers
        counts = np.zeros(max(M, 1), dtype=np.int32)
        total = self._fn["contact_pairs"](self._h, counts.ctypes.data_as(C.POINTER(C.c_int)),
                                          None, 0)
        lst = np.zeros(max(total, 1), dtype=np.int32)
        self._fn["contact_pairs"](self._h, counts.ctypes.data_as(C.POINTER(C.c_int)),
                                  lst.ctypes.data_as(C.POINTER(C.c_int)), total)
        return counts[:M], lst[:total]


def phi(r: float, impl: str = "sfo") -> float:
    if impl == "sfo":
        if not os.path.exists(SFO_LIB):
            build(False)
        _, fn = _load(SFO_LIB, "sfo_")
    else:
        _, fn = _load(REF_LIB, "sfr_")
    return fn["phi"](r)


def ref_available() -> bool:
    return os.path.exists(REF_LIB)
