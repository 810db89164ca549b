"""ctypes binding of libsoftflow_b200.so (include/softflow_gpu.h).

The library is built in-tree (``python -m softflow_b200.build``).  There is no
CPU fallback: if the library is missing or cannot be loaded, importing the
engine raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsoftflow_b200.so")

SFG_FP64, SFG_FP32, SFG_FP16S = 0, 1, 2
PRECISIONS = {"fp64": SFG_FP64, "fp32": SFG_FP32, "fp16s": SFG_FP16S}

STATUS_NAN_MARKER = 1
STATUS_LIST_OVERFLOW = 2
STATUS_CAPSULE_TOO_BIG = 4


class ChannelParamsC(C.Structure):
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


class MembraneParamsC(C.Structure):
    _fields_ = [
        ("model", C.c_int), ("k_stretch", C.c_double), ("G_s", C.c_double),
        ("C_skalak", C.c_double), ("wlc_L_max_ratio", C.c_double),
        ("wlc_kBT_p", C.c_double), ("wlc_k_pow", C.c_double), ("k_bend", C.c_double),
        ("use_helfrich", C.c_int), ("kappa_0", C.c_double), ("k_area", C.c_double),
        ("k_perimeter", C.c_double), ("gamma_visc", C.c_double), ("eta_membrane", C.c_double),
    ]


class CapsuleRestC(C.Structure):
    _fields_ = [
        ("num_nodes", C.c_int), ("rest_area", C.c_double), ("rest_perimeter", C.c_double),
        ("wlc_kBT_p", C.c_double), ("wlc_k_pow", C.c_double),
    ]


class ThermoRecordC(C.Structure):
    """sfg_thermo_record: per-channel reductions of the state."""
    _fields_ = [
        ("max_speed", C.c_double), ("mean_rho", C.c_double), ("mean_velocity", C.c_double),
        ("kinetic_energy", C.c_double), ("min_rho", C.c_double), ("max_rho", C.c_double),
        ("total_scalar", C.c_double), ("mean_deformation", C.c_double),
        ("max_deformation", C.c_double), ("fluid_cells", C.c_longlong),
        ("first_nonfinite", C.c_longlong), ("capped_nodes", C.c_longlong),
        ("num_capsules", C.c_int), ("reserved", C.c_int),
    ]


# sfg_capsule_stats: six doubles per capsule
CAPSULE_STATS_FIELDS = ("cx", "cy", "area", "perimeter", "deformation", "inclination")

THERMO_FN = C.CFUNCTYPE(C.c_int, C.c_longlong, C.POINTER(ThermoRecordC), C.c_int,
                        C.POINTER(C.c_double), C.c_int, C.c_void_p)


class ChemistryC(C.Structure):
    """sfg_chemistry: per capsule type vectors (8 entries, counts 0..8)."""
    _fields_ = [(n, C.c_int) for n in ("n_release", "n_absorb", "n_k_leach", "n_C_eq", "n_M_p",
                                       "n_k_adsorb", "n_k_desorb", "n_Gamma_max")] + \
               [(n, C.c_double * 8) for n in ("release", "absorb", "k_leach", "C_eq",
                                              "M_p_initial", "k_adsorb", "k_desorb",
                                              "Gamma_max")]


class SoftFlowGpuError(RuntimeError):
    """Raised when a C-ABI call returns a nonzero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[sfg status {code}] {message}")
        self.code = code


_lib = None

_P = C.POINTER
_D = _P(C.c_double)
_I = _P(C.c_int)
SIGNATURES = {
    "sfg_abi_version": (C.c_int, []),
    "sfg_last_error": (C.c_char_p, []),
    "sfg_build_circle_capsule": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_int,
                                           _P(MembraneParamsC), _P(CapsuleRestC), _D, _D, _D, _D,
                                           C.c_int]),
    "sfg_place_random": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                   C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int,
                                   C.c_int, C.c_int, C.c_int, C.c_int, _D, _D, C.c_int, _D, _D,
                                   _I, _I]),
    "sfg_place_random_pillars": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double,
                                           C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                           C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.c_int, _D, _D, C.c_int, _D, _D, _I, _I, C.c_int,
                                           _D]),
    "sfg_create": (C.c_int, [C.c_int, C.c_int, _P(C.c_void_p)]),
    "sfg_destroy": (C.c_int, [C.c_void_p]),
    "sfg_add_channel": (C.c_int, [C.c_void_p, _P(ChannelParamsC), _I]),
    "sfg_add_capsule": (C.c_int, [C.c_void_p, C.c_int, _P(MembraneParamsC), _P(CapsuleRestC),
                                  _D, _D, _D, _D, _I]),
    "sfg_initialize": (C.c_int, [C.c_void_p]),
    "sfg_step": (C.c_int, [C.c_void_p, C.c_int]),
    "sfg_synchronize": (C.c_int, [C.c_void_p, _P(C.c_uint)]),
    "sfg_get_populations": (C.c_int, [C.c_void_p, C.c_int, _D]),
    "sfg_set_populations": (C.c_int, [C.c_void_p, C.c_int, _D]),
    "sfg_set_all_populations": (C.c_int, [C.c_void_p, _D]),
    "sfg_get_macroscopic": (C.c_int, [C.c_void_p, C.c_int, _D, _D, _D, _D, _D]),
    "sfg_get_markers": (C.c_int, [C.c_void_p, C.c_int, _D, _D, _D]),
    "sfg_set_markers": (C.c_int, [C.c_void_p, C.c_int, _D, _D]),
    "sfg_get_all_markers": (C.c_int, [C.c_void_p, _D, _D]),
    "sfg_set_concentration": (C.c_int, [C.c_void_p, C.c_int, _D]),
    "sfg_get_concentration": (C.c_int, [C.c_void_p, C.c_int, _D, _D]),
    "sfg_get_capped_count": (C.c_int, [C.c_void_p, C.c_int, _I]),
    "sfg_get_contact_counts": (C.c_int, [C.c_void_p, C.c_int, _I]),
    "sfg_num_channels": (C.c_int, [C.c_void_p, _I]),
    "sfg_channel_counts": (C.c_int, [C.c_void_p, C.c_int, _I, _I]),
    "sfg_step_count": (C.c_int, [C.c_void_p, _P(C.c_longlong)]),
    "sfg_launches_per_step": (C.c_int, [C.c_void_p, _I]),
    "sfg_last_step_ms": (C.c_int, [C.c_void_p, _P(C.c_float)]),
    "sfg_get_stream": (C.c_int, [C.c_void_p, _P(C.c_void_p)]),
    "sfg_spread_forces": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "sfg_spread_forces_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                            C.c_void_p]),
    "sfg_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "sfg_set_lattice_variant": (C.c_int, [C.c_void_p, C.c_int]),
    "sfg_get_phase_times": (C.c_int, [C.c_void_p, _P(C.c_float), C.c_int]),
    "sfg_reset_phase_times": (C.c_int, [C.c_void_p]),
    "sfg_mlp_create": (C.c_int, [C.c_int, _P(C.c_void_p)]),
    "sfg_mlp_destroy": (C.c_int, [C.c_void_p]),
    "sfg_mlp_set_params": (C.c_int, [C.c_void_p, _P(C.c_float)]),
    "sfg_mlp_get_params": (C.c_int, [C.c_void_p, _P(C.c_float)]),
    "sfg_mlp_set_normalization": (C.c_int, [C.c_void_p, _P(C.c_float), _P(C.c_float),
                                            _P(C.c_float), _P(C.c_float)]),
    "sfg_mlp_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "sfg_mlp_gradients": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                    _P(C.c_float), _P(C.c_float), C.c_void_p]),
    "sfg_mlp_train": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float,
                                _P(C.c_float), C.c_void_p]),
    "sfg_mlp_step_count": (C.c_int, [C.c_void_p, _P(C.c_int)]),
    "sfg_set_mdf_model": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double]),
    "sfg_get_mdf_stats": (C.c_int, [C.c_void_p, C.c_int, _P(C.c_float), _P(C.c_float),
                                    _P(C.c_longlong), _P(C.c_longlong)]),
    "sfg_autotune": (C.c_int, [C.c_void_p, C.c_int, _P(C.c_int)]),
    "sfg_thermo": (C.c_int, [C.c_void_p, _P(ThermoRecordC), _D]),
    "sfg_get_all_markers_async": (C.c_int, [C.c_void_p, C.c_int, _D, _D]),
    "sfg_wait_markers": (C.c_int, [C.c_void_p, C.c_int]),
    "sfg_set_chemistry": (C.c_int, [C.c_void_p, C.c_int, _P(ChemistryC)]),
    "sfg_set_capsule_type": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "sfg_get_chemistry_state": (C.c_int, [C.c_void_p, C.c_int, _D, _D, _D, _D]),
    "sfg_add_pillar": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double,
                                 C.c_double, C.c_double]),
    "sfg_write_vtk_fluid": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p, C.c_int, C.c_int,
                                      C.c_uint]),
    "sfg_write_vtk_capsules": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p, C.c_int, C.c_int,
                                         _I]),
    "sfg_set_scalar_state": (C.c_int, [C.c_void_p, C.c_int, _D, _D]),
    "sfg_mark_restored": (C.c_int, [C.c_void_p]),
    "sfg_get_channel_params": (C.c_int, [C.c_void_p, C.c_int, _P(ChannelParamsC)]),
    "sfg_get_capsule_nodes": (C.c_int, [C.c_void_p, C.c_int, _I]),
    "sfg_get_capsule_base": (C.c_int, [C.c_void_p, C.c_int, _I]),
    "sfg_run": (C.c_int, [C.c_void_p, C.c_int, C.c_int, THERMO_FN, C.c_void_p, _P(C.c_int)]),
    "sfg_get_launch_config": (C.c_int, [C.c_void_p, _P(C.c_int), _P(C.c_int), _P(C.c_int),
                                        _P(C.c_int)]),
    "sfg_set_harvest": (C.c_int, [C.c_void_p, C.c_int]),
    "sfg_get_harvest": (C.c_int, [C.c_void_p, _P(C.c_float), _P(C.c_float), _P(C.c_int)]),
}

PHASES = ["membrane", "contact", "ibm_tiles", "ibm_spread", "mdf_interp", "lattice",
          "bookkeeping", "interp_move", "mdf_learned"]


def lib():
    """Load the library (once).  Raises if it is missing: no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing; build it with `python -m softflow_b200.build`")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(code: int) -> None:
    if code != 0:
        msg = lib().sfg_last_error().decode(errors="replace")
        raise SoftFlowGpuError(code, msg)


def dptr(a):
    """numpy float64 array -> double* (None passes through)."""
    if a is None:
        return None
    return a.ctypes.data_as(_D)


def iptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(_I)
