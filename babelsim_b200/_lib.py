"""ctypes binding of libbabelsim_b200.so (the C ABI declared in include/babelsim_b200.h).

The library is built in-tree by ``python -m babelsim_b200.build``.  There is no
fallback: if the shared library is missing or cannot be loaded, every entry point
raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbabelsim_b200.so")

# Entry points declared in include/babelsim_b200.h, in declaration order.
EXPORTS = [
    "bsg_context_create", "bsg_context_destroy", "bsg_last_error", "bsg_global_error", "bsg_context_launches",
    "bsg_context_synchronize", "bsg_context_profile", "bsg_context_profile_report", "bsg_context_phase_log",
    "bsg_context_phase_log_read", "bsg_context_event_record",
    "bsg_context_event_elapsed", "bsg_mesh_create", "bsg_mesh_create_polyhedral", "bsg_mesh_create_polyhedral_host",
    "bsg_mesh_destroy", "bsg_mesh_create_from_file", "bsg_mesh_file_info", "bsg_mesh_locality_order",
    "bsg_mesh_validate_polyhedral", "bsg_write_results",
    "bsg_mesh_sizes", "bsg_mesh_export", "bsg_field_create", "bsg_field_destroy", "bsg_field_set_boundary",
    "bsg_field_upload", "bsg_field_download", "bsg_field_set_boundary_flux", "bsg_math_grad",
    "bsg_math_interpolate", "bsg_math_flux", "bsg_math_div_flux", "bsg_math_normal_gradient",
    "bsg_equation_create", "bsg_equation_destroy", "bsg_equ_reset", "bsg_equ_div", "bsg_equ_laplacian",
    "bsg_equ_source", "bsg_equ_ddt", "bsg_equ_reaction", "bsg_equ_apply", "bsg_equ_residual", "bsg_equ_relax", "bsg_equ_scale", "bsg_equ_reference_if_unanchored", "bsg_equ_face_flux",
    "bsg_equ_relative_residual", "bsg_equ_solve", "bsg_equ_download", "bsg_solve_ldu", "bsg_pcg_jacobi_static",
    "bsg_system_create", "bsg_system_destroy", "bsg_system_solve", "bsg_system_counters_read",
    "bsg_simple_create",
    "bsg_simple_set_boundary", "bsg_simple_set_fields", "bsg_simple_set_flux", "bsg_simple_load_state",
    "bsg_simple_iterate", "bsg_simple_set_segments", "bsg_simple_segment_report", "bsg_simple_enable_komega", "bsg_simple_enable_kepsilon",
    "bsg_simple_enable_spalart_allmaras", "bsg_simple_set_wall_distance", "bsg_simple_set_turbulence_fields",
    "bsg_simple_get_turbulence_fields", "bsg_simple_get_fields",
    "bsg_simple_destroy", "bsg_piso_create", "bsg_piso_set_boundary", "bsg_piso_set_fields", "bsg_piso_advance",
    "bsg_piso_get_fields", "bsg_piso_destroy", "bsg_piso_enable_komega", "bsg_piso_enable_kepsilon",
    "bsg_piso_enable_spalart_allmaras", "bsg_piso_set_wall_distance", "bsg_piso_set_turbulence_fields",
    "bsg_piso_get_turbulence_fields", "bsg_piso_initialize_potential_flow",
]


class Options(C.Structure):
    """bsg_options (OperatorOptions)."""
    _fields_ = [("interpolation", C.c_int32), ("gradient", C.c_int32), ("convection", C.c_int32),
                ("diffusion", C.c_int32), ("coefficient_interpolation", C.c_int32),
                ("coefficient_gradient", C.c_int32)]


class SolverConfig(C.Structure):
    """bsg_solver_config (LinearSolverConfig + precision)."""
    _fields_ = [("solver", C.c_int32), ("preconditioner", C.c_int32), ("absolute_tolerance", C.c_double),
                ("relative_tolerance", C.c_double), ("max_iterations", C.c_int32), ("warm_start", C.c_int32),
                ("preconditioner_rebuild_interval", C.c_int32),
                ("preconditioner_reuse_iteration_growth", C.c_double), ("amg_max_levels", C.c_int32),
                ("amg_coarse_size", C.c_int32), ("amg_smoothing_steps", C.c_int32), ("precision", C.c_int32)]


class SystemCounters(C.Structure):
    """bsg_system_counters (EquationPerformanceCounters of one persistent system)."""
    _fields_ = [("linear_solves", C.c_uint64), ("krylov_iterations", C.c_uint64),
                ("matrix_value_updates", C.c_uint64), ("rhs_only_solves", C.c_uint64),
                ("preconditioner_setups", C.c_uint64), ("preconditioner_reuses", C.c_uint64),
                ("preconditioner_retries", C.c_uint64), ("true_residual_checks", C.c_uint64),
                ("matrix_update_seconds", C.c_double), ("preconditioner_seconds", C.c_double),
                ("solve_seconds", C.c_double), ("last_status", C.c_int32), ("last_initial_residual", C.c_double),
                ("last_final_residual", C.c_double), ("last_relative_residual", C.c_double)]


class SolveResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("initial_residual", C.c_double),
                ("final_residual", C.c_double), ("relative_residual", C.c_double)]


class MeshGeometry(C.Structure):
    _fields_ = [("n_cells", C.c_int32), ("n_faces", C.c_int32), ("n_patches", C.c_int32),
                ("face_owner", C.c_void_p), ("face_neighbour", C.c_void_p), ("face_patch", C.c_void_p),
                ("face_area_vectors", C.c_void_p), ("face_centres", C.c_void_p), ("face_areas", C.c_void_p),
                ("face_normals", C.c_void_p), ("face_owner_weights", C.c_void_p),
                ("face_orthogonal_coefficients", C.c_void_p), ("face_non_orthogonal", C.c_void_p),
                ("face_skewness", C.c_void_p), ("cell_centres", C.c_void_p), ("cell_volumes", C.c_void_p),
                ("orthogonal_geometry", C.c_int32)]


class SimpleConfig(C.Structure):
    _fields_ = [("density", C.c_double), ("viscosity", C.c_double), ("velocity_relaxation", C.c_double),
                ("pressure_relaxation", C.c_double), ("non_orthogonal_corrections", C.c_int32),
                ("continuity_tolerance", C.c_double), ("velocity_tolerance", C.c_double),
                ("momentum_tolerance", C.c_double), ("pressure_correction_tolerance", C.c_double),
                ("momentum", Options), ("pressure", Options), ("momentum_solver", SolverConfig),
                ("pressure_solver", SolverConfig)]


class SimpleReport(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("status", C.c_int32), ("mass", C.c_double),
                ("dU", C.c_double), ("rU", C.c_double), ("dP", C.c_double),
                ("linear_pressure_residual", C.c_double), ("momentum_iterations", C.c_int32),
                ("pressure_iterations", C.c_int32), ("turbulence_change", C.c_double),
                ("turbulence_residual", C.c_double)]


class KOmegaConfig(C.Structure):
    _fields_ = [("beta_star", C.c_double), ("beta", C.c_double), ("gamma", C.c_double), ("sigma_k", C.c_double),
                ("sigma_omega", C.c_double), ("k_min", C.c_double), ("omega_min", C.c_double),
                ("max_viscosity_ratio", C.c_double), ("relaxation", C.c_double), ("tolerance", C.c_double),
                ("k_transport", Options), ("omega_transport", Options), ("k_solver", SolverConfig),
                ("omega_solver", SolverConfig)]


class PisoConfig(C.Structure):
    _fields_ = [("density", C.c_double), ("viscosity", C.c_double), ("velocity_relaxation", C.c_double),
                ("max_iterations", C.c_int32), ("correctors", C.c_int32), ("max_correctors", C.c_int32),
                ("coupling_tolerance", C.c_double), ("non_orthogonal_corrections", C.c_int32),
                ("continuity_tolerance", C.c_double), ("velocity_tolerance", C.c_double),
                ("momentum_tolerance", C.c_double), ("pressure_correction_tolerance", C.c_double),
                ("time_method", C.c_int32), ("start_time", C.c_double), ("end_time", C.c_double),
                ("delta_t", C.c_double), ("momentum", Options), ("pressure", Options),
                ("momentum_solver", SolverConfig), ("pressure_solver", SolverConfig)]


class PisoReport(C.Structure):
    _fields_ = [("steps", C.c_int32), ("time", C.c_double), ("status", C.c_int32), ("accepted", C.c_int32),
                ("mass", C.c_double), ("dU", C.c_double), ("rU", C.c_double), ("dP", C.c_double),
                ("coupling", C.c_double), ("courant_max", C.c_double), ("courant_mean", C.c_double),
                ("correctors", C.c_int32), ("momentum_iterations", C.c_int32), ("pressure_iterations", C.c_int32),
                ("turbulence_change", C.c_double), ("turbulence_residual", C.c_double),
                ("turbulence_corrections", C.c_int32)]


class PisoTurbulenceControls(C.Structure):
    _fields_ = [("coupling", C.c_int32), ("max_iterations", C.c_int32), ("correctors", C.c_int32)]


class KEpsilonConfig(C.Structure):
    _fields_ = [("c_mu", C.c_double), ("c1", C.c_double), ("c2", C.c_double), ("sigma_k", C.c_double),
                ("sigma_epsilon", C.c_double), ("k_min", C.c_double), ("epsilon_min", C.c_double),
                ("relaxation", C.c_double), ("tolerance", C.c_double), ("k_transport", Options),
                ("epsilon_transport", Options), ("k_solver", SolverConfig), ("epsilon_solver", SolverConfig)]


class SaConfig(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("cb1", "cb2", "sigma", "kappa", "cw1", "cw2", "cw3", "cv1", "ct3", "ct4",
                                          "nu_tilda_min", "wall_distance_min", "relaxation", "tolerance")] + \
        [("nu_tilda_transport", Options), ("nu_tilda_solver", SolverConfig)]


_lib = None


def lib():
    """Load the shared library once; raise if it is absent (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m babelsim_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        pp = C.POINTER(C.c_void_p)
        sig = {
            "bsg_context_create": [i32, pp], "bsg_context_destroy": [vp], "bsg_last_error": [vp],
            "bsg_global_error": [], "bsg_context_launches": [vp, C.POINTER(i64)], "bsg_context_synchronize": [vp],
            "bsg_context_profile": [vp, i32], "bsg_context_profile_report": [vp, C.c_char_p, i32],
            "bsg_context_phase_log": [vp, i32], "bsg_context_phase_log_read": [vp, vp, i32, C.POINTER(i32)],
            "bsg_context_event_record": [vp, i32], "bsg_context_event_elapsed": [vp, i32, i32, C.POINTER(dbl)],
            "bsg_simple_load_state": [vp, vp, vp, vp],
            "bsg_mesh_create": [vp, C.POINTER(MeshGeometry), pp],
            "bsg_mesh_create_polyhedral": [vp, i32, vp, i32, vp, vp, vp, vp, vp, i32, pp],
            "bsg_mesh_create_polyhedral_host": [vp, i32, vp, i32, vp, vp, vp, vp, vp, i32, pp],
            "bsg_mesh_destroy": [vp], "bsg_mesh_create_from_file": [vp, C.c_char_p, pp],
            "bsg_mesh_file_info": [C.c_char_p, vp, C.c_char_p, i32],
            "bsg_mesh_locality_order": [i32, i32, vp, vp, vp, C.POINTER(i32)], "bsg_mesh_sizes": [vp, vp], "bsg_mesh_export": [vp, C.c_char_p, vp],
            "bsg_mesh_validate_polyhedral": [i32, vp, i32, vp, vp, vp, vp, vp, i32, C.POINTER(i32), C.POINTER(i32)],
            "bsg_write_results": [C.c_char_p, C.c_char_p, i32, vp, i32, vp, vp, vp, vp, vp, i32, i32, vp, vp, vp],
            "bsg_field_create": [vp, i32, i32, pp], "bsg_field_destroy": [vp],
            "bsg_field_set_boundary": [vp, i32, i32, vp], "bsg_field_upload": [vp, vp],
            "bsg_field_download": [vp, vp], "bsg_field_set_boundary_flux": [vp, vp],
            "bsg_math_grad": [vp, i32, vp], "bsg_math_interpolate": [vp, C.POINTER(Options), vp],
            "bsg_math_flux": [vp, C.POINTER(Options), vp], "bsg_math_div_flux": [vp, vp],
            "bsg_math_normal_gradient": [vp, vp, C.POINTER(Options), vp],
            "bsg_equation_create": [vp, C.POINTER(Options), pp], "bsg_equation_destroy": [vp],
            "bsg_equ_reset": [vp], "bsg_equ_div": [vp, vp, dbl, C.POINTER(Options)],
            "bsg_equ_laplacian": [vp, vp, dbl, dbl, C.POINTER(Options)], "bsg_equ_source": [vp, vp, dbl],
            "bsg_equ_ddt": [vp, vp, dbl, vp, vp, dbl, dbl, i32], "bsg_equ_reaction": [vp, vp, dbl, dbl],
            "bsg_equ_apply": [vp, vp, vp], "bsg_equ_residual": [vp, vp, vp],
            "bsg_equ_relax": [vp, vp, dbl], "bsg_equ_scale": [vp, dbl],
            "bsg_equ_reference_if_unanchored": [vp, dbl, C.POINTER(i32)], "bsg_equ_face_flux": [vp, vp, vp],
            "bsg_equ_relative_residual": [vp, vp, C.POINTER(dbl)],
            "bsg_equ_solve": [vp, C.POINTER(SolverConfig), C.POINTER(SolveResult)],
            "bsg_equ_download": [vp, vp, vp, vp, vp],
            "bsg_solve_ldu": [vp, C.POINTER(SolverConfig), i32, vp, vp, vp, vp, vp, C.POINTER(SolveResult)],
            "bsg_pcg_jacobi_static": [i32, vp, vp, vp, vp, vp, vp, dbl, dbl, i32, C.POINTER(SolveResult)],
            "bsg_system_create": [vp, i32, pp], "bsg_system_destroy": [vp],
            "bsg_system_solve": [vp, C.POINTER(SolverConfig), vp, vp, vp, vp, vp, C.POINTER(SolveResult)],
            "bsg_system_counters_read": [vp, C.POINTER(SystemCounters)],
            "bsg_simple_create": [vp, C.POINTER(SimpleConfig), pp],
            "bsg_simple_set_boundary": [vp, C.c_char_p, i32, i32, vp], "bsg_simple_set_fields": [vp, vp, vp],
            "bsg_simple_set_flux": [vp, vp],
            "bsg_simple_iterate": [vp, i32, C.POINTER(SimpleReport)],
            "bsg_simple_set_segments": [vp, i32, vp, vp],
            "bsg_simple_segment_report": [vp, i32, C.POINTER(SimpleReport)],
            "bsg_simple_enable_komega": [vp, C.POINTER(KOmegaConfig)],
            "bsg_simple_enable_kepsilon": [vp, C.POINTER(KEpsilonConfig)],
            "bsg_simple_enable_spalart_allmaras": [vp, C.POINTER(SaConfig)],
            "bsg_simple_set_wall_distance": [vp, vp],
            "bsg_simple_set_turbulence_fields": [vp, vp, vp], "bsg_simple_get_turbulence_fields": [vp, vp, vp, vp], "bsg_simple_get_fields": [vp, vp, vp, vp],
            "bsg_simple_destroy": [vp],
            "bsg_piso_create": [vp, C.POINTER(PisoConfig), pp],
            "bsg_piso_set_boundary": [vp, C.c_char_p, i32, i32, vp], "bsg_piso_set_fields": [vp, vp, vp],
            "bsg_piso_advance": [vp, i32, C.POINTER(PisoReport)], "bsg_piso_get_fields": [vp, vp, vp, vp],
            "bsg_piso_destroy": [vp],
            "bsg_piso_enable_komega": [vp, C.POINTER(KOmegaConfig), C.POINTER(PisoTurbulenceControls)],
            "bsg_piso_enable_kepsilon": [vp, C.POINTER(KEpsilonConfig), C.POINTER(PisoTurbulenceControls)],
            "bsg_piso_enable_spalart_allmaras": [vp, C.POINTER(SaConfig), C.POINTER(PisoTurbulenceControls)],
            "bsg_piso_set_wall_distance": [vp, vp], "bsg_piso_set_turbulence_fields": [vp, vp, vp],
            "bsg_piso_get_turbulence_fields": [vp, vp, vp, vp], "bsg_piso_initialize_potential_flow": [vp, i32],
        }
        for name in EXPORTS:
            fn = getattr(L, name)
            fn.argtypes = sig[name]
            fn.restype = C.c_char_p if name in ("bsg_last_error", "bsg_global_error") else C.c_int
        _lib = L
    return _lib


class BsgError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"babelsim_b200 error {code}: {message}")
        self.code = code


def check(code, ctx=None):
    if code != 0:
        L = lib()
        msg = (L.bsg_last_error(ctx) if ctx else L.bsg_global_error()) or b""
        raise BsgError(code, msg.decode(errors="replace"))


def ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)
