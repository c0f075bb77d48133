"""ctypes mirror of include/paracfd_b200.h and the loader for the in-tree native library.

The Python layer is a thin host: every compute call goes through the C ABI into
``libparacfd_b200.so`` (hand-written sm_100a kernels).  Loading fails loudly when the library
is missing; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libparacfd_b200.so")

PCFD_OK, PCFD_INVALID_ARG, PCFD_NOT_CONVERGED = 0, 1, 3
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "CUDA_ERROR", 3: "NOT_CONVERGED",
                4: "TOPOLOGY_UNRESOLVED", 5: "OUT_OF_MEMORY", 6: "TIMEOUT", 7: "INTERNAL"}

BRICK_XMIN, BRICK_XMAX, BRICK_YMIN, BRICK_YMAX, BRICK_ZMIN, BRICK_ZMAX = (1 << q for q in range(6))
BRICK_EMBEDDED_BOUNDARY, BRICK_COVERED = 1 << 6, 1 << 7

_i32p = C.POINTER(C.c_int32)
_u32p = C.POINTER(C.c_uint32)
_u8p = C.POINTER(C.c_uint8)
_i8p = C.POINTER(C.c_int8)
_f64p = C.POINTER(C.c_double)
_f32p = C.POINTER(C.c_float)


class Level(C.Structure):
    _fields_ = [("h", C.c_double), ("brick_count", C.c_int32), ("level_offset", C.c_int32),
                ("coord", _i32p), ("origin", _f64p), ("neighbors", _i32p), ("flags", _u32p),
                ("children", _i32p)]


class Connections(C.Structure):
    _fields_ = [("count", C.c_int32), ("coarse_dof", _i32p), ("fine_dof", _i32p),
                ("open_area", _f64p), ("centre_distance", _f64p), ("normal_distance", _f64p),
                ("axis", _i8p), ("direction", _i8p), ("face_centroid", _f64p),
                ("orthogonal_gradient_factor", _f64p), ("lower_gradient_node", _i32p),
                ("upper_gradient_node", _i32p), ("nonorthogonal_correction", _f64p),
                ("upper_gradient_weight", _f64p)]


class RegularCorrections(C.Structure):
    _fields_ = [("count", C.c_int32), ("lower_dof", _i32p), ("upper_dof", _i32p),
                ("level", _i32p), ("brick", _i32p), ("ijk", _i32p), ("axis", _i8p),
                ("open_area", _f64p), ("two_point_delta", _f64p),
                ("lower_gradient_node", _i32p), ("upper_gradient_node", _i32p),
                ("nonorthogonal_correction", _f64p), ("upper_gradient_weight", _f64p)]


class SurfacePatches(C.Structure):
    _fields_ = [("count", C.c_int32), ("area", _f64p), ("centroid", _f64p), ("normal", _f64p),
                ("plus_dof", _i32p), ("minus_dof", _i32p)]


class BoundaryFaces(C.Structure):
    _fields_ = [("count", C.c_int32), ("dof", _i32p), ("outward_area", _f64p),
                ("centroid", _f64p)]


class Topology(C.Structure):
    _fields_ = [("brick_size", C.c_int32), ("level_count", C.c_int32),
                ("levels", C.POINTER(Level)),
                ("domain_lo", C.c_double * 3), ("domain_hi", C.c_double * 3),
                ("storage_size", C.c_int32), ("pressure_outlet_xmax", C.c_int32),
                ("active", _u8p), ("freestream_connected", _u8p), ("cut_face_mask", _u8p),
                ("volume", _f64p), ("centroid", _f64p), ("preconditioner_aggregate", _i32p),
                ("coarse_fine", Connections), ("embedded", Connections),
                ("regular", RegularCorrections),
                ("gradient_node_count", C.c_int32), ("gradient_dof", _i32p),
                ("gradient_offset", _i32p), ("gradient_neighbour", _i32p),
                ("gradient_weight", _f64p),
                ("gauge_count", C.c_int32), ("gauge_dof", _i32p), ("gauge_coefficient", _f64p),
                ("patches", SurfacePatches), ("boundary_faces", BoundaryFaces),
                ("retained_count", C.c_int32), ("retained_dofs", _i32p)]


class Options(C.Structure):
    _fields_ = [("mg_precision", C.c_int32), ("device", C.c_int32), ("stream", C.c_void_p),
                ("momentum_min_volume_fraction", C.c_double), ("disable_fused_smoother", C.c_int32),
                ("mg_cycle", C.c_int32), ("gmres_restart", C.c_int32), ("mg_stage_sweeps", C.c_int32),
                ("mg_block_iterations", C.c_int32), ("mg_stage_chebyshev", C.c_int32), ("mg_fine_chebyshev", C.c_int32),
                ("gmres_delayed", C.c_int32), ("gmres_recycle", C.c_int32), ("mg_stage_fp16", C.c_int32),
                ("mg_stage_csr", C.c_int32)]


class SolveResult(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("relative_residual", C.c_double),
                ("converged", C.c_int32), ("preconditioner_applications", C.c_int32),
                ("recycle_rejections", C.c_int32), ("fallback_solves", C.c_int32)]

    def as_dict(self):
        return {"iterations": self.iterations, "relative_residual": self.relative_residual,
                "converged": bool(self.converged),
                "preconditioner_applications": self.preconditioner_applications,
                "recycle_rejections": self.recycle_rejections, "fallback_solves": self.fallback_solves}


class Case(C.Structure):
    _fields_ = [("speed", C.c_double), ("rho", C.c_double), ("nu", C.c_double), ("cfl", C.c_double),
                ("smagorinsky_cs", C.c_double), ("projection_tolerance", C.c_double),
                ("projection_max_iterations", C.c_int32), ("smooth_wall", C.c_int32),
                ("pressure_impulse", C.c_int32)]


class StepStats(C.Structure):
    _fields_ = [("dt", C.c_double), ("physical_time", C.c_double), ("max_abs_velocity", C.c_double),
                ("max_abs_special_velocity", C.c_double), ("max_outflow_rate", C.c_double),
                ("cfl_velocity", C.c_double), ("effective_cfl", C.c_double),
                ("max_diffusion_rate", C.c_double), ("diffusion_substeps", C.c_int32),
                ("pressure", SolveResult), ("step_ms", C.c_double), ("projection_ms", C.c_double)]

    def as_dict(self):
        out = {name: getattr(self, name) for name, _ in self._fields_ if name != "pressure"}
        out["pressure"] = self.pressure.as_dict()
        return out


class Loads(C.Structure):
    _fields_ = [("pressure_force", C.c_double * 3), ("pressure_moment", C.c_double * 3),
                ("viscous_force", C.c_double * 3), ("viscous_moment", C.c_double * 3),
                ("total_force", C.c_double * 3), ("total_moment", C.c_double * 3),
                ("cl", C.c_double), ("cd", C.c_double), ("cs", C.c_double)]

    def as_dict(self):
        out = {}
        for name, kind in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class ConservationStats(C.Structure):
    _fields_ = [("max_abs_divergence", C.c_double), ("volume_weighted_rms_divergence", C.c_double),
                ("worst_control_volume", C.c_double), ("max_integrated_flux_error", C.c_double),
                ("absolute_integrated_flux_error", C.c_double), ("net_integrated_flux_error", C.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class AutotuneReport(C.Structure):
    _fields_ = [("candidates", C.c_int32), ("ctas_per_sm", C.c_int32 * 8), ("apply_ms", C.c_double * 8),
                ("sweep_ms", C.c_double * 8), ("chosen", C.c_int32)]

    def as_dict(self):
        n = self.candidates
        return {"ctas_per_sm": list(self.ctas_per_sm[:n]), "apply_ms": [round(v, 5) for v in self.apply_ms[:n]],
                "sweep_ms": [round(v, 5) for v in self.sweep_ms[:n]], "chosen": self.chosen}


class Mesh(C.Structure):
    _fields_ = [("vertex_count", C.c_int64), ("positions", _f64p), ("triangle_count", C.c_int64),
                ("indices", _u32p)]


class AmrConfig(C.Structure):
    _fields_ = [("domain_lo", C.c_double * 3), ("domain_hi", C.c_double * 3), ("base_cell_size", C.c_double),
                ("max_levels", C.c_int32), ("brick_size", C.c_int32), ("wing_refinement_distance", C.c_double),
                ("surface_refinement_distance", C.c_double), ("wake_length", C.c_double),
                ("wake_radius", C.c_double), ("anchor_y_min", C.c_int32)]


def ptr(array: np.ndarray | None, ctype):
    """Pointer to a contiguous numpy array (None -> NULL)."""
    if array is None:
        return C.cast(None, C.POINTER(ctype))
    if not array.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return array.ctypes.data_as(C.POINTER(ctype))


# Exported symbols and their argument types; also the list the CPU tests check.
SIGNATURES = {
    "pcfd_last_error_message": (C.c_char_p, []),
    "pcfd_version": (C.c_char_p, []),
    "pcfd_system_create": (C.c_int, [C.POINTER(Topology), C.POINTER(Options), C.POINTER(C.c_void_p)]),
    "pcfd_system_destroy": (None, [C.c_void_p]),
    "pcfd_system_sizes": (C.c_int, [C.c_void_p] + [C.POINTER(C.c_int64)] * 5),
    "pcfd_system_synchronize": (C.c_int, [C.c_void_p]),
    "pcfd_pressure_apply_host": (C.c_int, [C.c_void_p, _f64p, _f64p, C.c_int32]),
    "pcfd_pressure_apply_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]),
    "pcfd_pressure_apply_device_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]),
    "pcfd_pressure_diagonal_host": (C.c_int, [C.c_void_p, _f64p]),
    "pcfd_pressure_precondition_host": (C.c_int, [C.c_void_p, _f64p, _f64p]),
    "pcfd_pressure_solve_host": (C.c_int, [C.c_void_p, _f64p, _f64p, C.c_double, C.c_int32,
                                           C.c_int32, C.POINTER(SolveResult)]),
    "pcfd_set_faces_host": (C.c_int, [C.c_void_p, _f32p, _f32p, _f32p]),
    "pcfd_get_faces_host": (C.c_int, [C.c_void_p, _f32p, _f32p, _f32p]),
    "pcfd_set_special_host": (C.c_int, [C.c_void_p, _f32p, _f32p]),
    "pcfd_get_special_host": (C.c_int, [C.c_void_p, _f32p, _f32p]),
    "pcfd_set_pressure_host": (C.c_int, [C.c_void_p, _f64p]),
    "pcfd_get_pressure_host": (C.c_int, [C.c_void_p, _f64p]),
    "pcfd_get_pressure_shadow_host": (C.c_int, [C.c_void_p, _f32p]),
    "pcfd_projection_divergence_host": (C.c_int, [C.c_void_p, _f32p]),
    "pcfd_projection_rhs_host": (C.c_int, [C.c_void_p, C.c_double, C.c_double, _f64p]),
    "pcfd_projection_correct": (C.c_int, [C.c_void_p, C.c_double, C.c_double]),
    "pcfd_projection_project": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double,
                                          C.c_int32, C.c_int32, C.POINTER(SolveResult)]),
    "pcfd_time_kernel": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double)]),
    "pcfd_momentum_set_state_host": (C.c_int, [C.c_void_p, _f32p, _f32p, _f32p]),
    "pcfd_momentum_get_state_host": (C.c_int, [C.c_void_p, _f32p, _f32p, _f32p]),
    "pcfd_momentum_transport": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_int32]),
    "pcfd_momentum_smagorinsky": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double,
                                            C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    "pcfd_momentum_smooth_wall": (C.c_int, [C.c_void_p, C.c_double, C.c_double]),
    "pcfd_momentum_wall_forces_host": (C.c_int, [C.c_void_p, _f32p, C.POINTER(C.c_int64)]),
    "pcfd_momentum_pressure_impulse": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_int32, C.c_int32]),
    "pcfd_momentum_reconstruct_fluxes": (C.c_int, [C.c_void_p]),
    "pcfd_apply_external_boundaries": (C.c_int, [C.c_void_p, C.c_double]),
    "pcfd_momentum_cfl": (C.c_int, [C.c_void_p, C.c_int32, _f64p]),
    "pcfd_core_configure": (C.c_int, [C.c_void_p, C.POINTER(Case)]),
    "pcfd_core_initialize": (C.c_int, [C.c_void_p, C.POINTER(StepStats)]),
    "pcfd_core_step": (C.c_int, [C.c_void_p, C.POINTER(StepStats)]),
    "pcfd_topology_build": (C.c_int, [C.POINTER(Mesh), C.POINTER(AmrConfig), C.c_int32, C.POINTER(C.c_void_p),
                                      C.POINTER(Topology)]),
    "pcfd_topology_free": (None, [C.c_void_p]),
    "pcfd_core_loads": (C.c_int, [C.c_void_p, C.c_double, _f64p, C.c_double, C.c_int32, C.POINTER(Loads)]),
    "pcfd_event_record": (C.c_int, [C.c_void_p, C.c_int32]),
    "pcfd_event_elapsed": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double)]),
    "pcfd_core_inflow_layout": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "pcfd_core_set_inflow_host": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int64]),
    "pcfd_launch_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "pcfd_preconditioner_fused": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "pcfd_stage_brick_structured": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "pcfd_profile_begin": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "pcfd_profile_end": (C.c_int, [C.c_void_p, _f64p, C.c_int32, C.POINTER(C.c_int32)]),
    "pcfd_builder_last_error": (C.c_char_p, []),
    "pcfd_set_preconditioner": (C.c_int, [C.c_void_p, C.c_int32]),
    "pcfd_projection_keep_start": (C.c_int, [C.c_void_p, C.c_int32]),
    "pcfd_core_set_initial_guess": (C.c_int, [C.c_void_p, C.c_int32]),
    "pcfd_projection_resolve": (C.c_int, [C.c_void_p, C.c_double, C.c_int32, C.POINTER(C.c_double),
                                          C.POINTER(SolveResult)]),
    "pcfd_learned_parameter_count": (C.c_int, [C.POINTER(C.c_int64)]),
    "pcfd_learned_set_parameters": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int64]),
    "pcfd_learned_get_parameters": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int64]),
    "pcfd_learned_harvest_begin": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_uint64, C.c_int32]),
    "pcfd_learned_harvest_stop": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "pcfd_learned_train": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_uint64, C.POINTER(C.c_double)]),
    "pcfd_learned_evaluate_host": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                             C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_float)]),
    "pcfd_learned_apply_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "pcfd_learned_set_wait": (C.c_int, [C.c_void_p, C.c_double, C.c_int32]),
    "pcfd_core_conservation_stats": (C.c_int, [C.c_void_p, C.POINTER(ConservationStats)]),
    "pcfd_profile_bytes": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]),
    "pcfd_autotune": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(AutotuneReport)]),
    "pcfd_locate_points_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "pcfd_sample_slice_host": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                         C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_float)]),
    "pcfd_mac_set_links": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint8), C.POINTER(C.c_uint8), C.POINTER(C.c_uint8)]),
    "pcfd_mac_advect": (C.c_int, [C.c_void_p, C.c_double]),
    "pcfd_mac_diffuse_smagorinsky": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double]),
    "pcfd_mac_eddy_viscosity_host": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "pcfd_mac_transport_apertures": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double]),
    "pcfd_core_set_momentum_mode": (C.c_int, [C.c_void_p, C.c_int32]),
    "pcfd_set_pipeline_ctas": (C.c_int, [C.c_void_p, C.c_int32]),
}

_lib = None


def load(path: str = LIBRARY_PATH):
    """Load the native library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"paracfd_b200 native library missing: {path}; run __graft_entry__.build()")
    lib = C.CDLL(path)
    for name, (restype, argtypes) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    _lib = lib
    return lib


class PcfdError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def check(status: int):
    if status != PCFD_OK:
        raise PcfdError(status, load().pcfd_last_error_message().decode(errors="replace"))
