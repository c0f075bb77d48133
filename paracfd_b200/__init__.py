"""paracfd_b200 -- B200-native (sm_100a) ParaCFD per-timestep solver path.

Host mirror of the reference's device classes (DeviceCompositeAmrPressureOperator / Solver,
DeviceCompositeAmrProjection, reference src/core/fluid/amr_pressure.h:292-584) over the C ABI
in include/paracfd_b200.h.  All compute runs in ``libparacfd_b200.so``; this module only moves
host arrays across the boundary.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .capi import Options, SolveResult, Topology, check, ptr

PROFILE_STRUCTURED_APPLY = 0
PROFILE_PRECONDITIONER = 1
PROFILE_STAGE_SMOOTH = 2
MG_FP64, MG_FP32 = 0, 1
MG_CYCLE_REFERENCE, MG_CYCLE_CORRECTED, MG_CYCLE_COMPOSITE = 0, 1, 2
PRECONDITIONER_MULTIGRID, PRECONDITIONER_LEARNED, PRECONDITIONER_JACOBI, PRECONDITIONER_LEARNED_MULTIGRID = 0, 1, 2, 3
LEARNED_TARGET_MULTIGRID, LEARNED_TARGET_BRICK_SOLVE = 0, 1
MOMENTUM_CELL, MOMENTUM_MAC = 0, 1


def learned_parameter_count() -> int:
    n = C.c_int64()
    check(capi.load().pcfd_learned_parameter_count(C.byref(n)))
    return n.value


class BuiltTopology:
    """Brick hierarchy + composite pressure system built from a closed wing surface
    (``pcfd_topology_build``).  ``topology`` is the C view consumed by CompositeSystem."""

    def __init__(self, vertices: np.ndarray, triangles: np.ndarray, domain_lo, domain_hi, base_cell_size: float,
                 max_levels: int, brick_size: int = 8, wing_refinement_distance: float = 1.0,
                 surface_refinement_distance: float = 0.35, wake_length: float = 8.0, wake_radius: float = 2.0,
                 anchor_y_min: bool = False, solid: bool = True):
        self._lib = capi.load()
        self._vertices = np.ascontiguousarray(vertices, np.float64)
        self._triangles = np.ascontiguousarray(triangles, np.uint32)
        mesh = capi.Mesh(len(self._vertices), ptr(self._vertices, C.c_double), len(self._triangles),
                         ptr(self._triangles, C.c_uint32))
        cfg = capi.AmrConfig()
        cfg.domain_lo[:] = list(domain_lo)
        cfg.domain_hi[:] = list(domain_hi)
        cfg.base_cell_size = base_cell_size
        cfg.max_levels = max_levels
        cfg.brick_size = brick_size
        cfg.wing_refinement_distance = wing_refinement_distance
        cfg.surface_refinement_distance = surface_refinement_distance
        cfg.wake_length = wake_length
        cfg.wake_radius = wake_radius
        cfg.anchor_y_min = int(anchor_y_min)
        self.config = cfg
        self.topology = Topology()
        handle = C.c_void_p()
        status = self._lib.pcfd_topology_build(C.byref(mesh), C.byref(cfg), int(solid), C.byref(handle), C.byref(self.topology))
        if status != capi.PCFD_OK:
            raise capi.PcfdError(status, self._lib.pcfd_builder_last_error().decode(errors="replace"))
        self.handle = handle
        t = self.topology
        self.storage_size = t.storage_size
        self.brick_counts = [t.levels[l].brick_count for l in range(t.level_count)]
        self.active = np.ctypeslib.as_array(t.active, shape=(t.storage_size,))
        self.leaf_cells = int(self.active.sum())

    def close(self):
        if getattr(self, "handle", None):
            self._lib.pcfd_topology_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CompositeSystem:
    """Resident topology + state on one GPU (one host thread at a time)."""

    def __init__(self, topology: Topology, mg_precision: int = MG_FP64, device: int = 0,
                 momentum_min_volume_fraction: float = 0.0, fused_smoother: bool = True,
                 mg_cycle: int = 0, gmres_restart: int = 0, mg_stage_sweeps: int = 0, mg_block_iterations: int = 0,
                 mg_stage_chebyshev: int = 0, mg_fine_chebyshev: int = 0, gmres_delayed: int = 0,
                 gmres_recycle: int = 0, mg_stage_fp16: int = 0, mg_stage_csr: int = 0):
        self._lib = capi.load()
        self._topology = topology   # keep the caller's arrays alive during creation
        opts = Options(mg_precision, device, None, momentum_min_volume_fraction, 0 if fused_smoother else 1, mg_cycle,
                       gmres_restart, mg_stage_sweeps, mg_block_iterations, mg_stage_chebyshev, mg_fine_chebyshev,
                       gmres_delayed, gmres_recycle, mg_stage_fp16, mg_stage_csr)
        handle = C.c_void_p()
        check(self._lib.pcfd_system_create(C.byref(topology), C.byref(opts), C.byref(handle)))
        self.handle = handle
        sizes = [C.c_int64() for _ in range(5)]
        check(self._lib.pcfd_system_sizes(self.handle, *[C.byref(x) for x in sizes]))
        self.storage_size, self.bricks, self.faces, self.coarse_fine_count, self.embedded_count = (x.value for x in sizes)
        per_brick = self.faces // max(self.bricks, 1)
        self.brick_size = next((b for b in range(1, 65) if (b + 1) * b * b == per_brick), 0)

    def close(self):
        if getattr(self, "handle", None):
            self._lib.pcfd_system_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- pressure operator / solver -------------------------------------------------------
    def _vec(self, x, dtype=np.float64):
        x = np.ascontiguousarray(x, dtype=dtype)
        if x.shape != (self.storage_size,):
            raise ValueError(f"expected a vector of {self.storage_size} DOFs")
        return x

    def apply(self, p, orthogonal: bool = False) -> np.ndarray:
        p = self._vec(p)
        out = np.empty(self.storage_size)
        check(self._lib.pcfd_pressure_apply_host(self.handle, ptr(p, C.c_double), ptr(out, C.c_double), int(orthogonal)))
        return out

    def diagonal(self) -> np.ndarray:
        out = np.empty(self.storage_size)
        check(self._lib.pcfd_pressure_diagonal_host(self.handle, ptr(out, C.c_double)))
        return out

    def precondition(self, r) -> np.ndarray:
        r = self._vec(r)
        out = np.empty(self.storage_size)
        check(self._lib.pcfd_pressure_precondition_host(self.handle, ptr(r, C.c_double), ptr(out, C.c_double)))
        return out

    def solve(self, b, tolerance: float, max_iterations: int, x0=None):
        b = self._vec(b)
        x = self._vec(x0).copy() if x0 is not None else np.zeros(self.storage_size)
        res = SolveResult()
        check(self._lib.pcfd_pressure_solve_host(self.handle, ptr(x, C.c_double), ptr(b, C.c_double), tolerance,
                                                 max_iterations, int(x0 is not None), C.byref(res)))
        return x, res.as_dict()

    def set_initial_guess(self, mode: int):
        """Step projections start from the last pressure (0, the reference's warm start), from
        2 p_n - p_(n-1) of the last two converged pressures (1) or from 3 p_n - 3 p_(n-1) + p_(n-2)
        of the last three (2)."""
        check(self._lib.pcfd_core_set_initial_guess(self.handle, int(mode)))

    def keep_projection_start(self, keep: bool = True):
        check(self._lib.pcfd_projection_keep_start(self.handle, int(keep)))

    def resolve_projection(self, tolerance: float, max_iterations: int):
        """The last projection solved again from its saved start: (device ms, solve result)."""
        ms = C.c_double()
        res = SolveResult()
        status = self._lib.pcfd_projection_resolve(self.handle, tolerance, max_iterations, C.byref(ms), C.byref(res))
        if status not in (capi.PCFD_OK, capi.PCFD_NOT_CONVERGED):
            check(status)
        return ms.value, res.as_dict()

    # ---- learned preconditioner ---------------------------------------------------------------
    def set_preconditioner(self, kind: int):
        check(self._lib.pcfd_set_preconditioner(self.handle, kind))

    def learned_parameters(self) -> np.ndarray:
        out = np.empty(learned_parameter_count(), np.float32)
        check(self._lib.pcfd_learned_get_parameters(self.handle, ptr(out, C.c_float), len(out)))
        return out

    def set_learned_parameters(self, params):
        params = np.ascontiguousarray(params, np.float32)
        check(self._lib.pcfd_learned_set_parameters(self.handle, ptr(params, C.c_float), len(params)))

    def harvest_begin(self, capacity_pairs: int, bricks_per_pair: int, seed: int = 1, target: int = 1):
        """target: LEARNED_TARGET_BRICK_SOLVE (default) or LEARNED_TARGET_MULTIGRID."""
        check(self._lib.pcfd_learned_harvest_begin(self.handle, capacity_pairs, bricks_per_pair, seed, target))

    def harvest_stop(self) -> int:
        n = C.c_int64()
        check(self._lib.pcfd_learned_harvest_stop(self.handle, C.byref(n)))
        return n.value

    def train(self, steps: int, batch: int = 32, learning_rate: float = 1e-3, seed: int = 1) -> float:
        loss = C.c_double()
        check(self._lib.pcfd_learned_train(self.handle, steps, batch, learning_rate, seed, C.byref(loss)))
        return loss.value

    def learned_evaluate(self, inputs, targets, gradients: bool = True):
        """inputs [n,512,2] (D^-1 r / s, mask), targets [n,512] -> (loss, zhat [n,512], grads or None)."""
        inputs = np.ascontiguousarray(inputs, np.float32)
        targets = np.ascontiguousarray(targets, np.float32)
        n = inputs.shape[0]
        zhat = np.empty((n, 512), np.float32)
        grads = np.empty(learned_parameter_count(), np.float32) if gradients else None
        loss = C.c_double()
        check(self._lib.pcfd_learned_evaluate_host(self.handle, n, ptr(inputs, C.c_float), ptr(targets, C.c_float),
                                                   ptr(zhat, C.c_float), C.byref(loss), ptr(grads, C.c_float)))
        return loss.value, zhat, grads

    # ---- resident state ---------------------------------------------------------------------
    def set_faces(self, u, v, w):
        u, v, w = (np.ascontiguousarray(a, np.float32) for a in (u, v, w))
        check(self._lib.pcfd_set_faces_host(self.handle, ptr(u, C.c_float), ptr(v, C.c_float), ptr(w, C.c_float)))

    def get_faces(self):
        u, v, w = (np.empty(self.faces, np.float32) for _ in range(3))
        check(self._lib.pcfd_get_faces_host(self.handle, ptr(u, C.c_float), ptr(v, C.c_float), ptr(w, C.c_float)))
        return u, v, w

    # ---- staggered MAC momentum mode (DeviceAmrAdvection) ----
    def set_mac_links(self, links_u, links_v, links_w):
        """Per-face link bytes [faces] each: bits 0..5 open same-side links, bit 6 near-fabric band."""
        lu, lv, lw = (np.ascontiguousarray(a, np.uint8) for a in (links_u, links_v, links_w))
        check(self._lib.pcfd_mac_set_links(self.handle, ptr(lu, C.c_uint8), ptr(lv, C.c_uint8), ptr(lw, C.c_uint8)))

    def mac_advect(self, dt: float):
        check(self._lib.pcfd_mac_advect(self.handle, dt))

    def mac_diffuse_smagorinsky(self, nu: float, cs: float, dt: float):
        check(self._lib.pcfd_mac_diffuse_smagorinsky(self.handle, nu, cs, dt))

    def set_momentum_mode(self, mode: int):
        """MOMENTUM_CELL (default) or MOMENTUM_MAC for initialize / step; re-initialize afterwards."""
        check(self._lib.pcfd_core_set_momentum_mode(self.handle, mode))

    def mac_transport_apertures(self, dt: float, nu: float, cs: float):
        check(self._lib.pcfd_mac_transport_apertures(self.handle, dt, nu, cs))

    def mac_eddy_viscosity(self) -> np.ndarray:
        out = np.empty(self.storage_size, np.float32)
        check(self._lib.pcfd_mac_eddy_viscosity_host(self.handle, ptr(out, C.c_float)))
        return out

    def set_special(self, coarse_fine, embedded):
        cf = np.ascontiguousarray(coarse_fine, np.float32)
        eb = np.ascontiguousarray(embedded, np.float32)
        check(self._lib.pcfd_set_special_host(self.handle, ptr(cf, C.c_float), ptr(eb, C.c_float)))

    def get_special(self):
        cf = np.empty(self.coarse_fine_count, np.float32)
        eb = np.empty(self.embedded_count, np.float32)
        check(self._lib.pcfd_get_special_host(self.handle, ptr(cf, C.c_float), ptr(eb, C.c_float)))
        return cf, eb

    def set_pressure(self, p):
        p = self._vec(p)
        check(self._lib.pcfd_set_pressure_host(self.handle, ptr(p, C.c_double)))

    def get_pressure(self) -> np.ndarray:
        out = np.empty(self.storage_size)
        check(self._lib.pcfd_get_pressure_host(self.handle, ptr(out, C.c_double)))
        return out

    def get_pressure_shadow(self) -> np.ndarray:
        out = np.empty(self.storage_size, np.float32)
        check(self._lib.pcfd_get_pressure_shadow_host(self.handle, ptr(out, C.c_float)))
        return out

    def time_kernel(self, which: int, iterations: int = 20) -> float:
        """Milliseconds per launch sequence, CUDA events on the system stream."""
        ms = C.c_double()
        check(self._lib.pcfd_time_kernel(self.handle, which, iterations, C.byref(ms)))
        return ms.value

    # ---- projection -------------------------------------------------------------------------
    def divergence(self) -> np.ndarray:
        out = np.empty(self.storage_size, np.float32)
        check(self._lib.pcfd_projection_divergence_host(self.handle, ptr(out, C.c_float)))
        return out

    def projection_rhs(self, rho: float, dt: float) -> np.ndarray:
        out = np.empty(self.storage_size)
        check(self._lib.pcfd_projection_rhs_host(self.handle, rho, dt, ptr(out, C.c_double)))
        return out

    def correct_fluxes(self, rho: float, dt: float):
        check(self._lib.pcfd_projection_correct(self.handle, rho, dt))

    def project(self, rho: float, dt: float, tolerance: float, max_iterations: int, warm_start: bool = False):
        res = SolveResult()
        status = self._lib.pcfd_projection_project(self.handle, rho, dt, tolerance, max_iterations, int(warm_start), C.byref(res))
        if status not in (capi.PCFD_OK, 3):   # 3 = NOT_CONVERGED is reported in the result
            check(status)
        return res.as_dict()

    # ---- cell momentum ---------------------------------------------------------------------------
    def set_state(self, x, y, z):
        x, y, z = (self._vec(a, np.float32) for a in (x, y, z))
        check(self._lib.pcfd_momentum_set_state_host(self.handle, ptr(x, C.c_float), ptr(y, C.c_float), ptr(z, C.c_float)))

    def get_state(self):
        x, y, z = (np.empty(self.storage_size, np.float32) for _ in range(3))
        check(self._lib.pcfd_momentum_get_state_host(self.handle, ptr(x, C.c_float), ptr(y, C.c_float), ptr(z, C.c_float)))
        return x, y, z

    def transport(self, dt: float, freestream: float = 0.0, external_aero: bool = False):
        check(self._lib.pcfd_momentum_transport(self.handle, dt, freestream, int(external_aero)))

    def smagorinsky(self, nu: float, cs: float, dt: float):
        rate, sub = C.c_double(), C.c_int32()
        check(self._lib.pcfd_momentum_smagorinsky(self.handle, nu, cs, dt, C.byref(rate), C.byref(sub)))
        return rate.value, sub.value

    def smooth_wall(self, dt: float, nu: float):
        check(self._lib.pcfd_momentum_smooth_wall(self.handle, dt, nu))

    def wall_forces(self) -> np.ndarray:
        sides = C.c_int64()
        check(self._lib.pcfd_momentum_wall_forces_host(self.handle, ptr(None, C.c_float), C.byref(sides)))
        out = np.empty(3 * sides.value, np.float32)
        check(self._lib.pcfd_momentum_wall_forces_host(self.handle, ptr(out, C.c_float), C.byref(sides)))
        return out.reshape(-1, 3)

    def pressure_impulse(self, dt: float, rho: float, physical_boundaries: bool = True, redistribute: bool = True):
        check(self._lib.pcfd_momentum_pressure_impulse(self.handle, dt, rho, int(physical_boundaries), int(redistribute)))

    def reconstruct_fluxes(self):
        check(self._lib.pcfd_momentum_reconstruct_fluxes(self.handle))

    def apply_external_boundaries(self, speed: float):
        check(self._lib.pcfd_apply_external_boundaries(self.handle, speed))

    def cfl(self, external_aero: bool = True):
        out = np.zeros(3)
        check(self._lib.pcfd_momentum_cfl(self.handle, int(external_aero), ptr(out, C.c_double)))
        return {"max_abs_velocity": out[0], "max_outflow_rate": out[1], "max_abs_special_velocity": out[2]}

    # ---- time step (ExternalAeroCore surface) --------------------------------------------------
    def configure(self, speed=10.0, rho=1.225, nu=1.5e-5, cfl=0.5, smagorinsky_cs=0.10,
                  projection_tolerance=1e-8, projection_max_iterations=600, smooth_wall=True,
                  pressure_impulse=True):
        case = capi.Case(speed, rho, nu, cfl, smagorinsky_cs, projection_tolerance, projection_max_iterations,
                         int(smooth_wall), int(pressure_impulse))
        check(self._lib.pcfd_core_configure(self.handle, C.byref(case)))

    def initialize(self) -> dict:
        stats = capi.StepStats()
        check(self._lib.pcfd_core_initialize(self.handle, C.byref(stats)))
        return stats.as_dict()

    def step(self) -> dict:
        stats = capi.StepStats()
        status = self._lib.pcfd_core_step(self.handle, C.byref(stats))
        if status not in (capi.PCFD_OK, 3):
            check(status)
        return stats.as_dict()

    def loads(self, pressure_reference: float = 0.0, moment_origin=(0.0, 0.0, 0.0), reference_area: float = 0.0,
              include_viscous: bool = True) -> dict:
        out = capi.Loads()
        origin = np.ascontiguousarray(moment_origin, np.float64)
        check(self._lib.pcfd_core_loads(self.handle, pressure_reference, ptr(origin, C.c_double), reference_area,
                                        int(include_viscous), C.byref(out)))
        return out.as_dict()

    def conservation_stats(self) -> dict:
        """ExternalAeroCore::conservation_stats of the resident divergence."""
        out = capi.ConservationStats()
        check(self._lib.pcfd_core_conservation_stats(self.handle, C.byref(out)))
        return out.as_dict()

    def profile_bytes(self, region: int) -> float:
        """Algorithmic bytes of one launch of a profiled region (pcfd_profile_bytes)."""
        out = C.c_double()
        check(self._lib.pcfd_profile_bytes(self.handle, region, C.byref(out)))
        return out.value

    def autotune(self, iterations: int = 10) -> dict:
        """Picks the brick pipeline's resident CTAs per SM by timing (pcfd_autotune)."""
        out = capi.AutotuneReport()
        check(self._lib.pcfd_autotune(self.handle, iterations, C.byref(out)))
        return out.as_dict()

    def set_pipeline_ctas(self, ctas_per_sm: int):
        check(self._lib.pcfd_set_pipeline_ctas(self.handle, ctas_per_sm))

    def sample_slice(self, origin, edge_u, edge_v, nu: int, nv: int, field: int = 0) -> np.ndarray:
        """Headless slice [nv, nu] of the resident state (field 0 |v|, 1..3 v_x..v_z, 4 pressure)."""
        o, u, v = (np.ascontiguousarray(a, np.float64) for a in (origin, edge_u, edge_v))
        out = np.empty((nv, nu), np.float32)
        check(self._lib.pcfd_sample_slice_host(self.handle, ptr(o, C.c_double), ptr(u, C.c_double), ptr(v, C.c_double), nu, nv,
                                               field, ptr(out, C.c_float)))
        return out

    def event_record(self, slot: int):
        check(self._lib.pcfd_event_record(self.handle, slot))

    def event_elapsed(self, start: int, stop: int) -> float:
        ms = C.c_double()
        check(self._lib.pcfd_event_elapsed(self.handle, start, stop, C.byref(ms)))
        return ms.value

    def inflow_layout(self) -> np.ndarray:
        """Brick slots of the X-min inflow faces; face (j, k) of brick n is n*bs*bs + k*bs + j."""
        count = C.c_int64()
        check(self._lib.pcfd_core_inflow_layout(self.handle, C.byref(count), None))
        slots = np.empty(count.value // (self.brick_size ** 2) if count.value else 0, np.int32)
        check(self._lib.pcfd_core_inflow_layout(self.handle, C.byref(count), ptr(slots, C.c_int32)))
        return slots

    def set_inflow(self, normal_velocity) -> None:
        """Per-face X-min inflow (float32, inflow_layout order); None restores the uniform freestream."""
        if normal_velocity is None:
            check(self._lib.pcfd_core_set_inflow_host(self.handle, None, 0))
            return
        check(self._lib.pcfd_core_set_inflow_host(self.handle, ptr(normal_velocity, C.c_float), normal_velocity.size))

    def synchronize(self) -> None:
        """Wait for all work queued on the system stream."""
        check(self._lib.pcfd_system_synchronize(self.handle))

    @property
    def fused_preconditioner(self) -> bool:
        flag = C.c_int32()
        check(self._lib.pcfd_preconditioner_fused(self.handle, C.byref(flag)))
        return bool(flag.value)

    @property
    def stage_brick_structured(self) -> bool:
        """Whether the composite cycle's first stage runs in brick-structured form."""
        flag = C.c_int32()
        check(self._lib.pcfd_stage_brick_structured(self.handle, C.byref(flag)))
        return bool(flag.value)

    def launch_count(self) -> int:
        """Kernels this system has launched on its stream so far."""
        n = C.c_int64()
        check(self._lib.pcfd_launch_count(self.handle, C.byref(n)))
        return n.value

    def profile_begin(self, region: int, capacity: int) -> None:
        check(self._lib.pcfd_profile_begin(self.handle, region, capacity))

    def profile_end(self, capacity: int) -> np.ndarray:
        """Per-launch device milliseconds of the armed region since profile_begin."""
        out = np.zeros(capacity, np.float64)
        used = C.c_int32()
        check(self._lib.pcfd_profile_end(self.handle, ptr(out, C.c_double), capacity, C.byref(used)))
        return out[: min(used.value, capacity)]
