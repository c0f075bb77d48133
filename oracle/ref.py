"""ctypes bridge to ``oracle/_ref/libparacfd_ref.so`` -- the reference ParaCFD host code
compiled from its own sources, plus the fixture shim in ``oracle/ref_shim.cpp``.

TEST INFRASTRUCTURE ONLY.  Tests and the CPU-baseline arm use it as the checker; the product
(``paracfd_b200``) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from paracfd_b200.capi import Topology, ptr

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIBRARY = os.path.join(HERE, "_ref", "libparacfd_ref.so")

CASE_BOX, CASE_NACA_SLAB, CASE_NACA_WING, CASE_BOX_CROPPED = 0, 1, 2, 3


class CaseParams(C.Structure):
    _fields_ = [("kind", C.c_int32), ("naca_digits", C.c_int32), ("section_points", C.c_int32),
                ("max_levels", C.c_int32), ("brick_size", C.c_int32),
                ("base_cell_size", C.c_double), ("chord", C.c_double), ("span", C.c_double),
                ("aoa_deg", C.c_double), ("domain_lo", C.c_double * 3),
                ("domain_hi", C.c_double * 3), ("surface_refinement_distance", C.c_double),
                ("wing_refinement_distance", C.c_double), ("wake_length", C.c_double),
                ("wake_radius", C.c_double), ("min_volume_fraction", C.c_double)]


class CoreCase(C.Structure):
    _fields_ = [("speed", C.c_double), ("rho", C.c_double), ("nu", C.c_double), ("cfl", C.c_double),
                ("smagorinsky_cs", C.c_double), ("projection_tolerance", C.c_double),
                ("projection_max_iterations", C.c_int32)]


_lib = None


def available() -> bool:
    return os.path.exists(REF_LIBRARY)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"reference oracle library missing: {REF_LIBRARY}")
        L = C.CDLL(REF_LIBRARY)
        vp, f64p, f32p = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_float)
        L.ref_default_params.argtypes = [C.c_int32, C.POINTER(CaseParams)]
        L.ref_case_create.restype = vp
        L.ref_case_create.argtypes = [C.POINTER(CaseParams)]
        L.ref_case_destroy.argtypes = [vp]
        L.ref_last_error.restype = C.c_char_p
        L.ref_case_topology.argtypes = [vp, C.POINTER(Topology)]
        L.ref_case_summary.argtypes = [vp, C.POINTER(C.c_int64)]
        L.ref_case_level_counts.argtypes = [vp, C.POINTER(C.c_int64)]
        L.ref_apply_cpu.argtypes = [vp, f64p, f64p]
        L.ref_diagonal_cpu.argtypes = [vp, f64p]
        L.ref_divergence_cpu.argtypes = [vp, f32p, f32p, f32p, f64p, f64p, f64p]
        L.ref_rhs_cpu.argtypes = [vp, f32p, f32p, f32p, f64p, f64p, C.c_double, C.c_double, f64p]
        L.ref_correct_fluxes_cpu.argtypes = [vp, f64p, C.c_double, C.c_double, f32p, f32p, f32p, f64p, f64p]
        L.ref_pressure_gradients_cpu.argtypes = [vp, f64p, f64p]
        L.ref_transport_cpu.argtypes = [vp, f32p, f32p, f32p, f64p, f64p, C.c_double, C.c_int, C.c_double, f32p, f32p, f32p]
        L.ref_smagorinsky_viscosity_cpu.argtypes = [vp, f32p, f32p, f32p, C.c_double, C.c_double, f64p]
        L.ref_diffuse_smagorinsky_cpu.argtypes = [vp, C.c_double, C.c_double, C.c_double, f32p, f32p, f32p]
        L.ref_diffuse_cpu.argtypes = [vp, C.c_double, C.c_double, f32p, f32p, f32p]
        L.ref_wall_cpu.argtypes = [vp, C.c_double, C.c_double, C.c_double, f32p, f32p, f32p, f64p, C.POINTER(C.c_int64)]
        L.ref_impulse_cpu.argtypes = [vp, f64p, C.c_double, C.c_double, C.c_int, f32p, f32p, f32p]
        L.ref_reconstruct_cpu.argtypes = [vp, f32p, f32p, f32p, f32p, f32p, f32p, f64p, f64p]
        L.ref_outflow_rate_cpu.argtypes = [vp, f32p, f32p, f32p, f64p, f64p, C.c_int, f64p]
        L.ref_core_create.restype = vp
        L.ref_core_create.argtypes = [vp, C.POINTER(CoreCase)]
        L.ref_core_destroy.argtypes = [vp]
        L.ref_core_initialize.argtypes = [vp, f64p]
        L.ref_core_step.argtypes = [vp, f64p]
        L.ref_core_state.argtypes = [vp, f32p, f32p, f32p, f64p]
        L.ref_pressure_loads.argtypes = [vp, f64p, C.c_double, f64p, f64p]
        L.ref_locate_points.argtypes = [vp, f32p, C.c_int64, C.POINTER(C.c_int32)]
        L.ref_wall_loads_cpu.argtypes = [vp, C.c_double, C.c_double, C.c_double, f32p, f32p, f32p, f64p, C.c_double,
                                         f64p, f64p]
        L.ref_import_topology.restype = vp
        L.ref_import_topology.argtypes = [C.POINTER(Topology)]
        L.ref_device_core_create.restype = vp
        L.ref_device_core_create.argtypes = [vp, C.POINTER(CoreCase), C.c_double]
        L.ref_device_core_destroy.argtypes = [vp]
        L.ref_device_core_initialize.argtypes = [vp, f64p]
        L.ref_device_core_step.argtypes = [vp, f64p]
        L.ref_device_core_state.argtypes = [vp, f32p, f32p, f32p, f64p]
        L.ref_device_core_create_mac.restype = vp
        L.ref_device_core_create_mac.argtypes = [vp, C.POINTER(CoreCase), C.c_int32]
        L.ref_device_core_faces.argtypes = [vp, f32p, f32p, f32p]
        L.ref_case_from_mesh.restype = vp
        L.ref_case_from_mesh.argtypes = [f64p, C.c_int64, C.POINTER(C.c_uint32), C.c_int64, f64p, f64p, C.c_double,
                                         C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double]
        L.ref_case_from_mesh_eb.restype = vp
        L.ref_case_from_mesh_eb.argtypes = [f64p, C.c_int64, C.POINTER(C.c_uint32), C.c_int64, f64p, f64p, C.c_double,
                                            C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double,
                                            C.c_double]
        u8p = C.POINTER(C.c_uint8)
        L.ref_mac_links.argtypes = [vp, C.c_double, u8p, u8p, u8p]
        L.ref_mac_create.restype = vp
        L.ref_mac_create.argtypes = [vp, C.c_double]
        L.ref_mac_destroy.argtypes = [vp]
        L.ref_mac_set_faces.argtypes = [vp, f32p, f32p, f32p]
        L.ref_mac_advect.argtypes = [vp, C.c_double]
        L.ref_mac_diffuse_smagorinsky.argtypes = [vp, C.c_double, C.c_double, C.c_double]
        L.ref_mac_state.argtypes = [vp, f32p, f32p, f32p, f32p]
        L.ref_mac_set_special.argtypes = [vp, f64p, f64p]
        L.ref_mac_transport_apertures.argtypes = [vp, C.c_double, C.c_double, C.c_double]
        L.ref_mac_special.argtypes = [vp, f64p, f64p]
        _lib = L
    return _lib


def _check(status):
    if status != 0:
        raise RuntimeError("reference oracle: " + lib().ref_last_error().decode(errors="replace"))


def default_params(kind: int, **overrides) -> CaseParams:
    p = CaseParams()
    lib().ref_default_params(kind, C.byref(p))
    for key, value in overrides.items():
        if key in ("domain_lo", "domain_hi"):
            getattr(p, key)[:] = value
        else:
            setattr(p, key, value)
    return p


class RefCase:
    """Reference preprocessing result (hierarchy + EB atlas + composite pressure system)."""

    def __init__(self, params: CaseParams | None, handle=None):
        self.params = params
        self.handle = handle if handle is not None else lib().ref_case_create(C.byref(params))
        if not self.handle:
            raise RuntimeError("reference case build failed: " + lib().ref_last_error().decode(errors="replace"))
        self.topology = Topology()
        _check(lib().ref_case_topology(self.handle, C.byref(self.topology)))
        s = (C.c_int64 * 12)()
        _check(lib().ref_case_summary(self.handle, s))
        keys = ("levels", "storage", "active", "coarse_fine", "embedded", "regular_corrections",
                "gradient_nodes", "gauges", "patches", "boundary_faces", "unresolved", "retained")
        self.summary = dict(zip(keys, list(s)))
        self.n = self.summary["storage"]
        self.bs = self.topology.brick_size
        self.bricks = sum(self.topology.levels[l].brick_count for l in range(self.topology.level_count))
        self.structured = self.bricks * self.bs ** 3
        self.faces = self.bricks * (self.bs + 1) * self.bs * self.bs
        self.active = np.ctypeslib.as_array(self.topology.active, shape=(self.n,)).copy()

    def close(self):
        if self.handle:
            lib().ref_case_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- reference host operators ------------------------------------------------------
    def apply(self, p: np.ndarray) -> np.ndarray:
        out = np.zeros(self.n)
        _check(lib().ref_apply_cpu(self.handle, ptr(np.ascontiguousarray(p, np.float64), C.c_double), ptr(out, C.c_double)))
        return out

    def diagonal(self) -> np.ndarray:
        out = np.zeros(self.n)
        _check(lib().ref_diagonal_cpu(self.handle, ptr(out, C.c_double)))
        return out

    def divergence(self, u, v, w, cf, eb) -> np.ndarray:
        out = np.zeros(self.n)
        _check(lib().ref_divergence_cpu(self.handle, ptr(u, C.c_float), ptr(v, C.c_float), ptr(w, C.c_float),
                                        ptr(cf, C.c_double), ptr(eb, C.c_double), ptr(out, C.c_double)))
        return out

    def rhs(self, u, v, w, cf, eb, rho, dt) -> np.ndarray:
        out = np.zeros(self.n)
        _check(lib().ref_rhs_cpu(self.handle, ptr(u, C.c_float), ptr(v, C.c_float), ptr(w, C.c_float),
                                 ptr(cf, C.c_double), ptr(eb, C.c_double), rho, dt, ptr(out, C.c_double)))
        return out

    def correct_fluxes(self, pressure, rho, dt, u, v, w, cf, eb):
        u, v, w = (np.array(x, np.float32) for x in (u, v, w))
        cf, eb = np.array(cf, np.float64), np.array(eb, np.float64)
        _check(lib().ref_correct_fluxes_cpu(self.handle, ptr(np.ascontiguousarray(pressure, np.float64), C.c_double),
                                            rho, dt, ptr(u, C.c_float), ptr(v, C.c_float), ptr(w, C.c_float),
                                            ptr(cf, C.c_double), ptr(eb, C.c_double)))
        return u, v, w, cf, eb

    def pressure_gradients(self, pressure) -> np.ndarray:
        out = np.zeros((self.n, 3))
        _check(lib().ref_pressure_gradients_cpu(self.handle, ptr(np.ascontiguousarray(pressure, np.float64), C.c_double),
                                                ptr(out, C.c_double)))
        return out


    # ---- cell-momentum host twins (state arrays are copied; new arrays returned) -------------
    @staticmethod
    def _state(x, y, z):
        return tuple(np.array(a, np.float32) for a in (x, y, z))

    def transport(self, u, v, w, cf, eb, dt, state, external=False, freestream=0.0):
        x, y, z = self._state(*state)
        _check(lib().ref_transport_cpu(self.handle, ptr(u, C.c_float), ptr(v, C.c_float), ptr(w, C.c_float),
                                       ptr(np.asarray(cf, np.float64), C.c_double), ptr(np.asarray(eb, np.float64), C.c_double),
                                       dt, int(external), freestream, ptr(x, C.c_float), ptr(y, C.c_float), ptr(z, C.c_float)))
        return x, y, z

    def smagorinsky_viscosity(self, state, nu, cs):
        x, y, z = self._state(*state)
        out = np.zeros(self.n)
        _check(lib().ref_smagorinsky_viscosity_cpu(self.handle, ptr(x, C.c_float), ptr(y, C.c_float), ptr(z, C.c_float), nu, cs,
                                                   ptr(out, C.c_double)))
        return out

    def diffuse_smagorinsky(self, state, nu, cs, dt):
        x, y, z = self._state(*state)
        _check(lib().ref_diffuse_smagorinsky_cpu(self.handle, nu, cs, dt, ptr(x, C.c_float), ptr(y, C.c_float), ptr(z, C.c_float)))
        return x, y, z

    def wall(self, state, nu, dt, rho):
        x, y, z = self._state(*state)
        sides = C.c_int64()
        forces = np.zeros(6 * max(1, self.summary["patches"]))
        _check(lib().ref_wall_cpu(self.handle, nu, dt, rho, ptr(x, C.c_float), ptr(y, C.c_float), ptr(z, C.c_float),
                                  ptr(forces, C.c_double), C.byref(sides)))
        return (x, y, z), forces[: 3 * sides.value].reshape(-1, 3)

    def impulse(self, pressure, dt, rho, state, physical=True):
        x, y, z = self._state(*state)
        _check(lib().ref_impulse_cpu(self.handle, ptr(np.ascontiguousarray(pressure, np.float64), C.c_double), dt, rho, int(physical),
                                     ptr(x, C.c_float), ptr(y, C.c_float), ptr(z, C.c_float)))
        return x, y, z

    def reconstruct(self, state, u, v, w):
        x, y, z = self._state(*state)
        u, v, w = (np.array(a, np.float32) for a in (u, v, w))
        cf = np.zeros(self.summary["coarse_fine"])
        eb = np.zeros(self.summary["embedded"])
        _check(lib().ref_reconstruct_cpu(self.handle, ptr(x, C.c_float), ptr(y, C.c_float), ptr(z, C.c_float), ptr(u, C.c_float),
                                         ptr(v, C.c_float), ptr(w, C.c_float), ptr(cf, C.c_double), ptr(eb, C.c_double)))
        return u, v, w, cf, eb

    def pressure_loads(self, pressure, pressure_reference=0.0, origin=(0.0, 0.0, 0.0)):
        out = np.zeros(6)
        o = np.ascontiguousarray(origin, np.float64)
        _check(lib().ref_pressure_loads(self.handle, ptr(np.ascontiguousarray(pressure, np.float64), C.c_double),
                                        pressure_reference, ptr(o, C.c_double), ptr(out, C.c_double)))
        return out[:3], out[3:]

    def wall_loads(self, state, nu, dt, rho, pressure, pressure_reference=0.0, origin=(0.0, 0.0, 0.0)):
        """Pressure and viscous (smooth-wall) loads: (Fp, Mp, Fv, Mv)."""
        x, y, z = self._state(*state)
        out = np.zeros(12)
        o = np.ascontiguousarray(origin, np.float64)
        _check(lib().ref_wall_loads_cpu(self.handle, nu, dt, rho, ptr(x, C.c_float), ptr(y, C.c_float), ptr(z, C.c_float),
                                        ptr(np.ascontiguousarray(pressure, np.float64), C.c_double), pressure_reference,
                                        ptr(o, C.c_double), ptr(out, C.c_double)))
        return out[0:3], out[3:6], out[6:9], out[9:12]

    def locate_points(self, points) -> np.ndarray:
        """The reference's DeviceAmrLocator (GPU): [n, 5] level, brick, i, j, k."""
        pts = np.ascontiguousarray(points, np.float32)
        out = np.zeros((len(pts), 5), np.int32)
        _check(lib().ref_locate_points(self.handle, ptr(pts, C.c_float), len(pts), ptr(out, C.c_int32)))
        return out

    def outflow_rate(self, u, v, w, cf, eb, external=True):
        out = C.c_double()
        _check(lib().ref_outflow_rate_cpu(self.handle, ptr(u, C.c_float), ptr(v, C.c_float), ptr(w, C.c_float),
                                          ptr(np.asarray(cf, np.float64), C.c_double), ptr(np.asarray(eb, np.float64), C.c_double),
                                          int(external), C.byref(out)))
        return out.value


    def mac_links(self, protection_cells=2.5):
        """The reference advection's per-face link bytes (compact layout), from the case surface."""
        out = [np.zeros(self.faces, np.uint8) for _ in range(3)]
        _check(lib().ref_mac_links(self.handle, protection_cells, *(ptr(a, C.c_uint8) for a in out)))
        return out


class RefMac:
    """The reference's staggered MAC momentum path (DeviceAmrAdvection on DeviceAmrFields); needs a GPU."""

    def __init__(self, case: RefCase, protection_cells=2.5):
        self.case = case
        self.handle = lib().ref_mac_create(case.handle, protection_cells)
        if not self.handle:
            raise RuntimeError("reference MAC: " + lib().ref_last_error().decode(errors="replace"))

    def set_faces(self, u, v, w):
        a = [np.ascontiguousarray(x, np.float32) for x in (u, v, w)]
        _check(lib().ref_mac_set_faces(self.handle, *(ptr(x, C.c_float) for x in a)))

    def advect(self, dt):
        _check(lib().ref_mac_advect(self.handle, dt))

    def diffuse_smagorinsky(self, nu, cs, dt):
        _check(lib().ref_mac_diffuse_smagorinsky(self.handle, nu, cs, dt))

    def set_special(self, coarse_fine, embedded):
        cf = np.ascontiguousarray(coarse_fine, np.float64)
        eb = np.ascontiguousarray(embedded, np.float64)
        _check(lib().ref_mac_set_special(self.handle, ptr(cf, C.c_double), ptr(eb, C.c_double)))

    def transport_apertures(self, dt, nu, cs):
        _check(lib().ref_mac_transport_apertures(self.handle, dt, nu, cs))

    def special(self):
        cf = np.zeros(self.case.summary["coarse_fine"])
        eb = np.zeros(self.case.summary["embedded"])
        _check(lib().ref_mac_special(self.handle, ptr(cf, C.c_double), ptr(eb, C.c_double)))
        return cf, eb

    def state(self):
        u, v, w = (np.zeros(self.case.faces, np.float32) for _ in range(3))
        nut = np.zeros(self.case.n, np.float32)
        _check(lib().ref_mac_state(self.handle, *(ptr(x, C.c_float) for x in (u, v, w, nut))))
        return (u, v, w), nut

    def close(self):
        if self.handle:
            lib().ref_mac_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefCore:
    """The reference's own ExternalAeroCore (its CUDA path) on a fixture; needs a GPU."""

    def __init__(self, case: RefCase, speed=10.0, rho=1.225, nu=1.5e-5, cfl=0.5, cs=0.10, tolerance=1e-8, max_iterations=600):
        self.case = case
        cfg = CoreCase(speed, rho, nu, cfl, cs, tolerance, max_iterations)
        self.handle = lib().ref_core_create(case.handle, C.byref(cfg))
        if not self.handle:
            raise RuntimeError("reference core: " + lib().ref_last_error().decode(errors="replace"))

    @staticmethod
    def _stats(a):
        return {"dt": a[0], "gpu_step_ms": a[1], "projection_ms": a[2], "iterations": int(a[3]), "converged": bool(a[4]),
                "relative_residual": a[5]}

    def initialize(self):
        a = np.zeros(6)
        _check(lib().ref_core_initialize(self.handle, ptr(a, C.c_double)))
        return self._stats(a)

    def step(self):
        a = np.zeros(6)
        _check(lib().ref_core_step(self.handle, ptr(a, C.c_double)))
        return self._stats(a)

    def state(self):
        n = self.case.n
        x, y, z = (np.zeros(n, np.float32) for _ in range(3))
        p = np.zeros(n)
        _check(lib().ref_core_state(self.handle, ptr(x, C.c_float), ptr(y, C.c_float), ptr(z, C.c_float), ptr(p, C.c_double)))
        return (x, y, z), p

    def close(self):
        if self.handle:
            lib().ref_core_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def import_topology(topology: Topology) -> RefCase:
    """The reference's hierarchy/system objects holding an externally built topology."""
    handle = lib().ref_import_topology(C.byref(topology))
    if not handle:
        raise RuntimeError("reference import failed: " + lib().ref_last_error().decode(errors="replace"))
    return RefCase(None, handle=handle)


class RefDeviceCore(RefCore):
    """The reference's device classes driven with ExternalAeroCore's step sequence on any case
    (mac=True: its staggered MAC momentum path, smooth fabric wall as asked)."""

    def __init__(self, case: RefCase, speed=10.0, rho=1.225, nu=1.5e-5, cfl=0.5, cs=0.10, tolerance=1e-8, max_iterations=600,
                 min_volume_fraction=0.25, mac=False, smooth_wall=True):
        self.case = case
        cfg = CoreCase(speed, rho, nu, cfl, cs, tolerance, max_iterations)
        if mac:
            self.handle = lib().ref_device_core_create_mac(case.handle, C.byref(cfg), int(smooth_wall))
        else:
            self.handle = lib().ref_device_core_create(case.handle, C.byref(cfg), min_volume_fraction)
        if not self.handle:
            raise RuntimeError("reference device core: " + lib().ref_last_error().decode(errors="replace"))

    def initialize(self):
        a = np.zeros(6)
        _check(lib().ref_device_core_initialize(self.handle, ptr(a, C.c_double)))
        return self._stats(a)

    def step(self):
        a = np.zeros(6)
        _check(lib().ref_device_core_step(self.handle, ptr(a, C.c_double)))
        return self._stats(a)

    def state(self):
        n = self.case.n
        x, y, z = (np.zeros(n, np.float32) for _ in range(3))
        p = np.zeros(n)
        _check(lib().ref_device_core_state(self.handle, ptr(x, C.c_float), ptr(y, C.c_float), ptr(z, C.c_float),
                                           ptr(p, C.c_double)))
        return (x, y, z), p

    def faces(self):
        u, v, w = (np.zeros(self.case.faces, np.float32) for _ in range(3))
        _check(lib().ref_device_core_faces(self.handle, ptr(u, C.c_float), ptr(v, C.c_float), ptr(w, C.c_float)))
        return u, v, w

    def close(self):
        if self.handle:
            lib().ref_device_core_destroy(self.handle)
            self.handle = None


def case_from_mesh(vertices, triangles, domain_lo, domain_hi, base_cell_size, max_levels, brick_size=8,
                   wing_refinement_distance=1.0, surface_refinement_distance=0.35, wake_length=8.0,
                   wake_radius=2.0) -> RefCase:
    """Reference hierarchy + embedded-boundary-free composite system for an arbitrary mesh."""
    v = np.ascontiguousarray(vertices, np.float64)
    t = np.ascontiguousarray(triangles, np.uint32)
    lo = np.ascontiguousarray(domain_lo, np.float64)
    hi = np.ascontiguousarray(domain_hi, np.float64)
    handle = lib().ref_case_from_mesh(ptr(v, C.c_double), len(v), ptr(t, C.c_uint32), len(t), ptr(lo, C.c_double),
                                      ptr(hi, C.c_double), base_cell_size, max_levels, brick_size,
                                      wing_refinement_distance, surface_refinement_distance, wake_length, wake_radius)
    if not handle:
        raise RuntimeError("reference mesh case failed: " + lib().ref_last_error().decode(errors="replace"))
    return RefCase(None, handle=handle)


def cut_cell_case_from_mesh(vertices, triangles, domain_lo, domain_hi, base_cell_size, max_levels, brick_size=8,
                            wing_refinement_distance=1.0, surface_refinement_distance=0.35, wake_length=8.0,
                            wake_radius=2.0, min_volume_fraction=0.25) -> RefCase:
    """Reference hierarchy + cut-cell embedded-boundary atlas + composite system for a closed
    triangle shell (the shell's own discrete inside test is the solid)."""
    v = np.ascontiguousarray(vertices, np.float64)
    t = np.ascontiguousarray(triangles, np.uint32)
    lo = np.ascontiguousarray(domain_lo, np.float64)
    hi = np.ascontiguousarray(domain_hi, np.float64)
    handle = lib().ref_case_from_mesh_eb(ptr(v, C.c_double), len(v), ptr(t, C.c_uint32), len(t), ptr(lo, C.c_double),
                                         ptr(hi, C.c_double), base_cell_size, max_levels, brick_size,
                                         wing_refinement_distance, surface_refinement_distance, wake_length,
                                         wake_radius, min_volume_fraction)
    if not handle:
        raise RuntimeError("reference cut-cell case failed: " + lib().ref_last_error().decode(errors="replace"))
    return RefCase(None, handle=handle)


def workload_case(spec) -> RefCase:
    """A named workload's grid built by the reference's own preprocessing: its brick hierarchy
    (AmrHierarchy::build_static over the workload's domain), the cut-cell embedded-boundary atlas
    of the workload's closed surface and the composite pressure system, as ExternalAeroCore's
    constructor builds them (external_aero_core.cpp:77-103, 199-200)."""
    vertices, triangles = spec.surface()
    return cut_cell_case_from_mesh(vertices, triangles, spec.domain_lo, spec.domain_hi, spec.base_cell_size,
                                   spec.max_levels, spec.brick_size, spec.wing_refinement_distance,
                                   spec.surface_refinement_distance, spec.wake_length, spec.wake_radius,
                                   spec.min_volume_fraction)


def box_case(**kw) -> RefCase:
    return RefCase(default_params(CASE_BOX, **kw))


def naca_slab_case(**kw) -> RefCase:
    return RefCase(default_params(CASE_NACA_SLAB, **kw))
