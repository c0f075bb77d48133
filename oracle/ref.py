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

    def __init__(self, params: CaseParams):
        self.params = params
        self.handle = lib().ref_case_create(C.byref(params))
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


def box_case(**kw) -> RefCase:
    return RefCase(default_params(CASE_BOX, **kw))


def naca_slab_case(**kw) -> RefCase:
    return RefCase(default_params(CASE_NACA_SLAB, **kw))
