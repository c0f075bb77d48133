"""ctypes bridge to ``oracle/_ref/libpcfd_oracle.so`` -- this repository's FP64 OpenMP CPU
restatement of the pressure operator, preconditioner, solvers and projection operators
(oracle/pcfd_oracle.cpp).  TEST INFRASTRUCTURE ONLY: tests and the CPU-baseline leg."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from paracfd_b200.capi import Topology, ptr

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIBRARY = os.path.join(HERE, "_ref", "libpcfd_oracle.so")
_lib = None


def available() -> bool:
    return os.path.exists(PORT_LIBRARY)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"oracle port library missing: {PORT_LIBRARY}")
        L = C.CDLL(PORT_LIBRARY)
        vp, f64p, f32p = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_float)
        L.po_create.restype = vp
        L.po_create.argtypes = [C.POINTER(Topology)]
        L.po_destroy.argtypes = [vp]
        L.po_threads.restype = C.c_int
        L.po_apply.argtypes = [vp, f64p, f64p, C.c_int]
        L.po_diagonal.argtypes = [vp, f64p]
        L.po_precondition.argtypes = [vp, f64p, f64p]
        L.po_set_composite.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.po_solve.restype = C.c_int
        L.po_solve.argtypes = [vp, f64p, f64p, C.c_double, C.c_int, C.c_int, f64p]
        L.po_divergence.argtypes = [vp, f32p, f32p, f32p, f32p, f64p, f64p]
        L.po_correct.argtypes = [vp, f64p, C.c_double, C.c_double, f32p, f32p, f32p, f32p]
        _lib = L
    return _lib


def threads() -> int:
    return lib().po_threads()


class PortSystem:
    def __init__(self, topology: Topology):
        self.topology = topology
        self.n = topology.storage_size
        self.handle = lib().po_create(C.byref(topology))

    def close(self):
        if self.handle:
            lib().po_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def apply(self, p, orthogonal=False):
        out = np.zeros(self.n)
        lib().po_apply(self.handle, ptr(np.ascontiguousarray(p, np.float64), C.c_double), ptr(out, C.c_double), int(orthogonal))
        return out

    def diagonal(self):
        out = np.zeros(self.n)
        lib().po_diagonal(self.handle, ptr(out, C.c_double))
        return out

    def set_composite(self, steps: int = 6, stage_ratio: int = 30, fine_ratio: int = 10):
        """Switch to the composite cycle (FP64 restatement of paracfd_b200's)."""
        lib().po_set_composite(self.handle, steps, stage_ratio, fine_ratio)

    def precondition(self, r):
        out = np.zeros(self.n)
        lib().po_precondition(self.handle, ptr(np.ascontiguousarray(r, np.float64), C.c_double), ptr(out, C.c_double))
        return out

    def solve(self, b, tolerance, max_iterations, x0=None):
        x = np.zeros(self.n) if x0 is None else np.array(x0, np.float64)
        out = np.zeros(3)
        ok = lib().po_solve(self.handle, ptr(x, C.c_double), ptr(np.ascontiguousarray(b, np.float64), C.c_double), tolerance,
                            max_iterations, int(x0 is not None), ptr(out, C.c_double))
        return x, {"converged": bool(ok), "relative_residual": out[0], "iterations": int(out[1]),
                   "preconditioner_applications": int(out[2])}

    def divergence(self, u, v, w, special):
        integrated, div = np.zeros(self.n), np.zeros(self.n)
        lib().po_divergence(self.handle, ptr(np.ascontiguousarray(u, np.float32), C.c_float),
                            ptr(np.ascontiguousarray(v, np.float32), C.c_float), ptr(np.ascontiguousarray(w, np.float32), C.c_float),
                            ptr(np.ascontiguousarray(special, np.float32), C.c_float), ptr(integrated, C.c_double), ptr(div, C.c_double))
        return integrated, div

    def correct(self, pressure, rho, dt, u, v, w, special):
        u, v, w, special = (np.array(a, np.float32) for a in (u, v, w, special))
        lib().po_correct(self.handle, ptr(np.ascontiguousarray(pressure, np.float64), C.c_double), rho, dt, ptr(u, C.c_float),
                         ptr(v, C.c_float), ptr(w, C.c_float), ptr(special, C.c_float))
        return u, v, w, special
