"""The allocation-free operator entry point (static device scratch) against the system-scratch
entry point, through the C ABI on device buffers, on two calls in a row.  Collected last.

Callers that cannot allocate at call time (device memory handed out by another pool, loops that
must never enter the allocator) use pcfd_pressure_apply_device_noalloc; these tests check that
it computes the same operator on every structured path (fused brick kernel, the 8^3 per-brick
kernel when the fused level is off, and when the vectors are not 16-byte aligned) and that it
rejects systems whose WLS gradient does not fit its fixed scratch."""
import ctypes as C

import numpy as np
import pytest

from oracle import ref
from paracfd_b200 import CompositeSystem, capi

pytestmark = pytest.mark.gpu


def _compare(lib, s, rc, rng, offset=0):
    import torch
    act = rc.active.astype(bool)
    for orthogonal in (0, 1):
        for call in range(2):
            # `offset` extra leading doubles shift the device pointers off 16-byte alignment
            p = torch.zeros(rc.n + offset, dtype=torch.float64, device="cuda:0")
            p[offset:] = torch.from_numpy(rng.standard_normal(rc.n) * rc.active)
            ref_out = torch.zeros(rc.n + offset, dtype=torch.float64, device="cuda:0")
            out = torch.full((rc.n + offset,), np.nan, dtype=torch.float64, device="cuda:0")
            torch.cuda.synchronize()
            pp = C.c_void_p(p.data_ptr() + 8 * offset)
            capi.check(lib.pcfd_pressure_apply_device(s.handle, pp, C.c_void_p(ref_out.data_ptr() + 8 * offset), orthogonal))
            capi.check(lib.pcfd_pressure_apply_device_noalloc(s.handle, pp, C.c_void_p(out.data_ptr() + 8 * offset),
                                                              orthogonal))
            s.synchronize()
            # both entry points write every entry of the active DOFs (covered-brick slots are
            # outside the operator and left untouched by either)
            a, b = out.cpu().numpy()[offset:][act], ref_out.cpu().numpy()[offset:][act]
            assert np.all(np.isfinite(a)), (orthogonal, call)
            # same kernels, same order: agreement to FP64 rounding (the operator tolerance)
            assert np.abs(a - b).max() <= 1e-12 * max(np.abs(b).max(), 1e-300), (orthogonal, call, offset)


@pytest.mark.parametrize("fused", [True, False])
def test_noalloc_apply_matches_device_apply_twice(gpu, fused):
    rc = ref.box_case()            # 2 levels, compact edges, gauges and WLS gradient nodes
    assert rc.summary["gradient_nodes"] > 0
    lib = capi.load()
    with CompositeSystem(rc.topology, fused_smoother=fused) as s:
        rng = np.random.default_rng(23)
        _compare(lib, s, rc, rng)
        _compare(lib, s, rc, rng, offset=1)          # unaligned vectors: the per-brick kernel path
    rc.close()


def test_noalloc_rejects_gradients_beyond_its_scratch(gpu):
    """A grid with more WLS gradient nodes than the static scratch holds (262,144) is refused for
    the full operator, before anything is launched; the orthogonal part needs no scratch and runs."""
    import torch
    from paracfd_b200.workloads import WORKLOADS
    rc = ref.workload_case(WORKLOADS["naca4412_wing"])
    assert rc.summary["gradient_nodes"] > 1 << 18
    lib = capi.load()
    with CompositeSystem(rc.topology) as s:
        p = torch.zeros(rc.n, dtype=torch.float64, device="cuda:0")
        out = torch.full((rc.n,), 7.0, dtype=torch.float64, device="cuda:0")
        torch.cuda.synchronize()
        status = lib.pcfd_pressure_apply_device_noalloc(s.handle, C.c_void_p(p.data_ptr()), C.c_void_p(out.data_ptr()), 0)
        assert status == capi.PCFD_INVALID_ARG
        assert b"static scratch" in lib.pcfd_last_error_message()
        s.synchronize()
        assert torch.all(out == 7.0)                 # nothing was launched
        capi.check(lib.pcfd_pressure_apply_device_noalloc(s.handle, C.c_void_p(p.data_ptr()),
                                                          C.c_void_p(out.data_ptr()), 1))
        s.synchronize()
        act = rc.active.astype(bool)
        assert np.abs(out.cpu().numpy()[act]).max() == 0.0   # orthogonal part of A 0
    rc.close()
