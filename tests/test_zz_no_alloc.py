"""The allocation-free operator entry point (static device scratch) against the system-scratch
entry point, through the C ABI on device buffers, on two calls in a row.  Collected last."""
import ctypes as C

import numpy as np
import pytest

from oracle import ref
from paracfd_b200 import CompositeSystem, capi

pytestmark = pytest.mark.gpu


def test_noalloc_apply_matches_device_apply_twice(gpu):
    import torch

    rc = ref.box_case()            # 2 levels, compact edges, gauges and WLS gradient nodes
    assert rc.summary["gradient_nodes"] > 0
    lib = capi.load()
    with CompositeSystem(rc.topology) as s:
        rng = np.random.default_rng(23)
        for orthogonal in (0, 1):
            for call in range(2):
                p = torch.from_numpy(rng.standard_normal(rc.n) * rc.active).to("cuda:0")
                ref_out = torch.zeros(rc.n, dtype=torch.float64, device="cuda:0")
                out = torch.full((rc.n,), np.nan, dtype=torch.float64, device="cuda:0")
                torch.cuda.synchronize()
                capi.check(lib.pcfd_pressure_apply_device(s.handle, C.c_void_p(p.data_ptr()),
                                                          C.c_void_p(ref_out.data_ptr()), orthogonal))
                capi.check(lib.pcfd_pressure_apply_device_noalloc(s.handle, C.c_void_p(p.data_ptr()),
                                                                  C.c_void_p(out.data_ptr()), orthogonal))
                s.synchronize()
                # both entry points write every entry of the active DOFs (covered-brick slots
                # are outside the operator and left untouched by either)
                act = rc.active.astype(bool)
                a, b = out.cpu().numpy()[act], ref_out.cpu().numpy()[act]
                assert np.all(np.isfinite(a)), (orthogonal, call)
                # same kernels, same order: agreement to FP64 rounding (the operator tolerance)
                assert np.abs(a - b).max() <= 1e-12 * max(np.abs(b).max(), 1e-300), (orthogonal, call)
    rc.close()
