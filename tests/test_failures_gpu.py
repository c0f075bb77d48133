"""Failure detection on the GPU without a GPU fault: non-finite host inputs are refused before
they reach the device, a projection that does not converge leaves the physical time where it was
(the reference's rule, external_aero_core.cpp:327), a first projection that does not converge
refuses stepping (:306), and the system stays usable after each."""
import ctypes as C

import numpy as np
import pytest

from oracle import ref
from paracfd_b200 import CompositeSystem, capi

pytestmark = pytest.mark.gpu

CASE = dict(speed=10.0, rho=1.225, nu=1.5e-5, cfl=0.5, smagorinsky_cs=0.10)


@pytest.fixture(scope="module")
def slab(gpu):
    rc = ref.naca_slab_case(base_cell_size=1 / 16)
    s = CompositeSystem(rc.topology, momentum_min_volume_fraction=rc.params.min_volume_fraction)
    yield rc, s
    s.close()
    rc.close()


def _step(s):
    stats = capi.StepStats()
    status = capi.load().pcfd_core_step(s.handle, C.byref(stats))
    return status, stats.as_dict()


def test_non_finite_host_inputs_are_refused(slab):
    rc, s = slab
    n = rc.n
    good = tuple(np.zeros(n, np.float32) for _ in range(3))
    bad = np.zeros(n, np.float32)
    bad[n // 3] = np.nan
    for call in (lambda: s.set_state(bad, good[1], good[2]),
                 lambda: s.set_faces(np.full(s.faces, np.inf, np.float32), np.zeros(s.faces, np.float32),
                                     np.zeros(s.faces, np.float32)),
                 lambda: s.set_pressure(np.where(np.arange(n) == 5, np.nan, 0.0)),
                 lambda: s.solve(np.full(n, np.nan), 1e-8, 10)):
        with pytest.raises(capi.PcfdError) as err:
            call()
        assert err.value.status == capi.PCFD_INVALID_ARG and "non-finite" in str(err.value)
    s.set_state(*good)                              # finite input still accepted afterwards
    assert np.array_equal(s.get_state()[0], good[0])


def test_unconverged_projection_leaves_time_unadvanced(slab):
    rc, s = slab
    s.configure(**CASE, projection_tolerance=1e-8, projection_max_iterations=600)
    assert s.initialize()["pressure"]["converged"]
    status, first = _step(s)
    assert status == capi.PCFD_OK and first["physical_time"] > 0
    # same flow case, a projection budget of one iteration at an unreachable tolerance
    s.configure(**CASE, projection_tolerance=1e-14, projection_max_iterations=1)
    status, failed = _step(s)
    assert status == capi.PCFD_NOT_CONVERGED
    assert not failed["pressure"]["converged"] and failed["physical_time"] == first["physical_time"]
    assert b"time not advanced" in capi.load().pcfd_last_error_message()
    # the budget restored, stepping continues from there
    s.configure(**CASE, projection_tolerance=1e-8, projection_max_iterations=600)
    status, again = _step(s)
    assert status == capi.PCFD_OK and again["physical_time"] > first["physical_time"]


def test_unconverged_initialization_refuses_stepping(slab):
    rc, s = slab
    s.configure(**dict(CASE, speed=9.0), projection_tolerance=1e-14, projection_max_iterations=1)
    stats = capi.StepStats()
    assert capi.load().pcfd_core_initialize(s.handle, C.byref(stats)) == capi.PCFD_NOT_CONVERGED
    status, _ = _step(s)
    assert status != capi.PCFD_OK and b"converged initialization" in capi.load().pcfd_last_error_message()
