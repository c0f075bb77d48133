"""Surface-load integration (pcfd_core_loads) against the reference's compute_pressure_loads and
accumulate_viscous_loads (aero_loads.cpp:183-204), on reference-built cut-cell topologies: the
2-level box, the 1-level NACA slab and a 3-level NACA 4412 wing, with the same pressure and the
same smooth-wall step."""
import dataclasses

import numpy as np
import pytest

from oracle import ref
from paracfd_b200 import CompositeSystem
from paracfd_b200.workloads import WORKLOADS

pytestmark = pytest.mark.gpu

# 3 levels of 8^3 bricks around the NACA 4412 wing (288,700 DOFs, 8,363 EB edges)
WING3 = dataclasses.replace(WORKLOADS["naca4412_wing"], name="wing3", base_cell_size=0.2, surface_refinement_distance=0.2,
                            wing_refinement_distance=0.4, wake_length=1.0, wake_radius=0.4)

CASES = {
    "box2": lambda: (ref.box_case(), 0.0),
    "naca16": lambda: (ref.naca_slab_case(base_cell_size=1 / 16), 0.0),
    "wing3": lambda: (ref.workload_case(WING3), WING3.min_volume_fraction),
}


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request, gpu):
    rc, mvf = CASES[request.param]()
    s = CompositeSystem(rc.topology, momentum_min_volume_fraction=mvf)
    s.configure(speed=10.0, rho=1.225, nu=1.5e-5)
    yield rc, s
    s.close()
    rc.close()


def smooth_state(rc, seed):
    rng = np.random.default_rng(seed)
    c = np.ctypeslib.as_array(rc.topology.centroid, shape=(rc.n, 3))
    k = rng.uniform(0.5, 2.0, size=(3, 3))
    return tuple(((np.sin(c @ k[a]) + (10.0 if a == 0 else 0.0)) * rc.active).astype(np.float32) for a in range(3))


def test_pressure_and_viscous_loads_match_reference(case):
    rc, s = case
    c = np.ctypeslib.as_array(rc.topology.centroid, shape=(rc.n, 3))
    # a smooth pressure with a linear part (closed surfaces integrate it to -V grad p) and a
    # curved part; the device integrates the FP32 shadow, as the reference's pressure_loads
    # integrates its downloaded FP32 pressure widened to double
    p = (40.0 + 25.0 * c[:, 0] - 12.0 * c[:, 2] + 6.0 * np.sin(2.0 * c[:, 1]) * c[:, 0]) * rc.active
    p32 = p.astype(np.float32).astype(np.float64)
    state = smooth_state(rc, 3)
    nu, dt, rho, pref, origin = 1.5e-5, 1e-3, 1.225, 0.3, (0.25, 0.1, -0.05)
    s.set_state(*state)
    s.set_pressure(p32)
    s.smooth_wall(dt, nu)
    got = s.loads(pressure_reference=pref, moment_origin=origin, include_viscous=True)
    fp, mp, fv, mv = rc.wall_loads(state, nu, dt, rho, p32, pref, origin)
    # pressure loads: the same FP64 terms summed in another order
    assert np.abs(np.array(got["pressure_force"]) - fp).max() <= 1e-10 * np.abs(fp).max()
    assert np.abs(np.array(got["pressure_moment"]) - mp).max() <= 1e-10 * np.abs(mp).max()
    # viscous loads: sums of the FP32 smooth-wall patch forces (the wall model's own tolerance)
    assert np.abs(np.array(got["viscous_force"]) - fv).max() <= 1e-4 * max(np.abs(fv).max(), 1e-30)
    assert np.abs(np.array(got["viscous_moment"]) - mv).max() <= 1e-4 * max(np.abs(mv).max(), 1e-30)
    assert np.allclose(got["total_force"], np.array(got["pressure_force"]) + np.array(got["viscous_force"]), rtol=1e-12)


def _reference_conservation(divergence, volume, active):
    """ExternalAeroCore::conservation_stats (external_aero_core.cpp:347-356), restated in numpy."""
    ok = active.astype(bool) & (volume > 0)
    d = np.asarray(divergence, np.float64)[ok]
    v = volume[ok]
    a = np.abs(d)
    first = int(np.argmax(a))            # first DOF on ties, as the reference's strict '>' scan
    integrated = d * v
    return {"max_abs_divergence": a[first], "worst_control_volume": v[first],
            "max_integrated_flux_error": np.abs(integrated).max(), "absolute_integrated_flux_error": np.abs(integrated).sum(),
            "net_integrated_flux_error": integrated.sum(),
            "volume_weighted_rms_divergence": np.sqrt((d * d * v).sum() / v.sum())}


def test_conservation_stats_match_reference(case):
    rc, s = case
    state = smooth_state(rc, 9)
    s.set_state(*state)
    s.reconstruct_fluxes()
    u, v, w = s.get_faces()
    cf, eb = s.get_special()
    ours_div = s.divergence()
    got = s.conservation_stats()
    volume = np.ctypeslib.as_array(rc.topology.volume, shape=(rc.n,))
    # the device reductions restate the reference's loop on the same FP32 divergence
    want = _reference_conservation(ours_div, volume, rc.active)
    for key, value in want.items():
        # sums in another order: 1e-12 of the value, or for the signed net flux (a sum that
        # cancels) 1e-12 of the sum of magnitudes
        scale = want["absolute_integrated_flux_error"] if key == "net_integrated_flux_error" else abs(value)
        assert abs(got[key] - value) <= 1e-12 * max(scale, 1e-300) + 1e-300, (key, got[key], value)
    # and on the reference twin's divergence (composite_amr_divergence_cpu, rounded to FP32 like the
    # reference's device field) the statistics agree to FP32 rounding
    twin = _reference_conservation(rc.divergence(u, v, w, cf.astype(np.float64), eb.astype(np.float64)).astype(np.float32),
                                   volume, rc.active)
    for key in ("max_abs_divergence", "volume_weighted_rms_divergence", "absolute_integrated_flux_error"):
        assert abs(got[key] - twin[key]) <= 1e-5 * max(abs(twin[key]), 1e-30), (key, got[key], twin[key])
