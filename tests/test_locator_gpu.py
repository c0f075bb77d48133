"""Device point location against the reference's own DeviceAmrLocator (its GPU code, oracle/_ref):
the same (level, brick, i, j, k) for every point, inside, outside and on brick and cell edges; and
the headless slice sampler against a numpy gather through those locations."""
import ctypes as C

import numpy as np
import pytest

from oracle import ref
from paracfd_b200 import CompositeSystem, capi

pytestmark = pytest.mark.gpu


def _points(rc, seed, n=20000):
    t = rc.topology
    lo, hi = np.array(t.domain_lo[:]), np.array(t.domain_hi[:])
    rng = np.random.default_rng(seed)
    inside = lo + rng.random((n, 3)) * (hi - lo)
    # points on the finest lattice lines (brick and cell edges) and a margin outside the box
    h = t.levels[t.level_count - 1].h
    lattice = lo + np.round((inside - lo) / h) * h
    outside = lo - 0.1 * (hi - lo) + rng.random((n // 10, 3)) * 1.2 * (hi - lo)
    return np.concatenate([inside, lattice, outside, [lo, hi, (lo + hi) / 2]]).astype(np.float32)


@pytest.mark.parametrize("make", [lambda: ref.box_case(), lambda: ref.naca_slab_case(base_cell_size=1 / 16)])
def test_locations_match_reference_locator(gpu, make):
    import torch
    rc = make()
    pts = _points(rc, 5)
    want = rc.locate_points(pts)
    with CompositeSystem(rc.topology) as s:
        d_pts = torch.from_numpy(pts).to("cuda:0")
        d_out = torch.full((len(pts), 5), -7, dtype=torch.int32, device="cuda:0")
        torch.cuda.synchronize()
        capi.check(capi.load().pcfd_locate_points_device(s.handle, C.c_void_p(d_pts.data_ptr()), len(pts),
                                                         C.c_void_p(d_out.data_ptr())))
        s.synchronize()
        got = d_out.cpu().numpy()
    rc.close()
    assert (want[:, 0] >= 0).sum() > len(pts) // 2         # most points land in a brick
    np.testing.assert_array_equal(got, want)


def test_slice_samples_the_finest_active_cell(gpu):
    rc = ref.box_case()
    t = rc.topology
    lo, hi = np.array(t.domain_lo[:]), np.array(t.domain_hi[:])
    rng = np.random.default_rng(3)
    state = tuple((rng.standard_normal(rc.n) * rc.active).astype(np.float32) for _ in range(3))
    origin = np.array([lo[0], lo[1], 0.5 * (lo[2] + hi[2]) + 0.013])
    eu, ev = np.array([hi[0] - lo[0], 0.0, 0.0]), np.array([0.0, hi[1] - lo[1], 0.0])
    nu, nv = 97, 61
    with CompositeSystem(rc.topology) as s:
        s.set_state(*state)
        speed = s.sample_slice(origin, eu, ev, nu, nv, 0)
        vy = s.sample_slice(origin, eu, ev, nu, nv, 2)
    a, b = np.meshgrid((np.arange(nu) + 0.5) / nu, (np.arange(nv) + 0.5) / nv)
    pts = (origin[None, None, :] + a[..., None] * eu + b[..., None] * ev).reshape(-1, 3).astype(np.float32)
    where = rc.locate_points(pts)
    starts = np.cumsum([0] + [t.levels[l].brick_count for l in range(t.level_count)])
    want_speed = np.full(len(pts), np.nan, np.float32)
    want_vy = np.full(len(pts), np.nan, np.float32)
    for q, (level, brick, i, j, k) in enumerate(where):
        if level < 0:
            continue
        dof = (starts[level] + brick) * 512 + (k * 8 + j) * 8 + i
        if rc.active[dof]:
            x, y, z = (st[dof] for st in state)
            want_speed[q] = np.sqrt(np.float32(x * x + y * y + z * z))
            want_vy[q] = y
    rc.close()
    np.testing.assert_allclose(speed.ravel(), want_speed, rtol=1e-6, equal_nan=True)
    np.testing.assert_array_equal(vy.ravel(), want_vy)
    assert np.isfinite(speed).sum() > 0.8 * speed.size
