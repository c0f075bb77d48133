"""Staggered MAC momentum mode against the reference's own DeviceAmrAdvection on the GPU.

The same face velocities, the same link bytes (the reference constructor's recipe over the case
surface) and the same dt go through the reference's advect / diffuse_smagorinsky
(amr_advection.cu:1663-1690, run through the oracle shim) and through pcfd_mac_advect /
pcfd_mac_diffuse_smagorinsky, on a 3-level cut-cell wing: faces of every non-covered brick, and
the cell eddy viscosity, agree to FP32 rounding (both compute in FP32 with the same operation
order; 1e-6 of the velocity scale is asserted).
"""
import numpy as np
import pytest

from oracle import ref
from paracfd_b200 import CompositeSystem

pytestmark = pytest.mark.gpu


def face_positions(topology):
    """Face-centre coordinates [3][faces] per component in the compact per-brick layout."""
    bs = topology.brick_size
    out = []
    for c in range(3):
        n = [bs + 1 if c == a else bs for a in range(3)]
        k, j, i = np.meshgrid(np.arange(n[2]), np.arange(n[1]), np.arange(n[0]), indexing="ij")
        offs = [(i + (0.0 if c == 0 else 0.5)).ravel(), (j + (0.0 if c == 1 else 0.5)).ravel(), (k + (0.0 if c == 2 else 0.5)).ravel()]
        per_level = []
        for l in range(topology.level_count):
            lev = topology.levels[l]
            origin = np.ctypeslib.as_array(lev.origin, shape=(lev.brick_count * 3,)).reshape(-1, 3)
            per_level.append(np.stack([origin[:, a][:, None] + offs[a][None, :] * lev.h for a in range(3)]).reshape(3, -1))
        out.append(np.concatenate(per_level, axis=1))
    return out


def initial_faces(topology, speed=10.0):
    """A smooth three-component flow with O(1) variation over a chord."""
    pos = face_positions(topology)
    x, y, z = pos[0]
    u = speed * (1.0 + 0.2 * np.sin(1.3 * x + 0.7 * y) * np.cos(0.9 * z))
    x, y, z = pos[1]
    v = speed * 0.15 * np.cos(0.8 * x - 1.1 * z) * np.sin(0.6 * y + 0.3)
    x, y, z = pos[2]
    w = speed * 0.1 * np.sin(0.5 * x + 0.9 * y - 0.4 * z)
    return [a.astype(np.float32) for a in (u, v, w)]


def non_covered_faces(topology):
    bs = topology.brick_size
    keep = []
    for l in range(topology.level_count):
        lev = topology.levels[l]
        flags = np.ctypeslib.as_array(lev.flags, shape=(lev.brick_count,))
        keep.append(np.repeat((flags & 128) == 0, (bs + 1) * bs * bs))   # PCFD_BRICK_COVERED
    return np.concatenate(keep)


@pytest.fixture(scope="module")
def wing(gpu):
    from tests.test_loads_gpu import WING3
    rc = ref.workload_case(WING3)
    yield rc
    rc.close()


def test_links_mark_a_fabric_band(wing):
    links = wing.mac_links(2.5)
    band = sum(int(((a & 0x40) != 0).sum()) for a in links)
    assert band > 1000
    # band faces that are not on the surface have at least one open direction
    assert all(int(((a & 0x40) != 0).sum()) > int((a == 0x40).sum()) for a in links)


def test_mac_advection_and_diffusion_match_reference(wing):
    t = wing.topology
    u, v, w = initial_faces(t)
    links = wing.mac_links(2.5)
    h = min(t.levels[l].h for l in range(t.level_count))
    dt = 0.5 * h / 12.0
    keep = non_covered_faces(t)
    cell_keep = np.repeat(keep[::(t.brick_size + 1) * t.brick_size ** 2], t.brick_size ** 3)
    cell_keep = np.concatenate([cell_keep, np.zeros(wing.n - cell_keep.size, bool)])
    refm = ref.RefMac(wing, 2.5)
    with CompositeSystem(t) as s:
        s.set_mac_links(*links)
        # a viscosity large enough that one explicit step visibly changes the smooth field
        # (dt nu / h^2 = 0.17 on the finest level, inside the explicit limit)
        for name, step in (("advect", lambda m: m.advect(dt)), ("diffuse", lambda m: m.diffuse_smagorinsky(0.2, 0.17, dt))):
            refm.set_faces(u, v, w)
            s.set_faces(u, v, w)
            step(refm)
            if name == "advect":
                s.mac_advect(dt)
            else:
                s.mac_diffuse_smagorinsky(0.2, 0.17, dt)
            want, want_nut = refm.state()
            got = s.get_faces()
            for c in range(3):
                err = np.abs(got[c][keep] - want[c][keep]).max()
                changed = np.abs(want[c][keep] - (u, v, w)[c][keep]).max()
                print(f"{name} component {c}: max |diff| {err:.3e}, max change {changed:.3e}")
                assert changed > 1e-4, (name, c)           # the step did something
                assert err <= 1e-6 * 12.0, (name, c, err)
            if name == "diffuse":
                nut = s.mac_eddy_viscosity()
                scale = float(np.abs(want_nut[cell_keep]).max())
                assert scale > 0
                assert np.abs(nut[cell_keep] - want_nut[cell_keep]).max() <= 1e-6 * scale
            # the next check starts from the reference's result
            u, v, w = want
    refm.close()


def flow_at(points, component, speed=10.0):
    """The initial_faces flow evaluated at arbitrary points [n][3], one component per point."""
    x, y, z = points[:, 0], points[:, 1], points[:, 2]
    u = speed * (1.0 + 0.2 * np.sin(1.3 * x + 0.7 * y) * np.cos(0.9 * z))
    v = speed * 0.15 * np.cos(0.8 * x - 1.1 * z) * np.sin(0.6 * y + 0.3)
    w = speed * 0.1 * np.sin(0.5 * x + 0.9 * y - 0.4 * z)
    return np.choose(component, [u, v, w]).astype(np.float32)


def test_aperture_transport_matches_reference(wing):
    """transport_embedded_apertures (the MAC step's compact EB face transport) against the
    reference's own projection on the same faces and special velocities.  Both accumulate node
    sums with FP32 atomics in launch order, so the results agree to FP32 rounding of those sums
    (1e-5 of the velocity scale asserted)."""
    t = wing.topology
    u, v, w = initial_faces(t)
    ncf, neb = wing.summary["coarse_fine"], wing.summary["embedded"]
    assert neb > 0
    cf_pts = np.ctypeslib.as_array(t.coarse_fine.face_centroid, shape=(ncf * 3,)).reshape(-1, 3)
    cf_axis = np.ctypeslib.as_array(t.coarse_fine.axis, shape=(ncf,)).astype(int)
    eb_pts = np.ctypeslib.as_array(t.embedded.face_centroid, shape=(neb * 3,)).reshape(-1, 3)
    eb_axis = np.ctypeslib.as_array(t.embedded.axis, shape=(neb,)).astype(int)
    cf = flow_at(cf_pts, cf_axis)
    eb = flow_at(eb_pts, eb_axis)
    h = min(t.levels[l].h for l in range(t.level_count))
    dt = 0.5 * h / 12.0
    keep = non_covered_faces(t)
    refm = ref.RefMac(wing, 2.5)
    refm.set_faces(u, v, w)
    refm.set_special(cf.astype(np.float64), eb.astype(np.float64))
    refm.transport_apertures(dt, 1.5e-5, 0.17)
    (ru, rv, rw), _ = refm.state()
    rcf, reb = refm.special()
    refm.close()
    with CompositeSystem(t) as s:
        s.set_faces(u, v, w)
        s.set_special(cf, eb)
        s.mac_transport_apertures(dt, 1.5e-5, 0.17)
        gu, gv, gw = s.get_faces()
        gcf, geb = s.get_special()
    changed = np.abs(reb - eb).max()
    err = np.abs(geb - reb).max()
    print(f"apertures: max |diff| {err:.3e}, max change {changed:.3e}")
    assert changed > 1e-3
    assert err <= 1e-5 * 12.0
    assert np.abs(gcf - rcf).max() <= 1e-6 * 12.0
    for g, r, orig in ((gu, ru, u), (gv, rv, v), (gw, rw, w)):
        moved = np.abs(r - orig)[keep].max()
        diff = np.abs(g - r)[keep].max()
        print(f"carrier faces: max |diff| {diff:.3e}, max change {moved:.3e}")
        assert diff <= 1e-5 * 12.0


@pytest.mark.parametrize("smooth_wall", [0, 1])
def test_mac_steps_track_reference(wing, smooth_wall):
    """Whole MAC-mode steps (ExternalAeroCore::step's staggered branch: advection, LES + diffusion,
    boundaries, compact aperture transport, the smooth fabric wall when on, coarse/fine sync,
    projection to 1e-8) against the reference's own device classes in the same sequence: dt and
    the regular face velocities agree to 1e-4 of the freestream after each of 3 steps."""
    from paracfd_b200 import MOMENTUM_MAC
    t = wing.topology
    settings = dict(speed=10.0, rho=1.225, nu=1.5e-5, cfl=0.5, smagorinsky_cs=0.10, projection_tolerance=1e-8,
                    projection_max_iterations=600)
    keep = non_covered_faces(t)
    core = ref.RefDeviceCore(wing, settings["speed"], settings["rho"], settings["nu"], settings["cfl"],
                             settings["smagorinsky_cs"], settings["projection_tolerance"],
                             settings["projection_max_iterations"], mac=True, smooth_wall=bool(smooth_wall))
    with CompositeSystem(t) as s:
        s.configure(smooth_wall=smooth_wall, **settings)
        s.set_mac_links(*wing.mac_links(2.5))
        s.set_momentum_mode(MOMENTUM_MAC)
        a, b = s.initialize(), core.initialize()
        assert a["pressure"]["converged"] and b["converged"]
        for step in range(3):
            a, b = s.step(), core.step()
            assert a["pressure"]["converged"] and b["converged"], (step, a, b)
            assert abs(a["dt"] - b["dt"]) <= 1e-4 * b["dt"], (step, a["dt"], b["dt"])
            got, want = s.get_faces(), core.faces()
            err = max(np.abs(g - r)[keep].max() for g, r in zip(got, want)) / settings["speed"]
            print(f"MAC step {step} (wall {smooth_wall}): dt {a['dt']:.6e} / {b['dt']:.6e}, face error {err:.3e} of U, "
                  f"iterations {a['pressure']['iterations']} / {b['iterations']}")
            assert err <= 1e-4, (step, err)
    core.close()
