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
