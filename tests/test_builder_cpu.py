"""Host preprocessing parity (no GPU): the brick hierarchy and the composite pressure system
built by paracfd_b200 from a closed wing surface are bit-identical to the reference's
AmrHierarchy::build_static + build_composite_amr_pressure_system on the same mesh."""
import numpy as np
import pytest

from oracle import ref
from paracfd_b200 import BuiltTopology, geometry

CASES = {
    # finite NACA 4412 wing, 3 levels (2:1 tiles, skew coarse/fine WLS stencils)
    "naca4412_3lv": dict(section=(4412, 48, 6.0), span=3.0, domain_lo=(-3, -3, -3), domain_hi=(5, 3, 3),
                         base_cell_size=0.25, max_levels=3, wing_refinement_distance=0.3,
                         surface_refinement_distance=0.1, wake_length=2.0, wake_radius=0.5),
    # NACA 0012, 2 levels, different padding (domain not a brick multiple)
    "naca0012_2lv": dict(section=(12, 32, 4.0), span=2.0, domain_lo=(-1.1, -1.3, -0.9), domain_hi=(2.9, 1.2, 1.05),
                         base_cell_size=0.125, max_levels=2, wing_refinement_distance=0.2,
                         surface_refinement_distance=0.2, wake_length=1.0, wake_radius=0.4),
}


def arr(p, n):
    return np.ctypeslib.as_array(p, shape=(n,)).copy()


@pytest.fixture(scope="module", params=sorted(CASES))
def built(request):
    c = dict(CASES[request.param])
    digits, pts, aoa = c.pop("section")
    span = c.pop("span")
    v, t = geometry.extruded_wing(geometry.rotate_section(geometry.naca4_section(digits, pts), aoa), -span / 2, span / 2)
    r = ref.case_from_mesh(v, t, brick_size=8, **c)
    b = BuiltTopology(v, t, c["domain_lo"], c["domain_hi"], c["base_cell_size"], c["max_levels"], 8,
                      c["wing_refinement_distance"], c["surface_refinement_distance"], c["wake_length"],
                      c["wake_radius"], solid=False)
    yield r, b
    b.close()
    r.close()


def test_hierarchy_bit_exact(built):
    r, b = built
    R, B = r.topology, b.topology
    assert R.level_count == B.level_count
    assert list(R.domain_lo) == list(B.domain_lo) and list(R.domain_hi) == list(B.domain_hi)
    for l in range(R.level_count):
        lr, lb = R.levels[l], B.levels[l]
        assert (lr.h, lr.brick_count, lr.level_offset) == (lb.h, lb.brick_count, lb.level_offset)
        for name, k in (("coord", 3), ("origin", 3), ("neighbors", 6), ("flags", 1), ("children", 8)):
            assert np.array_equal(arr(getattr(lr, name), lr.brick_count * k), arr(getattr(lb, name), lb.brick_count * k)), name


def test_composite_system_bit_exact(built):
    r, b = built
    R, B = r.topology, b.topology
    S = R.storage_size
    assert S == B.storage_size
    for name, k in (("active", 1), ("freestream_connected", 1), ("cut_face_mask", 1), ("volume", 1), ("centroid", 3),
                    ("preconditioner_aggregate", 1)):
        assert np.array_equal(arr(getattr(R, name), S * k), arr(getattr(B, name), S * k)), name
    cr, cb = R.coarse_fine, B.coarse_fine
    assert cr.count == cb.count and cr.count > 0
    for name, k in (("coarse_dof", 1), ("fine_dof", 1), ("open_area", 1), ("centre_distance", 1), ("normal_distance", 1),
                    ("axis", 1), ("direction", 1), ("face_centroid", 3), ("orthogonal_gradient_factor", 1),
                    ("lower_gradient_node", 1), ("upper_gradient_node", 1), ("nonorthogonal_correction", 3),
                    ("upper_gradient_weight", 1)):
        assert np.array_equal(arr(getattr(cr, name), cr.count * k), arr(getattr(cb, name), cb.count * k)), name
    n = R.gradient_node_count
    assert n == B.gradient_node_count and n > 0
    assert np.array_equal(arr(R.gradient_dof, n), arr(B.gradient_dof, n))
    assert np.array_equal(arr(R.gradient_offset, n + 1), arr(B.gradient_offset, n + 1))
    nnz = R.gradient_offset[n]
    assert np.array_equal(arr(R.gradient_neighbour, nnz), arr(B.gradient_neighbour, nnz))
    assert np.array_equal(arr(R.gradient_weight, 3 * nnz), arr(B.gradient_weight, 3 * nnz))
    assert R.gauge_count == B.gauge_count == 0 and R.regular.count == B.regular.count == 0


def test_solid_classification_closes_every_control_volume():
    """Staircase solid: every fluid CV's oriented area vectors (open faces, 2:1 tiles, wall
    patches, physical boundary) sum to zero -- the reference's closure contract (< 1e-7 h^2)."""
    v, t = geometry.extruded_wing(geometry.rotate_section(geometry.naca4_section(4412, 48), 6.0), -1.5, 1.5)
    b = BuiltTopology(v, t, (-3, -3, -3), (5, 3, 3), 0.25, 3, 8, 0.3, 0.1, 2.0, 0.5, solid=True)
    T = b.topology
    S, bs = T.storage_size, T.brick_size
    active = arr(T.active, S).astype(bool)
    assert 0 < (~active).sum() and T.patches.count > 0
    closure = np.zeros((S, 3))
    c3 = bs ** 3
    for l in range(T.level_count):
        lev = T.levels[l]
        area = lev.h * lev.h
        nb = arr(lev.neighbors, lev.brick_count * 6).reshape(-1, 6)
        fl = arr(lev.flags, lev.brick_count)
        for brick in range(lev.brick_count):
            if fl[brick] & 128:
                continue
            base = lev.level_offset + brick * c3
            idx = np.arange(c3).reshape(bs, bs, bs)   # [k][j][i]
            for axis in range(3):
                for side in (-1, 1):
                    # faces of cells on the brick boundary along axis, pointing outward (side)
                    sl = [slice(None)] * 3
                    sl[2 - axis] = 0 if side < 0 else bs - 1
                    cells = base + idx[tuple(sl)].ravel()
                    inner = [slice(None)] * 3
                    n = nb[brick, 2 * axis + (side > 0)]
                    boundary = fl[brick] & (1 << (2 * axis + (side > 0)))
                    if boundary:
                        closure[cells, axis] += side * area * active[cells]
            # interior faces inside the brick
            a3 = active[base:base + c3].reshape(bs, bs, bs)
            for axis in range(3):
                lo = [slice(None)] * 3
                hi = [slice(None)] * 3
                lo[2 - axis] = slice(0, bs - 1)
                hi[2 - axis] = slice(1, bs)
                both = a3[tuple(lo)] & a3[tuple(hi)]
                ids_lo = (base + idx[tuple(lo)])[both]
                ids_hi = (base + idx[tuple(hi)])[both]
                closure[ids_lo, axis] += area
                closure[ids_hi, axis] -= area
            # faces to the same-level neighbour brick
            for axis in range(3):
                n = nb[brick, 2 * axis + 1]
                if n < 0 or fl[n] & 128:
                    continue
                sl_a = [slice(None)] * 3
                sl_b = [slice(None)] * 3
                sl_a[2 - axis] = bs - 1
                sl_b[2 - axis] = 0
                ca = base + idx[tuple(sl_a)].ravel()
                cb = lev.level_offset + n * c3 + idx[tuple(sl_b)].ravel()
                both = active[ca] & active[cb]
                closure[ca[both], axis] += area
                closure[cb[both], axis] -= area
    cf = T.coarse_fine
    coarse = arr(cf.coarse_dof, cf.count)
    fine = arr(cf.fine_dof, cf.count)
    ax = arr(cf.axis, cf.count)
    di = arr(cf.direction, cf.count)
    ar = arr(cf.open_area, cf.count)
    lower = np.where(di > 0, coarse, fine)
    upper = np.where(di > 0, fine, coarse)
    np.add.at(closure, (lower, ax), ar)
    np.add.at(closure, (upper, ax), -ar)
    P = T.patches
    normal = arr(P.normal, 3 * P.count).reshape(-1, 3)
    plus = arr(P.plus_dof, P.count)
    np.add.at(closure, plus, -normal * arr(P.area, P.count)[:, None])
    h_fine = T.levels[T.level_count - 1].h
    assert np.abs(closure[active]).max() <= 1e-7 * h_fine * h_fine
