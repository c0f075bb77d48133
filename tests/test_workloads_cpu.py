"""The BASELINE config workloads as built here (CPU builder, no GPU): grid sizes, level counts
and the seeded angle sweep's per-batch cell totals."""
import numpy as np

from paracfd_b200.workloads import WORKLOADS, sweep_instances


def test_single_level_slab_is_the_128x64x64_grid():
    spec = WORKLOADS["naca0012_slab"]
    built = spec.build()
    try:
        assert built.brick_counts == [1024]          # 128 x 64 x 64 cells of h = c/32 in 8^3 bricks
        assert built.storage_size == 1024 * 512
        assert 0.95 * built.storage_size < built.leaf_cells < built.storage_size   # the section is solid
    finally:
        built.close()


def test_three_level_wing_has_about_four_million_cells():
    built = WORKLOADS["naca4412_wing"].build()
    try:
        assert len(built.brick_counts) == 3
        assert 3.8e6 < built.leaf_cells < 4.6e6
    finally:
        built.close()


def test_sweep_instances_are_seeded_and_batches_fit_8_to_20_million_cells():
    specs = sweep_instances()
    assert [s.aoa for s in specs] == [float(a) for a in range(-4, 12)]
    assert specs == sweep_instances()               # the seed fixes the refinement bands
    cells = []
    for spec in specs:
        built = spec.build()
        cells.append(built.leaf_cells)
        built.close()
    batches = [sum(cells[i:i + 4]) for i in range(0, 16, 4)]
    assert all(8e6 <= b <= 20e6 for b in batches), batches
    assert np.std(cells) > 0                         # uneven brick counts between instances


def test_cut_cell_grids_come_from_the_reference_preprocessing():
    """The bench grids: the reference's own hierarchy + cut-cell atlas + composite system of the
    workload surfaces, with no unresolved cell (the closed paraglider shell's planar tips keep its
    composite system valid)."""
    from oracle import ref
    for name, levels in (("naca0012_slab", 1), ("paraglider1m", 3)):
        case = ref.workload_case(WORKLOADS[name])
        try:
            s = case.summary
            assert s["levels"] == levels and s["unresolved"] == 0
            assert s["embedded"] > 0 and s["gradient_nodes"] > 0 and s["patches"] > 0
            assert s["storage"] > case.structured                       # EB fragments follow the bricks
        finally:
            case.close()


def test_paraglider_shell_is_closed_and_outward():
    from paracfd_b200.workloads import WORKLOADS as W
    v, t = W["paraglider16m"].surface()
    edges = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]]).astype(np.int64)
    directed = set(map(tuple, edges))
    assert len(directed) == len(edges)                                    # each directed edge once
    assert all((b, a) in directed for a, b in directed)                   # and its reverse: closed, consistent
    p0, p1, p2 = (v[t[:, q]] for q in range(3))
    assert np.einsum("ij,ij->i", p0, np.cross(p1, p2)).sum() > 0          # outward (positive volume)
