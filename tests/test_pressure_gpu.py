"""GPU parity of the composite pressure operator, projection and solver against the reference's
own host implementation (oracle/_ref, compiled from the reference sources) on reference-built
cut-cell topologies."""
import numpy as np
import pytest

from oracle import port, ref
from paracfd_b200 import CompositeSystem, MG_FP32, MG_FP64

pytestmark = pytest.mark.gpu

CASES = {
    "box2": lambda: ref.box_case(),                                  # 2 levels, 8192 c/f + EB, WLS
    "naca16": lambda: ref.naca_slab_case(base_cell_size=1 / 16),     # 1 level, NACA 0012 slab
}


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request, gpu):
    rc = CASES[request.param]()
    sysm = CompositeSystem(rc.topology)
    yield rc, sysm
    sysm.close()
    rc.close()


def rel(a, b, mask=None):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    if mask is not None:
        a, b = a[mask], b[mask]
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_operator_apply_matches_reference(case):
    rc, sysm = case
    rng = np.random.default_rng(7)
    p = rng.standard_normal(rc.n) * rc.active
    # FP64 operator: <= 1e-12 relative max-norm against CompositeAmrPressureSystem::apply_cpu
    assert rel(sysm.apply(p), rc.apply(p)) <= 1e-12


def test_diagonal_matches_reference(case):
    rc, sysm = case
    assert rel(sysm.diagonal(), rc.diagonal()) <= 1e-13


def random_faces(rc, seed):
    rng = np.random.default_rng(seed)
    u, v, w = (rng.standard_normal(rc.faces).astype(np.float32) for _ in range(3))
    cf = rng.standard_normal(rc.summary["coarse_fine"]).astype(np.float32)
    eb = rng.standard_normal(rc.summary["embedded"]).astype(np.float32)
    return u, v, w, cf, eb


def test_divergence_and_rhs_match_reference(case):
    rc, sysm = case
    u, v, w, cf, eb = random_faces(rc, 11)
    sysm.set_faces(u, v, w)
    sysm.set_special(cf, eb)
    div_ref = rc.divergence(u, v, w, cf.astype(np.float64), eb.astype(np.float64))
    # FP32 output of an FP64 sum: one rounding -> 2 ulp of float relative to the field scale
    assert rel(sysm.divergence(), div_ref) <= 2e-6
    rho, dt = 1.225, 3e-3
    rhs_ref = rc.rhs(u, v, w, cf.astype(np.float64), eb.astype(np.float64), rho, dt)
    assert rel(sysm.projection_rhs(rho, dt), rhs_ref) <= 1e-12


def test_flux_correction_matches_reference(case):
    rc, sysm = case
    u, v, w, cf, eb = random_faces(rc, 13)
    p = np.random.default_rng(5).standard_normal(rc.n) * rc.active
    rho, dt = 1.225, 2e-3
    sysm.set_faces(u, v, w)
    sysm.set_special(cf, eb)
    sysm.set_pressure(p)
    sysm.correct_fluxes(rho, dt)
    gu, gv, gw = sysm.get_faces()
    gcf, geb = sysm.get_special()
    ru, rv, rw, rcf, reb = rc.correct_fluxes(p, rho, dt, u, v, w, cf.astype(np.float64), eb.astype(np.float64))
    # Special velocities: FP64 derivative, one FP32 rounding on both sides.
    assert rel(geb, reb.astype(np.float32)) <= 1e-6 if len(reb) else True
    assert rel(gcf, rcf.astype(np.float32)) <= 1e-6 if len(rcf) else True
    # Regular faces: the device additionally re-syncs 2:1 tile faces from the compact
    # velocities (reference device bridge); compare every face the host twin owns.
    if rc.summary["coarse_fine"] == 0:
        for g, r in ((gu, ru), (gv, rv), (gw, rw)):
            assert rel(g, r) <= 1e-6
    else:
        for g, r, orig in ((gu, ru, u), (gv, rv, v), (gw, rw, w)):
            moved_by_twin = r != orig
            assert rel(g[moved_by_twin], r[moved_by_twin]) <= 1e-6


@pytest.mark.parametrize("precision,cycle", [(MG_FP64, 0), (MG_FP32, 0), (MG_FP64, 1), (MG_FP32, 1)])
def test_solve_reaches_tolerance_on_reference_operator(case, precision, cycle):
    rc, _ = case
    rng = np.random.default_rng(3)
    b = rng.standard_normal(rc.n) * rc.active
    with CompositeSystem(rc.topology, mg_precision=precision, mg_cycle=cycle) as s:
        x, res = s.solve(b, 1e-8, 600)
    assert res["converged"], res
    true = np.linalg.norm((b - rc.apply(x))[rc.active.astype(bool)]) / np.linalg.norm(b)
    assert true <= 1e-8 * 1.01, (true, res)


@pytest.mark.parametrize("cycle", [0, 2])
def test_delayed_orthogonalisation_reaches_tolerance(case, cycle):
    """Delayed CGS2 (one dot and one update pass per column, the previous basis vector
    reorthogonalised late) solves to the same true residual as the three-pass CGS2, and in about
    the same number of iterations."""
    rc, _ = case
    rng = np.random.default_rng(5)
    b = rng.standard_normal(rc.n) * rc.active
    act = rc.active.astype(bool)
    out = {}
    for delayed in (0, 1):
        with CompositeSystem(rc.topology, mg_cycle=cycle, gmres_delayed=delayed) as s:
            for _ in range(2):   # the second solve starts from the recycled subspace
                x, res = s.solve(b * (1.0 + 0.1 * _), 1e-8, 600)
                assert res["converged"], (delayed, res)
                true = np.linalg.norm((b * (1.0 + 0.1 * _) - rc.apply(x))[act]) / np.linalg.norm(b * (1.0 + 0.1 * _))
                assert true <= 1e-8 * 1.01, (delayed, true, res)
            out[delayed] = res["iterations"]
    assert out[1] <= out[0] + 2, out


def test_fp16_stage_coefficients_reach_tolerance(case):
    """The composite stages with FP16 coefficients (FP32 multigrid) still precondition a solve
    to the FP64 true residual of the reference operator."""
    rc, _ = case
    rng = np.random.default_rng(8)
    b = rng.standard_normal(rc.n) * rc.active
    act = rc.active.astype(bool)
    with CompositeSystem(rc.topology, mg_precision=MG_FP32, mg_cycle=2, mg_stage_fp16=1) as s:
        x, res = s.solve(b, 1e-8, 600)
    assert res["converged"], res
    true = np.linalg.norm((b - rc.apply(x))[act]) / np.linalg.norm(b)
    assert true <= 1e-8 * 1.01, (true, res)


def test_fused_preconditioner_matches_separate_launches_and_oracle(case):
    """The brick-fused fine level runs the same Jacobi sweeps; only the aggregate restriction
    sums in another order, so the result agrees with the separate-launch path and with the CPU
    restatement of the reference cycle to FP64 rounding."""
    rc, fused = case
    assert fused.fused_preconditioner
    rng = np.random.default_rng(17)
    r = rng.standard_normal(rc.n) * rc.active
    with CompositeSystem(rc.topology, fused_smoother=False) as plain:
        assert not plain.fused_preconditioner
        z_plain = plain.precondition(r)
    z = fused.precondition(r)
    act = rc.active.astype(bool)
    assert rel(z, z_plain, act) <= 1e-12
    oracle = port.PortSystem(rc.topology)
    assert rel(z, oracle.precondition(r), act) <= 1e-12
    oracle.close()
    # repeated applications are identical (deterministic reductions, ping-pong buffers reset)
    assert np.array_equal(z, fused.precondition(r))


def test_corrected_cycle_fused_matches_separate_launches(case):
    """The over-corrected cycle scales the same prolongations in both implementations."""
    rc, _ = case
    r = np.random.default_rng(19).standard_normal(rc.n) * rc.active
    with CompositeSystem(rc.topology, mg_cycle=1) as fused, CompositeSystem(rc.topology, mg_cycle=1,
                                                                            fused_smoother=False) as plain:
        assert fused.fused_preconditioner and not plain.fused_preconditioner
        act = rc.active.astype(bool)
        assert rel(fused.precondition(r), plain.precondition(r), act) <= 1e-12


def test_fp32_fused_fine_level_matches_fp64_fine_level(case):
    """FP32 multigrid: the fused cycle runs the fine sweeps on float copies; the separate-launch
    cycle keeps the fine level in double.  They agree to float rounding."""
    rc, _ = case
    r = np.random.default_rng(29).standard_normal(rc.n) * rc.active
    with CompositeSystem(rc.topology, mg_precision=MG_FP32) as fused, \
            CompositeSystem(rc.topology, mg_precision=MG_FP32, fused_smoother=False) as plain:
        assert fused.fused_preconditioner
        act = rc.active.astype(bool)
        assert rel(fused.precondition(r), plain.precondition(r), act) <= 1e-5


@pytest.mark.parametrize("precision", [MG_FP64, MG_FP32])
def test_composite_cycle_solves_reference_fixtures(case, precision):
    """Composite cycle on the reference fixtures (1 and 2 levels: no intermediate stage, the
    weighted prolongations and the residual-gather restriction)."""
    rc, _ = case
    b = np.random.default_rng(31).standard_normal(rc.n) * rc.active
    with CompositeSystem(rc.topology, mg_cycle=2, mg_precision=precision) as s:
        x, res = s.solve(b, 1e-8, 600)
    assert res["converged"], res
    true = np.linalg.norm((b - rc.apply(x))[rc.active.astype(bool)]) / np.linalg.norm(b)
    assert true <= 1e-8 * 1.01, (true, res)


def test_composite_cycle_on_three_level_wing_halves_iterations():
    """3-level wing grid (one intermediate composite stage): the composite cycle converges to
    1e-8 on the oracle's operator in markedly fewer iterations than the reference cycle."""
    from paracfd_b200.workloads import WORKLOADS
    built = WORKLOADS["paraglider1m"].build()
    oracle = port.PortSystem(built.topology)
    act = built.active.astype(bool)
    b = oracle.apply(np.where(act, np.random.default_rng(37).standard_normal(built.storage_size), 0.0))
    its = {}
    for cycle, precision in ((0, MG_FP64), (2, MG_FP64), (3, MG_FP32)):
        with CompositeSystem(built.topology, mg_cycle=min(cycle, 2), mg_precision=precision) as s:
            x, res = s.solve(b, 1e-8, 600)
        assert res["converged"], (cycle, res)
        true = np.linalg.norm((b - oracle.apply(x))[act]) / np.linalg.norm(b[act])
        assert true <= 1e-8 * 1.01, (cycle, true)
        its[cycle] = res["iterations"]
    oracle.close()
    built.close()
    assert its[2] <= 0.8 * its[0] and its[3] <= 0.8 * its[0], its


def test_fp64_composite_cycle_matches_oracle_restatement(case):
    """The default preconditioner (composite cycle: Galerkin stages, Chebyshev stage smoothing on
    [2/30, 2] with 6 steps, exact coarsest stage, Chebyshev-Richardson fine steps on [2/10, 2]) in
    FP64 against its CPU restatement (oracle po_set_composite), element by element."""
    rc, _ = case
    r = np.random.default_rng(41).standard_normal(rc.n) * rc.active
    act = rc.active.astype(bool)
    oracle = port.PortSystem(rc.topology)
    oracle.set_composite(6, 30, 10)
    want = oracle.precondition(r)
    oracle.close()
    with CompositeSystem(rc.topology, mg_cycle=2, mg_precision=MG_FP64, mg_stage_sweeps=6, mg_stage_chebyshev=30,
                         mg_fine_chebyshev=10) as s:
        got = s.precondition(r)
    assert rel(got, want, act) <= 1e-12


def test_composite_cycle_matches_oracle_on_three_level_cut_cell_wing(gpu):
    from tests.test_loads_gpu import WING3
    rc = ref.workload_case(WING3)
    r = np.random.default_rng(43).standard_normal(rc.n) * rc.active
    act = rc.active.astype(bool)
    oracle = port.PortSystem(rc.topology)
    want_ref = oracle.precondition(r)             # the reference cycle (lattice hierarchy)
    oracle.set_composite(6, 30, 10)
    want = oracle.precondition(r)
    oracle.close()
    with CompositeSystem(rc.topology, mg_cycle=2, mg_precision=MG_FP64) as s:
        got = s.precondition(r)
    with CompositeSystem(rc.topology, mg_cycle=0, mg_precision=MG_FP64) as s:
        got_ref = s.precondition(r)
    rc.close()
    assert rel(got, want, act) <= 1e-12
    assert rel(got_ref, want_ref, act) <= 1e-12


@pytest.mark.parametrize("precision", [MG_FP64, MG_FP32])
def test_pipeline_results_do_not_depend_on_its_grid(gpu, precision):
    """The brick pipeline's persistent CTAs walk bricks b, b + G, ... through a ring of staged
    bricks; with 1 CTA per SM each CTA walks 7 of the 1,024 bricks of the NACA slab grid, with 6
    only one or two.  The operator and the composite preconditioner (FP64 and FP32 fine levels)
    give the same bits for every grid."""
    rc = ref.naca_slab_case(base_cell_size=1 / 16)
    r = np.random.default_rng(61).standard_normal(rc.n) * rc.active
    out = []
    with CompositeSystem(rc.topology, mg_cycle=2, mg_precision=precision) as s:
        for ctas in (6, 1, 2, 3):
            s.set_pipeline_ctas(ctas)
            out.append((s.apply(r), s.precondition(r)))
    rc.close()
    for a, z in out[1:]:
        assert np.array_equal(a, out[0][0]) and np.array_equal(z, out[0][1])


def test_orthogonal_pcg_on_a_grid_without_wls_nodes(gpu):
    """A grid with no cut cells has no WLS gradient nodes; the solve then takes the reference's
    multigrid PCG (solve_orthogonal, amr_pressure.cu:1267-1353): true residual of apply_cpu <= 1e-8."""
    from paracfd_b200.workloads import WORKLOADS
    spec = WORKLOADS["paraglider1m"]
    v, t = spec.surface()
    rc = ref.case_from_mesh(v, t, spec.domain_lo, spec.domain_hi, 0.25, 1, 8, 1.0, 0.5, 2.0, 1.0)   # one level: no 2:1 tiles
    assert rc.summary["gradient_nodes"] == 0 and rc.summary["embedded"] == 0
    act = rc.active.astype(bool)
    b = rc.apply(np.random.default_rng(47).standard_normal(rc.n) * rc.active)
    for precision in (MG_FP64, MG_FP32):
        with CompositeSystem(rc.topology, mg_precision=precision) as s:
            x, res = s.solve(b, 1e-8, 600)
        assert res["converged"], res
        true = np.linalg.norm((b - rc.apply(x))[act]) / np.linalg.norm(b[act])
        assert true <= 1e-8 * 1.01, (precision, true, res)
    rc.close()


@pytest.mark.parametrize("precision,fp16,tolerance", [(MG_FP64, 0, 1e-13), (MG_FP32, 0, 1e-5), (MG_FP32, 1, 1e-5)])
def test_brick_structured_first_stage_matches_csr_stage(gpu, precision, fp16, tolerance):
    """The first composite stage as 64 rows per 8^3 brick (face neighbours from the row index,
    the other couplings as rest entries) holds the same couplings as its CSR rows; only the order
    of each row's double-precision sum differs.  On the NACA slab (1 level) and the 3-level
    cut-cell wing (coarse/fine and cut-cell couplings in the rest entries) the preconditioner
    agrees with the CSR stage to rounding."""
    from tests.test_loads_gpu import WING3
    for rc in (ref.naca_slab_case(base_cell_size=1 / 16), ref.workload_case(WING3)):
        r = np.random.default_rng(67).standard_normal(rc.n) * rc.active
        act = rc.active.astype(bool)
        out = []
        for csr in (0, 1):
            with CompositeSystem(rc.topology, mg_cycle=2, mg_precision=precision, mg_stage_fp16=fp16,
                                 mg_stage_csr=csr) as s:
                assert s.stage_brick_structured == (csr == 0)
                out.append(s.precondition(r))
        rc.close()
        assert rel(out[0], out[1], act) <= tolerance
