"""Batched angle sweep: instances stepped concurrently (one host thread and one non-blocking stream
each, bench.py --sweep) give bit-identical states to the same instances stepped one after the
other (every reduction and every update of the path is deterministic); and the launch-shape
autotuner changes no result."""
import dataclasses
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from oracle import ref
from paracfd_b200 import MG_CYCLE_COMPOSITE, MG_FP32, CompositeSystem
from paracfd_b200.workloads import WORKLOADS

pytestmark = pytest.mark.gpu

SMALL = dataclasses.replace(WORKLOADS["naca4412_wing"], base_cell_size=0.2, surface_refinement_distance=0.2,
                            wing_refinement_distance=0.4, wake_length=1.0, wake_radius=0.4)


def _systems(cases):
    out = []
    for spec, rc in cases:
        s = CompositeSystem(rc.topology, MG_FP32, mg_cycle=MG_CYCLE_COMPOSITE, gmres_delayed=1, gmres_recycle=-1,
                            mg_stage_fp16=1, momentum_min_volume_fraction=spec.min_volume_fraction)
        s.configure(speed=spec.speed, **spec.case)
        out.append(s)
    return out


def _run(s, steps=3):
    s.initialize()
    iterations = [s.step()["pressure"]["iterations"] for _ in range(steps)]
    s.synchronize()
    return iterations, s.get_state(), s.get_pressure()


def test_concurrent_instances_match_sequential(gpu):
    specs = [dataclasses.replace(SMALL, aoa=a) for a in (-2.0, 3.0, 7.0)]
    cases = [(spec, ref.workload_case(spec)) for spec in specs]
    try:
        first = _systems(cases)
        sequential = [_run(s) for s in first]
        for s in first:
            s.close()
        systems = _systems(cases)
        with ThreadPoolExecutor(max_workers=len(systems)) as pool:
            concurrent = list(pool.map(_run, systems))
        for s in systems:
            s.close()
        for (its_a, state_a, p_a), (its_b, state_b, p_b) in zip(sequential, concurrent):
            assert its_a == its_b
            for a, b in zip(state_a, state_b):
                assert np.array_equal(a, b)
            assert np.array_equal(p_a, p_b)
    finally:
        for _, rc in cases:
            rc.close()


def test_autotuned_launch_shape_keeps_results(gpu):
    """The brick-pipeline autotuner times every resident-CTA count it may use and keeps the fastest;
    the grid size changes no result (each brick is computed the same way whichever CTA takes it)."""
    rc = ref.workload_case(SMALL)
    r = np.random.default_rng(5).standard_normal(rc.n) * rc.active
    with CompositeSystem(rc.topology, MG_FP32, mg_cycle=MG_CYCLE_COMPOSITE, mg_stage_fp16=1) as s:
        before = (s.apply(r), s.precondition(r))
        report = s.autotune(5)
        assert 1 <= len(report["ctas_per_sm"]) <= 8 and report["chosen"] in report["ctas_per_sm"]
        assert all(t > 0 for t in report["apply_ms"] + report["sweep_ms"])
        after = (s.apply(r), s.precondition(r))
    rc.close()
    for a, b in zip(before, after):
        assert np.array_equal(a, b)
