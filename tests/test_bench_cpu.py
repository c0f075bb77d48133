"""bench.py's reference arm on the CPU: whole reference steps, the reported timing fits the run,
and the arm never loads this library (only the reference build in oracle/_ref)."""
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_PROBE = r"""
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--workload", "naca0012_slab", "--steps", "2", "--warmup", "1",
            "--no-reference-gpu"]
try:
    runpy.run_path("bench.py", run_name="__main__")
finally:
    maps = open("/proc/self/maps").read()
    print("MAPS", int("libparacfd_b200" in maps), int("libparacfd_ref" in maps))
"""


def test_reference_arm_runs_whole_steps_without_this_library():
    t0 = time.time()
    out = subprocess.run([sys.executable, "-c", _PROBE], cwd=ROOT, capture_output=True, text=True, timeout=900)
    wall = time.time() - t0
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    maps = [l for l in out.stdout.splitlines() if l.startswith("MAPS")][0].split()
    assert maps[1:] == ["0", "1"]                      # reference build loaded, libparacfd_b200 never
    line = json.loads(lines[-1])
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 1
    assert line["ms_per_step"] * line["steps"] / 1e3 <= wall   # the timed steps ran inside this process
    cpu = line["cpu_baseline"]
    assert cpu["value"] == line["value"] and cpu["kind"] == "reference" and cpu["cores"] >= 1
    assert cpu["sample_converged_steps"] == 2
    assert line["config"]["grid"].startswith("cut-cell") and line["config"]["embedded_edges"] > 0


def test_cpu_step_boundaries_touch_exactly_the_domain_faces():
    import bench
    from paracfd_b200 import capi
    from paracfd_b200.workloads import WORKLOADS
    grid = bench.Grid(WORKLOADS["naca0012_slab"], "cutcell")
    stepper = bench.CpuStepper(grid)
    try:
        t = grid.topology
        flags = np.ctypeslib.as_array(t.levels[0].flags, shape=(t.levels[0].brick_count,))
        bs = t.brick_size
        count = lambda f: int(((flags & f) != 0).sum()) * bs * bs
        assert len(stepper.xmin) == count(capi.BRICK_XMIN)
        assert len(stepper.ywall) == count(capi.BRICK_YMIN) + count(capi.BRICK_YMAX)
        assert len(stepper.zwall) == count(capi.BRICK_ZMIN) + count(capi.BRICK_ZMAX)
        for idx in (stepper.xmin, stepper.ywall, stepper.zwall):
            assert len(np.unique(idx)) == len(idx) and idx.max() < t.levels[0].brick_count * (bs + 1) * bs * bs
        # X-min faces sit at i = 0, Y-wall faces at j = 0 / bs, Z-wall faces at k = 0 / bs
        per = (bs + 1) * bs * bs
        assert np.all((stepper.xmin % per) % (bs + 1) == 0)
        assert np.all(np.isin(((stepper.ywall % per) // bs) % (bs + 1), (0, bs)))
        assert np.all(np.isin((stepper.zwall % per) // (bs * bs), (0, bs)))
        info = stepper.initialize()
        assert info["converged"]
    finally:
        stepper.close()
        grid.close()
