"""The reference-side adapter (oracle/adapter/external_aero_core_b200.h), compiled against the
reference headers with the reference's real ParagliderConfig fields, runs initialize + steps on
this library beside the reference's own ExternalAeroCore on the NACA slab fixture."""
import json
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROBE = os.path.join(ROOT, "oracle", "_ref", "adapter_probe")


def test_adapter_steps_beside_the_reference_core(gpu):
    assert os.path.exists(PROBE), "build the oracle (make -C oracle adapter)"
    out = subprocess.run([PROBE, "3"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    records = json.loads(out.stdout.strip().splitlines()[-1])["records"]
    steps = [r for r in records if "step" in r or "initialize" in r]
    assert len(steps) == 4
    for r in steps:
        rec = next(iter(r.values()))
        assert rec["converged"] == [1, 1]
        assert abs(rec["dt"][0] - rec["dt"][1]) <= 1e-5 * rec["dt"][1]
        assert rec["state_error"] <= 1e-4          # the whole-step tolerance of tests/test_core_gpu.py
    loads = records[-1]["loads"]
    ours, theirs = np.array(loads["adapter"]), np.array(loads["reference"])
    assert np.abs(ours - theirs).max() <= 1e-3 * np.abs(theirs).max()
