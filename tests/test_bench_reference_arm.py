"""bench.py --impl reference prints one JSON line with the contract keys
(small grid; skipped without the reference build)."""
import json
import os
import subprocess
import sys

import pytest

import harmtest as ht

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("n,fluxadjust", [(16, 0), (32, 3)])
def test_reference_arm_json_line(n, fluxadjust):
    if ht.ref_lib_path(n, n, "torusfa" if fluxadjust else "torus") is None:
        pytest.skip("reference build (oracle/_ref) not present")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", str(n),
                          "--steps", "3", "--warmup", "1", "--fluxadjust", str(fluxadjust)], capture_output=True,
                         text=True, timeout=300, check=True)
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "dtype", "config", "impl", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
    # the same window and work as the b200 arm's same_window row, the baseline built for this host
    assert line["window"] == "steps 3-5 from init" and line["config"]["fluxadjust"] == fluxadjust
    assert "-O3 -march=native" in line["build"]
