"""bench.py's reference arm runs the reference's own CPU path (no GPU): one
JSON line with the contract's keys, on the same metric and config (the op
included) as the CUDA arm's line."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

KEYS = {"impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
        "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"}


@pytest.mark.parametrize("op", ["refine", "points"])
def test_reference_arm_prints_the_contract_line(op):
    from oracle import refimpl
    if not refimpl.available():
        pytest.skip("oracle/_ref not built")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--op", op,
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert KEYS <= set(line), KEYS - set(line)
    assert line["impl"] == "reference"
    assert line["metric"] == "refined halfedges/s" and line["unit"] == "halfedges/s"
    assert line["config"]["op"] == op and line["config"]["workload"].startswith("mixed_torus")
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0


def test_reference_arm_has_no_batch_run():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "batch"],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" in line
