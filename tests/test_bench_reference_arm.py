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


def test_reference_arm_loads_no_cuda_library():
    """The reference arm times the reference alone: after a full run of it in
    one process, no shared object of the CUDA package is mapped there, and its
    halfedge total is the reference's own count."""
    from oracle import refimpl
    if not refimpl.available():
        pytest.skip("oracle/_ref not built")
    code = (
        "import sys, json, io, contextlib\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0']\n"
        "import bench\n"
        "buf = io.StringIO()\n"
        "with contextlib.redirect_stdout(buf):\n"
        "    rc = bench.run_reference(bench.parse())\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'rc': rc, 'line': buf.getvalue().strip().splitlines()[-1],\n"
        "                  'cuda_lib': 'libccs_cuda' in maps, 'ref_lib': 'libccref.so' in maps}))\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["rc"] == 0 and out["ref_lib"] and not out["cuda_lib"]
    line = json.loads(out["line"])
    from halfedgecatmullclark_b200 import configs, metrics
    from halfedgecatmullclark_b200.subd import level_counts
    w = configs.mixed_torus(depth=6)
    assert line["config"]["refined_halfedges_per_step"] == metrics.total_halfedges(level_counts(w.cage, 6))
