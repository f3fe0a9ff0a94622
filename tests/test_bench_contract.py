"""CPU check of bench.py's reference arm: it runs the CPU restatement of the
path on the host cores and prints one JSON line with the keys the benchmark
contract asks for (metric, unit and config shared with the GPU arm, a
cpu_baseline object, an e2e object with zero transfer bytes)."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3", "--grid", "64,17,33"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.strip().splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["warmup"] >= 3 and d["steps"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    # the arm runs and reports the grid it was given (the full workload grid by default)
    assert d["config"]["workload"] and d["config"]["grid"] == [64, 17, 33]
    assert "64x17x33" in cb["sample"]


def test_reference_arm_maps_only_the_oracle():
    """The reference arm imports host-only modules of the package; the solver
    library must stay unmapped in that process."""
    code = ("import sys; sys.path.insert(0, %r); import bench; "
            "bench.WORKLOAD.update(Nx=16, Ny=9, Nz=17, xmax=10.0); "
            "import argparse; a = argparse.Namespace(gpus=1, steps=1, warmup=3); bench.run_reference(a); "
            "maps = open('/proc/self/maps').read(); "
            "assert 'libkg_b200' not in maps, 'solver library mapped'; "
            "assert 'libkg_oracle' in maps" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
