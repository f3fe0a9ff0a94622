"""The profiling harness the profiles/ summaries cite parses its arguments on
the CPU, and its byte counts agree with the ones bench.py reports."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_profile_cases_help_lists_every_case():
    out = subprocess.run([sys.executable, "-m", "kg_b200.profile_cases", "--help"], cwd=ROOT, capture_output=True,
                         text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    for case in ("pirk", "mixed", "proj", "configured", "batch", "refine", "diag", "steppers"):
        assert case in out.stdout


def test_stage_bytes_agree_with_bench():
    sys.path.insert(0, ROOT)
    import bench
    from kg_b200.profile_cases import STAGE_BYTES
    for k, v in bench.ALG_BYTES.items():
        assert STAGE_BYTES[k] == v
