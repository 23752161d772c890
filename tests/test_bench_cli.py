"""bench.py command-line contract that needs no GPU: the reference arm's
answers for the workloads it does not time, and the argument surface."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("workload", ["rhf_h2o16_ccpvdz", "df_h2o16_ccpvdz", "clusters256"])
def test_reference_arm_unavailable_for_non_jk_workloads(workload):
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", workload,
                        "--steps", "1", "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" in line


def test_help_lists_the_contract_flags():
    r = subprocess.run([sys.executable, "bench.py", "--help"], cwd=ROOT, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0
    for flag in ("--gpus", "--steps", "--warmup", "--impl", "--workload"):
        assert flag in r.stdout
