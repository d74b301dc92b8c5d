"""python -m aerocfd_b200.run: one synthetic workload through the library,
its JSON line and a clean device status."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("args", [["--case", "bump", "--no-autotune"],
                                  ["--case", "naca", "--mixed", "--no-autotune", "--inviscid", "8"]])
def test_runner_prints_throughput(args):
    p = subprocess.run([sys.executable, "-m", "aerocfd_b200.run", "--steps", "3", "--warmup", "3", *args],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["value"] > 0 and line["device_status"] == 0
