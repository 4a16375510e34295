"""bench.py --impl reference: the reference's own CPU step (oracle/_ref),
timed on the host cores, prints one JSON line with the own arm's metric and
unit, impl "reference", a cpu_baseline describing the run and an e2e object
with no host-device copies. On CPU the test runs it on the 100k dam
(--scene 100k); the bench's default is the 1M dam itself."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from oracle import ref_oracle as R  # noqa: E402

import bench  # noqa: E402


@pytest.mark.skipif(not (R.available("omp") or R.available("serial")), reason="oracle/_ref is not built")
def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3", "--scene", "100k"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [x for x in out.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT and d["higher_is_better"] is True
    assert d["steps"] == 1 and 1 <= d["warmup"] <= 3 and d["value"] > 0
    assert d["config"]["same_config"] is False   # the 100k dam stands in for the 1M dam here, for time
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
