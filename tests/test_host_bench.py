"""bench.py's reference arm on the CPU: the reference's own code (the
library compiled from its sources into oracle/_ref) timed on the 147-atom
workload, printing one JSON line with the keys of the GPU arm's line."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def test_reference_arm_prints_one_contract_line():
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("the reference library is not built (no reference sources here)")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "c1",
                        "--steps", "2", "--warmup", "3"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["metric"] == "atom-steps/s" and line["unit"] == "atom-steps/s"
    assert line["higher_is_better"] is True and line["value"] > 0 and line["steps"] == 2
    assert line["config"]["name"] == "c1"
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
