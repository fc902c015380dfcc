"""bench.py's reference arm on the host (CPU): the compiled reference runs the S workload through
its own code path and the JSON line carries the contract's keys. Needs the reference checkout to
compile it (the development container), so it is skipped where that is absent."""
import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

from oracle import build_ref as R  # noqa: E402


@pytest.mark.skipif(not os.path.isdir(R.REF_SRC) and not os.path.exists(os.path.join(R.OUT, "S", "ref_driver")),
                    reason="the reference checkout is not available to compile the reference arm")
def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "S", "--steps", "1",
                          "--warmup", "1"], cwd=REPO, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    line = [ln for ln in out.stdout.splitlines() if ln.startswith("{")][-1]
    d = json.loads(line)
    assert d["impl"] == "reference"
    assert d["metric"] == "ray-cell crossings/s" and d["unit"] == "crossings/s" and d["value"] > 0
    assert d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "crossings/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
