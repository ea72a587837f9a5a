"""The reference arm of bench.py keeps its JSON-line contract on the CPU: one line with
impl "reference", the headline metric and unit, a cpu_baseline describing the run and
an e2e block with no host-device traffic.  One bounded step (about 20 s of the
reference's own CPU solver)."""
import json
import os
import subprocess
import sys

import pytest

import oracle as O
from conftest import ROOT


@pytest.mark.skipif(not O.have_ref(), reason="compiled reference (oracle/_ref) not present")
def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"].startswith("3D 256^3 PCG solve ms") and d["unit"] == "ms"
    assert d["higher_is_better"] is False and d["value"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] == 1 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "ms", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["config"]["iterations"] > 0
