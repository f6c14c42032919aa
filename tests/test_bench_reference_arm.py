"""bench.py's reference arm runs the unmodified reference engine (oracle/_ref)
and nothing of the package under test: no import of it and no load of its
shared library.  Run at a small size on the host."""
import json
import os
import subprocess
import sys

import pytest

from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import json, runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--qubits", "16", "--steps", "4", "--warmup", "1"]
runpy.run_path("bench.py", run_name="__main__")
maps = [l.split()[-1] for l in open("/proc/self/maps") if l.rstrip().endswith(".so")]
print(json.dumps({"modules": sorted(m for m in sys.modules if "qlassical" in m),
                  "libs": sorted({p for p in maps if "qlassical" in p or "/oracle/" in p})}))
"""


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
def test_reference_arm_is_independent_of_the_package():
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [json.loads(x) for x in r.stdout.strip().splitlines()]
    line, probe = lines[0], lines[1]
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"]["sample_gates_per_step"] == 16 + 8      # whole layers: rotations + CZs
    assert probe["modules"] == []
    assert probe["libs"] and all("/oracle/_ref/" in p for p in probe["libs"]), probe["libs"]
