"""bench.py's reference arm on the CPU: the compiled reference's own query path on the small
closed-search workload, one JSON line with the fields the bench contract names, and no library
of this repository mapped into the process (the arm must time the reference alone)."""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")

RUN = """
import runpy, sys
sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'closed-1k', '--steps', '1', '--warmup', '3']
try:
    runpy.run_path('bench.py', run_name='__main__')
except SystemExit as e:
    if e.code not in (0, None):
        raise
maps = open('/proc/self/maps').read()
print('REPO_LIBRARY_MAPPED', 'libgicops_b200' in maps, file=sys.stderr)
"""


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="compiled reference harness not built (make -C oracle)")
def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, "-c", RUN], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["unit"] == "spectra/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 3
    assert d["config"]["workload"] == "closed-1k"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert "REPO_LIBRARY_MAPPED False" in r.stderr, r.stderr[-2000:]
