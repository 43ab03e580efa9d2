"""bench.py's reference arm runs QUICK's own kernel (compiled for the host)
and loads nothing of this package's native library: checked on a small
cluster in a fresh process by reading the process's own memory map."""
import json
import os
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not oracle.ref_available(), reason="QUICK host build not present")
def test_reference_arm_loads_only_the_checker():
    code = r"""
import json, sys
sys.path.insert(0, %r)
import bench
bench.WORKLOAD.update(grid=(2, 1, 1))
qps, nq, sec, raw = bench.cpu_reference(2, steps=2, warmup=1)
maps = open("/proc/self/maps").read()
print(json.dumps({"nq": nq, "raw": raw, "qps": qps,
                  "ours": "libquickb200" in maps, "quick": "libquickref" in maps}))
""" % ROOT
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    r = json.loads(out.stdout.strip().splitlines()[-1])
    assert r["quick"] and not r["ours"]
    # QUICK's own walk counts every unordered pair of kept shell pairs once
    assert 0 < r["nq"] <= r["raw"] and r["qps"] > 0
