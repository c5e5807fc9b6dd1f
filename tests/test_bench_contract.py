"""The bench's reference arm on the CPU: one JSON line with the fields the
driver reads (the reference's own sources built against the oracle shims,
timed on this host's cores), and no output from ranks other than 0."""
import json
import os
import subprocess
import sys

import pytest

import oracle
from conftest import ROOT


@pytest.mark.skipif(not oracle.REF_BIN.exists(), reason="oracle/_ref not built")
def test_reference_arm_line():
    p = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"], cwd=ROOT, capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    lines = [l for l in p.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "probe*slices/s"
    assert d["higher_is_better"] is True and d["steps"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_print_nothing():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"], cwd=ROOT, capture_output=True,
                       text=True, timeout=120, env=env)
    assert p.returncode == 0 and p.stdout.strip() == ""
