"""CPU: the JSON-line contract of bench.py's reference arm, and the
reference Dslash timing mode (both run the reference's host code from
oracle/_ref on the host cores; no GPU).

The reference arm must print exactly one JSON line on stdout with the keys the
benchmark driver reads, with its cpu_baseline and e2e objects; the reference
host code's own progress lines go to stderr."""
import json
import os
import subprocess
import sys

import pytest

from conftest import orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    if not os.path.exists(orc.REF_LIB):
        pytest.skip("reference host-code oracle not built (reference sources absent)")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, p.stdout[-2000:]
    return json.loads(lines[0])


def test_reference_arm_prints_one_contract_line():
    d = _run("--impl", "reference", "--steps", "1", "--warmup", "0", "--ref-iters", "2")
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "s" and d["higher_is_better"] is False
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_dslash_mode():
    d = _run("--mode", "dslash", "--impl", "reference", "--lattice", "8x8x8x8", "--reps", "2")
    assert d["impl"] == "reference" and d["lattice"] == "8x8x8x8"
    for prec in ("F", "D"):
        assert d[prec]["us"] > 0 and d[prec]["gbs"] > 0
