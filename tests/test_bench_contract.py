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
    """Every timed step is one full FP64 solve, measured: on a small lattice
    here (the benchmark runs 24^3x48), the solve reaches the tolerance and
    the config object is the one the GPU arm prints."""
    sys.path.insert(0, ROOT)
    import bench

    d = _run("--impl", "reference", "--steps", "2", "--warmup", "1", "--ref-iters", "2", "--lattice", "8x8x8x8")
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "s" and d["higher_is_better"] is False
    assert d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1
    assert d["config"] == bench.bench_config(1, (8, 8, 8, 8))
    assert "FP64 CG" in d["solver"] and d["dtype"] == "f64"
    sol = d["solve"]
    # the reference's OpenMP reductions are not reproducible run to run: at this
    # light mass two solves of the same system can differ by a few per cent
    its = sol["iterations"]
    assert len(sol["s_each"]) == 2 and min(its) > 50 and max(its) <= 1.05 * min(its)
    assert sol["true_rsq_rel"] < 1e-20
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_dslash_mode():
    d = _run("--mode", "dslash", "--impl", "reference", "--lattice", "8x8x8x8", "--reps", "2")
    assert d["impl"] == "reference" and d["lattice"] == "8x8x8x8"
    for prec in ("F", "D"):
        assert d[prec]["us"] > 0 and d[prec]["gbs"] > 0
