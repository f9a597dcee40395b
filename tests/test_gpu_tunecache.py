"""GPU: the autotuner's persistent cache (QPHIX_B200_TUNECACHE).

A first process times the Dslash variants and writes one line per (kernel,
GPU model, volume, vector precision, link storage) to the cache file; a
second process with the same file reads the choice and the timings back
instead of timing again (its reported timings are the first process's,
digit for digit).  An unreadable or stale line only costs a new timing.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.gpu

CHILD = r"""
import json, sys
sys.path.insert(0, ROOT)
import numpy as np
import __graft_entry__ as e
e.load_package()
from milc_qphix_b200 import LIB_PATH, capi, synthetic
dims = (8, 8, 8, 8)
lib = capi.QphixLib(LIB_PATH)
assert lib.init(dims) == 0, lib.last_error()
links = synthetic.asqtad_links(dims, seed=1001)
src = synthetic.gaussian_source(dims, seed=5, parity="evenodd")
L = lib.create_L("F", links)
vi = lib.create_V("F", src)
vo = lib.create_V("F", np.zeros_like(src))
lib.dslash("F", L, vo, vi, "even")
print(json.dumps(lib.tuning("single")))
lib.finalize()
""".replace("ROOT", repr(ROOT))


def _child(cache):
    env = dict(os.environ, QPHIX_B200_TUNECACHE=str(cache))
    env.pop("QPHIX_B200_DSLASH", None)
    p = subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    return json.loads(p.stdout.strip().splitlines()[-1])


def test_second_process_reads_the_choice(tmp_path):
    cache = tmp_path / "tune.txt"
    v1, us1 = _child(cache)
    lines = cache.read_text().splitlines()
    assert any(ln.startswith("dslash:") and ":vh2048:v1:l1 " in ln for ln in lines), lines
    v2, us2 = _child(cache)
    assert (v1, us1) == (v2, us2)
    # a line of the wrong length is ignored and the variant timed again
    cache.write_text("\n".join(ln.split()[0] + " 1 2" for ln in lines) + "\n")
    v3, us3 = _child(cache)
    assert v3 in (0, 1, 2, 3) and us3 != [1.0, 2.0, 0.0, 0.0]
