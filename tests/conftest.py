"""Shared fixtures of the qphix_b200 test suite.

Markers: ``gpu`` -- needs a B200 (run with ``-m gpu``); everything else runs
on CPU.  CPU tests cover the oracle against the reference host code and the
golden fixtures, the host logic and the C-ABI exports; GPU tests compare the
product library, called through its C ABI, with the oracle.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import __graft_entry__ as entry  # noqa: E402

entry.load_package()

from milc_qphix_b200 import LIB_PATH, capi, synthetic  # noqa: E402
import orc  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (product library on cuda:0)")


@pytest.fixture(scope="session")
def product_lib_path():
    if not os.path.exists(LIB_PATH):
        entry._make(os.path.join(ROOT, "milc-qphix_b200"))
    return LIB_PATH


@pytest.fixture(scope="session")
def ref_lib():
    """The reference's own host code + restated kernel (oracle/_ref)."""
    if not os.path.exists(orc.REF_LIB):
        # the oracle recipe builds oracle/_ref only where the reference sources are
        entry.make_oracle()
        if not os.path.exists(orc.REF_LIB):
            pytest.skip("reference host-code oracle not built (reference sources absent)")
    return capi.QphixLib(orc.REF_LIB)


class Session:
    """Product library initialised for one lattice at a time."""

    def __init__(self, path):
        self.lib = capi.QphixLib(path)
        self.dims = None

    def use(self, dims):
        dims = tuple(dims)
        if self.dims != dims:
            if self.dims is not None:
                self.lib.finalize()
            rc = self.lib.init(dims)
            assert rc == 0, self.lib.last_error()
            self.dims = dims
        return self.lib


@pytest.fixture(scope="session")
def gpu(product_lib_path):
    s = Session(product_lib_path)
    yield s
    if s.dims is not None:
        s.lib.finalize()


_field_cache = {}


def fields(dims, seed=1001, smear=False, eps_fat=0.3, eps_long=0.3):
    key = (tuple(dims), seed, smear, eps_fat, eps_long)
    if key not in _field_cache:
        _field_cache[key] = synthetic.asqtad_links(dims, seed=seed, smear=smear,
                                                   eps_fat=eps_fat, eps_long=eps_long)
    return _field_cache[key]


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
