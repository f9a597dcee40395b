"""GPU: the allocation-free operator entry point, QPHIX_B200_D3_asqtad_mdagm_noalloc.

Callers that cannot allocate GPU memory when they apply the operator (a
budget reserved up front, another framework's allocator in charge) use this
entry point; its scratch is a fixed array inside the library.  The test
calls it through the C ABI twice in a row -- the second call reuses the
array the first one left behind -- and compares each result with the same
quantity formed from the ordinary entry point QPHIX_D3_asqtad_dslash
(D D in - 4 m^2 in), within the FP64 Dslash tolerance of the other tests.
This file sorts last so a run stopping at the first failure has already run
everything else.
"""
import numpy as np
import pytest

from conftest import fields, rel_err, synthetic

pytestmark = pytest.mark.gpu

TOL = 1e-13  # FP64 Dslash tolerance used throughout the GPU tests


def _reference_ttt(lib, L, src, mass, parity):
    """D D in - 4 m^2 in through two QPHIX_D3_asqtad_dslash calls."""
    other = "odd" if parity == "even" else "even"
    hin = lib.create_V("D", src)
    tmp = lib.create_V("D", np.zeros_like(src))
    out = lib.create_V("D", np.zeros_like(src))
    lib.dslash("D", L, tmp, hin, other)
    lib.dslash("D", L, out, tmp, parity)
    dd = lib.extract_V("D", out)
    for h in (hin, tmp, out):
        lib.destroy_V("D", h)
    V = src.size // 6
    sl = slice(0, V * 3) if parity == "even" else slice(V * 3, V * 6)
    return dd[sl] - 4 * mass * mass * src[sl], sl


@pytest.mark.parametrize("parity", ["even", "odd"])
def test_noalloc_matches_existing_entry_point_twice(gpu, parity):
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims, seed=11)
    mass = 0.05
    L = lib.create_L("D", links)
    for call, seed in enumerate((31, 32)):
        src = synthetic.gaussian_source(dims, seed=seed, parity="evenodd")
        want, sl = _reference_ttt(lib, L, src, mass, parity)
        hin = lib.create_V("D", src)
        hout = lib.create_V("D", np.zeros_like(src))
        rc, dot = lib.mdagm_noalloc(L, hout, hin, mass, parity)
        assert rc == 0, lib.last_error()
        got = lib.extract_V("D", hout)[sl]
        lib.destroy_V("D", hin)
        lib.destroy_V("D", hout)
        assert rel_err(got, want) < TOL, f"call {call}"
        want_dot = float(np.dot(src[sl], want))
        assert abs(dot - want_dot) <= TOL * abs(want_dot) * 10, f"call {call}"
    lib.destroy_L("D", L)


def test_noalloc_refuses_lattices_beyond_its_scratch(gpu):
    lib = gpu.use((32, 32, 32, 32))  # 524288 sites per parity > 262144
    rc, _ = lib.mdagm_noalloc(None, None, None, 0.1, "even")
    assert rc == 1
    assert "at most 262144" in lib.last_error()
