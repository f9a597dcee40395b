"""GPU: failure paths end in QPHIX_FAIL -- never in a fault, a trap or a
hang -- and leave the library usable.

* Bounded waits.  The TMA-pipeline Dslash (variant 2) waits on mbarriers
  for its bulk copies with a poll limit.  QPHIX_B200_set_wait_limit(0) makes
  every wait give up at once: the kernel lets the copies it issued land,
  sets the device error word and returns, and the call reports the
  failure.  Restoring the limit restores correct results.
* Breakdown guards.  The reference CG and multi-shift divide by p.Ap and
  |r|^2 unchecked (ks_d_congrad_fn.cpp:511, ks_multicg_offset.cpp:475-520),
  so a NaN source, a NaN initial guess, an Inf link or a singular operator
  (zero links at zero mass: p.Ap = 0) runs to the iteration limit and
  returns garbage.  Here every solver path -- FP64 CG, mixed CG, FP64 and
  mixed multi-shift, batched CG -- stops with QPHIX_FAIL and a message.
"""
import numpy as np
import pytest

from conftest import fields, orc, rel_err, synthetic

pytestmark = pytest.mark.gpu

DIMS = (8, 8, 8, 8)
V = int(np.prod(DIMS))


def _solve(lib, links, src, mass=0.05, inner="double", guess=None, multi=None):
    lib.set_inner_precision(inner)
    try:
        L = lib.create_L("D", links)
        b = lib.create_V("D", src, "even")
        if multi is None:
            x = lib.create_V("D", np.zeros_like(src) if guess is None else guess, "even")
            it, info, res = lib.invert("D", L, x, b, mass, parity="even", max_iter=500, nrestart=4, resid=1e-20)
            xs = [x]
        else:
            xs = [lib.create_V("D", np.zeros_like(src), "even") for _ in multi]
            it, info, res = lib.invert_multi("D", L, xs, b, multi, parity="even", max_iter=500, nrestart=4,
                                             resid=1e-20)
        err = lib.last_error()
        sol = lib.extract_V("D", xs[0], "even")
        for x in xs:
            lib.destroy_V("D", x)
        lib.destroy_V("D", b)
        lib.destroy_L("D", L)
    finally:
        lib.set_inner_precision("double")
    return info.status, err, sol


def _healthy(lib):
    """A normal solve after a failure: converged and equal to the oracle's."""
    links = fields(DIMS, seed=1001)
    src = synthetic.gaussian_source(DIMS, seed=2002, parity="even")
    status, err, x = _solve(lib, links, src)
    assert status == 0, err
    xo = orc.invert(DIMS, links, src, 0.05, "even", "D", max_iter=500, nrestart=4, resid=1e-20)[1]
    assert rel_err(x[: 3 * V], xo[: 3 * V]) < 1e-10


def test_tma_wait_timeout_reports_failure(gpu):
    lib = gpu.use(DIMS)
    links = fields(DIMS, seed=1001)
    src = synthetic.gaussian_source(DIMS, seed=3, parity="evenodd")
    L = lib.create_L("D", links)
    vin = lib.create_V("D", src)
    vout = lib.create_V("D", np.zeros_like(src))
    try:
        assert lib.set_dslash_variant(2) == 0
        assert lib.set_wait_limit(0) == 0
        lib.dslash("D", L, vout, vin, "even")  # void in the reference ABI: the error is in last_error
        assert "timed out" in lib.last_error()
        # the fused M^dag M pipeline inside a solve (graph while loop), FP64 and mixed
        for inner in ("double", "single"):
            status, err, _ = _solve(lib, links, src, inner=inner)
            assert status != 0 and "timed out" in err, (inner, err)
        assert lib.set_wait_limit(-1) == 0
        lib.dslash("D", L, vout, vin, "even")
        assert lib.last_error() == ""
        got = lib.extract_V("D", vout)[: 3 * V]
        assert rel_err(got, orc.asqtad_dslash(DIMS, links, src, "even", "D")[: 3 * V]) < 1e-13
        _healthy(lib)
    finally:
        lib.set_wait_limit(-1)
        lib.set_dslash_variant(-1)
        lib.destroy_V("D", vin)
        lib.destroy_V("D", vout)
        lib.destroy_L("D", L)


MASSES = list(np.sqrt(0.05 ** 2 + np.array([0.0, 0.01, 0.1]) / 4))


@pytest.mark.parametrize("inner", ["double", "single"])
@pytest.mark.parametrize("solver", ["cg", "multishift"])
def test_non_finite_source_and_guess(gpu, inner, solver):
    lib = gpu.use(DIMS)
    links = fields(DIMS, seed=1001)
    src = synthetic.gaussian_source(DIMS, seed=2002, parity="even")
    bad = src.copy()
    bad[17] = np.nan
    multi = MASSES if solver == "multishift" else None
    status, err, _ = _solve(lib, links, bad, inner=inner, multi=multi)
    assert status != 0 and "not finite" in err, err
    if solver == "cg":
        guess = np.zeros_like(src)
        guess[5] = np.inf
        status, err, _ = _solve(lib, links, src, inner=inner, guess=guess)
        assert status != 0 and "not finite" in err, err
    _healthy(lib)


@pytest.mark.parametrize("inner", ["double", "single"])
@pytest.mark.parametrize("solver", ["cg", "multishift"])
def test_breakdown_zero_operator(gpu, inner, solver):
    """Zero links at zero mass: M = 0, so p.Ap = 0 in the first iteration."""
    lib = gpu.use(DIMS)
    zero = {k: np.zeros(V * 72) for k in ("fat", "lng", "fatback", "lngback")}
    src = synthetic.gaussian_source(DIMS, seed=2002, parity="even")
    multi = [0.0, 0.1, 0.2] if solver == "multishift" else None
    status, err, _ = _solve(lib, zero, src, mass=0.0, inner=inner, multi=multi)
    assert status != 0 and "breakdown" in err, err
    _healthy(lib)


def test_inf_link(gpu):
    lib = gpu.use(DIMS)
    links = dict(fields(DIMS, seed=1001))
    links["fat"] = links["fat"].copy()
    links["fat"][72 * 11 + 3] = np.inf
    src = synthetic.gaussian_source(DIMS, seed=2002, parity="even")
    for inner in ("double", "single"):
        status, err, _ = _solve(lib, links, src, inner=inner)
        assert status != 0 and ("breakdown" in err or "not finite" in err), (inner, err)
    _healthy(lib)


def test_batch_non_finite_and_breakdown(gpu):
    lib = gpu.use(DIMS)
    links = fields(DIMS, seed=1001)
    src = synthetic.gaussian_source(DIMS, seed=2002, parity="even")
    bad = src.copy()
    bad[3] = np.nan
    B = lib.batch_create_L([(DIMS, links)])
    try:
        it, info, res, xs = lib.batch_invert(B, [(0, 0.05, src), (0, 0.05, bad)])
        assert info.status != 0 and "non-finite" in lib.last_error()
        it, info, res, xs = lib.batch_invert(B, [(0, 0.05, src), (0, 0.07, src)])
        assert info.status == 0, lib.last_error()
    finally:
        lib.batch_destroy_L(B)
    zero = {k: np.zeros(V * 72) for k in ("fat", "lng", "fatback", "lngback")}
    B = lib.batch_create_L([(DIMS, zero)])
    try:
        it, info, res, xs = lib.batch_invert(B, [(0, 0.0, src)])
        assert info.status != 0 and "breakdown" in lib.last_error()
    finally:
        lib.batch_destroy_L(B)
    _healthy(lib)
