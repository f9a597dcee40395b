"""GPU: CG through the C ABI against the oracle.

FP64 (reference mode): identical iteration and restart counts, solution
within 1e-10 relative, final squared residual below the requested 1e-20.
FP32 (F3 API): iteration count within a few of the oracle (the reductions
accumulate in FP64 here, in float in the reference), solution within 1e-5.
Mixed precision (D3 with a 32- or 16-bit inner solve): FP64 true residual
|r|/|b| < 1e-10 and the solution within 1e-8 of the FP64 oracle solution.
"""
import numpy as np
import pytest

from conftest import fields, orc, rel_err, synthetic

pytestmark = pytest.mark.gpu


def _solve(lib, prec, dims, links, src, mass, parity, **kw):
    L = lib.create_L(prec, links)
    b = lib.create_V(prec, src, parity)
    x = lib.create_V(prec, np.zeros_like(src), parity)
    assert L and b and x, lib.last_error()
    it, info, res = lib.invert(prec, L, x, b, mass, parity=parity, **kw)
    assert info.status == 0, lib.last_error()
    xs = lib.extract_V(prec, x, parity)
    lib.destroy_V(prec, b)
    lib.destroy_V(prec, x)
    lib.destroy_L(prec, L)
    return it, xs, res


@pytest.mark.parametrize("parity", ["even", "odd", "evenodd"])
def test_cg_fp64_matches_oracle(gpu, parity):
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    lib.set_inner_precision("double")
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    it, x, res = _solve(lib, "D", dims, links, src, 0.05, parity, max_iter=1000, nrestart=5, resid=1e-20)
    ito, xo, reso = orc.invert(dims, links, src, 0.05, parity, "D", 1000, 5, 1e-20)
    assert (it, res.final_iter, res.final_restart) == (ito, reso.final_iter, reso.final_restart)
    assert rel_err(x, xo) < 1e-10
    assert res.final_rsq < 1e-20


def test_cg_fp64_restarts_and_cap(gpu):
    """Short restart interval and an iteration cap: the restart bookkeeping of
    ks_d_congrad_fn.cpp:360-448 (restart counts, capped iteration count)."""
    dims = (8, 4, 4, 8)
    lib = gpu.use(dims)
    lib.set_inner_precision("double")
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=9, parity="evenodd")
    for max_iter, nrestart in ((7, 40), (13, 3), (50, 1)):
        it, x, res = _solve(lib, "D", dims, links, src, 0.02, "even", max_iter=max_iter, nrestart=nrestart,
                            resid=1e-24)
        ito, xo, reso = orc.invert(dims, links, src, 0.02, "even", "D", max_iter, nrestart, 1e-24)
        assert (it, res.final_iter, res.final_restart) == (ito, reso.final_iter, reso.final_restart)
        assert rel_err(x, xo) < 1e-9
        assert abs(res.final_rsq - reso.final_rsq) <= 1e-6 * reso.final_rsq + 1e-30


def test_cg_relresid(gpu):
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    lib.set_inner_precision("double")
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    it, x, res = _solve(lib, "D", dims, links, src, 0.05, "even", max_iter=50, nrestart=8, resid=1e-16,
                        relresid=1e-6)
    ito, xo, reso = orc.invert(dims, links, src, 0.05, "even", "D", 50, 8, 1e-16, relresid=1e-6)
    assert (it, res.final_iter, res.final_restart) == (ito, reso.final_iter, reso.final_restart)
    assert abs(res.final_rel - reso.final_rel) <= 1e-6 * abs(reso.final_rel)
    assert rel_err(x, xo) < 1e-10


def test_cg_zero_source(gpu):
    dims = (8, 4, 4, 8)
    lib = gpu.use(dims)
    links = fields(dims)
    src = np.zeros(int(np.prod(dims)) * 6)
    it, x, res = _solve(lib, "D", dims, links, src, 0.05, "even", max_iter=100, nrestart=5, resid=1e-20)
    assert it == 0 and res.final_iter == 0 and res.final_rsq == 0
    assert not x.any()


def test_cg_fp32_close_to_oracle(gpu):
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    it, x, res = _solve(lib, "F", dims, links, src, 0.05, "even", max_iter=1000, nrestart=5, resid=1e-12)
    ito, xo, reso = orc.invert(dims, links, src, 0.05, "even", "F", 1000, 5, 1e-12)
    assert abs(res.final_iter - reso.final_iter) <= 5
    assert rel_err(x, xo) < 1e-5


def test_cg_parity_mismatch_is_an_error(gpu):
    dims = (8, 4, 4, 8)
    lib = gpu.use(dims)
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=9, parity="evenodd")
    L = lib.create_L("D", links)
    b = lib.create_V("D", src, "even")
    x = lib.create_V("D", np.zeros_like(src), "odd")
    it, info, res = lib.invert("D", L, x, b, 0.05, parity="even")
    assert info.status == 1 and "parities" in lib.last_error()
    lib.destroy_V("D", b)
    lib.destroy_V("D", x)
    lib.destroy_L("D", L)


@pytest.mark.parametrize("inner", ["single", "half", "half-links"])
def test_cg_mixed_reaches_fp64_tolerance(gpu, inner):
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    mass = 0.02
    lib.set_inner_precision(inner)
    try:
        it, x, res = _solve(lib, "D", dims, links, src, mass, "even", max_iter=4000, nrestart=5, resid=1e-20)
        st = lib.last_stats()
    finally:
        lib.set_inner_precision("double")
    assert res.final_rsq < 1e-20
    assert st.reliable_updates >= 2
    # FP64 true residual recomputed by the oracle
    assert orc.true_residual(dims, links, x, src, mass, "even") < 1e-20
    _, xo, _ = orc.invert(dims, links, src, mass, "even", "D", 4000, 5, 1e-22)
    V = int(np.prod(dims))
    assert rel_err(x[: V * 3], xo[: V * 3]) < 1e-8


def test_cg_mixed_evenodd(gpu):
    dims = (8, 4, 4, 8)
    lib = gpu.use(dims)
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=4, parity="evenodd")
    lib.set_inner_precision("single")
    try:
        it, x, res = _solve(lib, "D", dims, links, src, 0.05, "evenodd", max_iter=2000, nrestart=5, resid=1e-20)
    finally:
        lib.set_inner_precision("double")
    _, xo, _ = orc.invert(dims, links, src, 0.05, "evenodd", "D", 2000, 5, 1e-22)
    assert rel_err(x, xo) < 1e-8
