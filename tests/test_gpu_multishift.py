"""GPU: multi-shift CG through the C ABI against the oracle.

Reference mode (FP64 D3 / FP32 F3): the reference's recurrence on the
device; FP64 must give the oracle's iteration count, flop count and
solutions to 1e-10.  Mixed mode (D3 with a 32- or 16-bit inner solve): every
shift reaches its FP64 true-residual tolerance.
"""
import numpy as np
import pytest

from conftest import fields, orc, rel_err, synthetic

pytestmark = pytest.mark.gpu


def _masses(m0=0.05, n=5):
    sig = np.logspace(-3, 0, n)
    m = np.sqrt(m0 ** 2 + sig / 4)
    return np.concatenate([m[2:], m[:2]])  # the lightest mass is not first


def _multi(lib, prec, links, src, masses, parity, **kw):
    L = lib.create_L(prec, links)
    b = lib.create_V(prec, src, parity)
    outs = [lib.create_V(prec, np.zeros_like(src), parity) for _ in masses]
    it, info, res = lib.invert_multi(prec, L, outs, b, masses, parity=parity, **kw)
    assert info.status == 0, lib.last_error()
    xs = [lib.extract_V(prec, o, parity) for o in outs]
    for h in outs + [b]:
        lib.destroy_V(prec, h)
    lib.destroy_L(prec, L)
    return it, xs, res, info


@pytest.mark.parametrize("parity", ["even", "odd", "evenodd"])
def test_multishift_fp64_matches_oracle(gpu, parity):
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    lib.set_inner_precision("double")
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    masses = _masses()
    it, xs, res, info = _multi(lib, "D", links, src, masses, parity, max_iter=1000, nrestart=5, resid=1e-20)
    ito, xo, reso, info_o = orc.invert_multi(dims, links, src, masses, parity, "D", 1000, 5, 1e-20)
    assert it == ito
    assert [r.final_iter for r in res] == [r.final_iter for r in reso]
    assert info.final_flop == info_o.final_flop
    for a, b in zip(xs, xo):
        assert rel_err(a, b) < 1e-10


def test_multishift_fp64_not_converged_path(gpu):
    """Iteration cap reached (ks_multicg_offset.cpp:626-653)."""
    dims = (8, 4, 4, 8)
    lib = gpu.use(dims)
    lib.set_inner_precision("double")
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=3, parity="evenodd")
    masses = _masses(0.01, 4)
    it, xs, res, info = _multi(lib, "D", links, src, masses, "even", max_iter=10, nrestart=3, resid=1e-30)
    ito, xo, reso, _ = orc.invert_multi(dims, links, src, masses, "even", "D", 10, 3, 1e-30)
    assert it == ito == 30
    assert abs(res[0].final_rsq - reso[0].final_rsq) <= 1e-8 * reso[0].final_rsq
    for a, b in zip(xs, xo):
        assert rel_err(a, b) < 1e-10


def test_multishift_fp32_close(gpu):
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    masses = _masses()
    it, xs, res, info = _multi(lib, "F", links, src, masses, "even", max_iter=1000, nrestart=5, resid=1e-12)
    ito, xo, reso, _ = orc.invert_multi(dims, links, src, masses, "even", "F", 1000, 5, 1e-12)
    assert abs(it - ito) <= 5
    for a, b in zip(xs, xo):
        assert rel_err(a, b) < 2e-5


@pytest.mark.parametrize("inner", ["single", "half", "half-links"])
def test_multishift_mixed_every_shift_converges(gpu, inner):
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    masses = _masses(0.02, 6)
    lib.set_inner_precision(inner)
    try:
        it, xs, res, info = _multi(lib, "D", links, src, masses, "even", max_iter=4000, nrestart=5, resid=1e-20)
    finally:
        lib.set_inner_precision("double")
    for m, x, r in zip(masses, xs, res):
        assert r.final_rsq < 1e-20
        assert orc.true_residual(dims, links, x, src, m, "even") < 1e-20


def test_multishift_mixed_deferred_matches_explicit_updates(gpu, monkeypatch):
    """The deferred shift updates (stored residuals, coefficients expanded on
    the device, one FP64 flush per segment) against the per-iteration
    updates they replace (QPHIX_B200_MS_DEFER=0: x_j and p_j updated every
    iteration, x_j in FP32 partial sums): the base recurrence takes the same
    iterations to within the rounding of the base solution its reliable
    updates read (FP64 expansion against FP32 partial sums), both meet every
    shift's tolerance against the oracle, and the two sets of solutions agree
    to the tolerance's level."""
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="even")
    masses = _masses(0.01, 6)
    V = int(np.prod(dims))
    out = {}
    lib.set_inner_precision("single")
    try:
        for defer in ("1", "0"):
            monkeypatch.setenv("QPHIX_B200_MS_DEFER", defer)
            out[defer] = _multi(lib, "D", links, src, masses, "even", max_iter=4000, nrestart=5, resid=1e-20)
    finally:
        lib.set_inner_precision("double")
    assert abs(out["1"][0] - out["0"][0]) <= 2, (out["1"][0], out["0"][0])
    for defer in ("1", "0"):
        it, xs, res, info = out[defer]
        for m, x, r in zip(masses, xs, res):
            assert r.final_rsq < 1e-20
            assert orc.true_residual(dims, links, x, src, m, "even") < 1e-20, defer
    for a, b in zip(out["1"][1], out["0"][1]):
        assert rel_err(a[: 3 * V], b[: 3 * V]) < 1e-8


def test_multishift_mixed_short_segments(gpu, monkeypatch):
    """FP32 Krylov vectors: the shifted solutions and directions are rebuilt
    from the stored base residuals once per segment.  Segments of 16
    iterations (QPHIX_B200_MS_SEGMENT) hand over many times inside one
    recurrence; the solutions still meet every shift's tolerance against the
    oracle, and the sloppy recurrence takes the iterations of the run with
    the default segments (the base direction is updated identically; only
    the summation order of the deferred solutions differs)."""
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="even")
    masses = _masses(0.01, 6)
    lib.set_inner_precision("single")
    try:
        it0, xs0, res0, _ = _multi(lib, "D", links, src, masses, "even", max_iter=4000, nrestart=5, resid=1e-20)
        monkeypatch.setenv("QPHIX_B200_MS_SEGMENT", "16")
        it1, xs1, res1, info = _multi(lib, "D", links, src, masses, "even", max_iter=4000, nrestart=5, resid=1e-20)
    finally:
        lib.set_inner_precision("double")
    assert info.status == 0
    assert it0 > 3 * 16, "the recurrence must span several segments"
    assert abs(it1 - it0) <= 2, (it0, it1)
    for m, x, r in zip(masses, xs1, res1):
        assert r.final_rsq < 1e-20
        assert orc.true_residual(dims, links, x, src, m, "even") < 1e-20


@pytest.mark.parametrize("refine,storage", [("sequential", None), ("sequential", "single"),
                                            ("sequential", "half"), ("batched", None)])
def test_multishift_mixed_refinement_paths(gpu, monkeypatch, refine, storage):
    """After the sloppy recurrence every shift is refined to its own
    tolerance: by default one mixed CG per shift on the 16-bit links
    (continuing on FP32 links if it stagnates), with
    QPHIX_B200_MS_REFINE_STORAGE=single on the FP32 links, =half with 16-bit
    vectors too, and with QPHIX_B200_MS_REFINE=batched all shifts in one
    batched solve (the batched solver's kernels, FP64 reliable updates per
    shift).  Every path meets every shift's tolerance on the oracle's true
    residual and agrees with the FP64 multi-shift."""
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="even")
    masses = _masses(0.01, 6)
    V = int(np.prod(dims))
    lib.set_inner_precision("double")
    _, x64, _, _ = _multi(lib, "D", links, src, masses, "even", max_iter=4000, nrestart=5, resid=1e-20)
    monkeypatch.setenv("QPHIX_B200_MS_REFINE", refine)
    if storage:
        monkeypatch.setenv("QPHIX_B200_MS_REFINE_STORAGE", storage)
    lib.set_inner_precision("single")
    try:
        it, xs, res, info = _multi(lib, "D", links, src, masses, "even", max_iter=4000, nrestart=5, resid=1e-20)
    finally:
        lib.set_inner_precision("double")
    for m, x, xd, r in zip(masses, xs, x64, res):
        assert r.final_rsq < 1e-20
        assert orc.true_residual(dims, links, x, src, m, "even") < 1e-20
        assert rel_err(x[: 3 * V], xd[: 3 * V]) < 1e-8


@pytest.mark.parametrize("inner", ["single", "half"])
def test_multishift_mixed_edge_cases(gpu, inner):
    """A single shift (the base is the only shift the deferred updates and
    the refinement see) meets the tolerance against the oracle; a zero
    source returns zero solutions with success, as the reference does
    (ks_multicg_offset.cpp:377-419)."""
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="even")
    lib.set_inner_precision(inner)
    try:
        it, xs, res, info = _multi(lib, "D", links, src, [0.03], "even", max_iter=4000, nrestart=5, resid=1e-20)
        assert info.status == 0
        assert res[0].final_rsq < 1e-20
        assert orc.true_residual(dims, links, xs[0], src, 0.03, "even") < 1e-20
        zero = np.zeros_like(src)
        it0, xs0, res0, info0 = _multi(lib, "D", links, zero, _masses(0.02, 4), "even", max_iter=4000, nrestart=5,
                                       resid=1e-20)
        assert info0.status == 0
        for x, r in zip(xs0, res0):
            assert not np.any(x) and r.final_rsq == 0.0
    finally:
        lib.set_inner_precision("double")


def _crossed(v, V):
    """The reference's multi-shift with EVENODD solves the even half with the
    odd-checkerboard operator and then the odd half with the even one
    (parity = parity0 & 1 = 1 first, ks_multicg_offset.cpp:294, then
    :533-537).  Moving each half to the other parity turns that into the
    ordinary system the oracle checks."""
    h = 3 * V
    return np.concatenate([v[h:], v[:h]])


@pytest.mark.parametrize("parity,inner", [("odd", "single"), ("evenodd", "single"), ("evenodd", "double")])
def test_multishift_mixed_both_parities(gpu, parity, inner):
    """The mixed multi-shift on the odd and on both parities: each parity's
    shifted solutions (accumulated in FP32 partial sums between reliable
    updates and added into FP64) reach the tolerance on the FP64 residual of
    the system the reference solves there (the FP64 path, which follows the
    reference statement for statement, checks that reading of EVENODD)."""
    dims = (8, 8, 8, 8)
    V = int(np.prod(dims))
    lib = gpu.use(dims)
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    masses = _masses(0.02, 6)
    lib.set_inner_precision(inner)
    try:
        it, xs, res, info = _multi(lib, "D", links, src, masses, parity, max_iter=4000, nrestart=5, resid=1e-20)
    finally:
        lib.set_inner_precision("double")
    for m, x in zip(masses, xs):
        if parity == "odd":
            assert orc.true_residual(dims, links, x, src, m, "odd") < 1e-20, m
        else:
            xc, bc = _crossed(x, V), _crossed(src, V)
            for p in ("even", "odd"):
                assert orc.true_residual(dims, links, xc, bc, m, p) < 1e-20, (m, p)
