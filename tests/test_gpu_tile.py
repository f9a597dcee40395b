"""GPU: the TMA neighbour-tile Dslash (variant 3).

Each CTA stages the nine (z, t) input planes of an output plane in shared
memory with cp.async.bulk copies and gathers every neighbour from there.
Forced with QPHIX_B200_set_dslash_variant(3), it must give the oracle's
Dslash (1e-13 FP64, 1e-6 FP32) on cubic and non-cubic lattices, in the
inner-solve storages that use FP32 vectors (18-, 12-, 13-real links, 16-bit
links), and run whole solves (its fused M^dag M form, K2) to the oracle's
iteration count and solution.  Its bounded wait reports a failure when made
to run out, and the autotuner times it beside the other variants.
"""
import numpy as np
import pytest

from conftest import fields, orc, rel_err, synthetic

pytestmark = pytest.mark.gpu

LATTICES = [(8, 8, 8, 8), (16, 8, 4, 12), (8, 12, 8, 4)]


@pytest.fixture
def tile(gpu):
    lib = gpu.lib
    assert lib.set_dslash_variant(3) == 0
    yield
    lib.set_dslash_variant(-1)
    lib.set_wait_limit(-1)


@pytest.mark.parametrize("dims", LATTICES)
@pytest.mark.parametrize("prec", ["D", "F"])
def test_tile_dslash_matches_oracle(gpu, tile, dims, prec):
    lib = gpu.use(dims)
    V = int(np.prod(dims))
    links = fields(dims, seed=1001)
    src = synthetic.gaussian_source(dims, seed=51, parity="evenodd")
    L = lib.create_L(prec, links)
    vi = lib.create_V(prec, src)
    vo = lib.create_V(prec, np.zeros_like(src))
    try:
        for parity in ("even", "odd"):
            lib.dslash(prec, L, vo, vi, parity)
            assert lib.last_error() == "", lib.last_error()
            got = lib.extract_V(prec, vo)
            s = slice(0, 3 * V) if parity == "even" else slice(3 * V, 6 * V)
            want = orc.asqtad_dslash(dims, links, src, parity, "D")[s]
            assert rel_err(got[s], want) < (1e-13 if prec == "D" else 1e-6), (dims, prec, parity)
    finally:
        lib.destroy_V(prec, vi)
        lib.destroy_V(prec, vo)
        lib.destroy_L(prec, L)


@pytest.mark.parametrize("storage", ["single", "single-r12", "single-r13", "half-links"])
def test_tile_inner_storages(gpu, tile, storage):
    dims = (8, 8, 8, 8)
    V = int(np.prod(dims))
    lib = gpu.use(dims)
    links = fields(dims, seed=1001)
    src = synthetic.gaussian_source(dims, seed=52, parity="evenodd")
    L = lib.create_L("D", links)
    vi = lib.create_V("D", src)
    vo = lib.create_V("D", np.zeros_like(src))
    try:
        assert lib.dslash_inner(L, vo, vi, "odd", storage) == 0, lib.last_error()
        got = lib.extract_V("D", vo)[3 * V:]
    finally:
        lib.destroy_V("D", vi)
        lib.destroy_V("D", vo)
        lib.destroy_L("D", L)
    want = orc.asqtad_dslash(dims, links, src, "odd", "D")[3 * V:]
    assert rel_err(got, want) < (1e-6 if storage.startswith("single") else 6e-5), storage


@pytest.mark.parametrize("inner", ["double", "single"])
def test_tile_solves(gpu, tile, inner):
    dims = (8, 8, 8, 8)
    V = int(np.prod(dims))
    lib = gpu.use(dims)
    links = fields(dims, seed=1001)
    src = synthetic.gaussian_source(dims, seed=2002, parity="even")
    lib.set_inner_precision(inner)
    try:
        L = lib.create_L("D", links)
        b = lib.create_V("D", src, "even")
        x = lib.create_V("D", np.zeros_like(src), "even")
        it, info, res = lib.invert("D", L, x, b, 0.05, parity="even", max_iter=2000, nrestart=5, resid=1e-20)
        assert info.status == 0, lib.last_error()
        xs = lib.extract_V("D", x, "even")
        for h in (x, b):
            lib.destroy_V("D", h)
        lib.destroy_L("D", L)
    finally:
        lib.set_inner_precision("double")
    ito, xo, reso = orc.invert(dims, links, src, 0.05, "even", "D", max_iter=2000, nrestart=5, resid=1e-20)
    if inner == "double":
        assert res.final_iter == reso.final_iter
    assert orc.true_residual(dims, links, xs, src, 0.05, "even") < 1.5e-20
    assert rel_err(xs[: 3 * V], xo[: 3 * V]) < 1e-8


def test_tile_wait_timeout(gpu, tile):
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims, seed=1001)
    src = synthetic.gaussian_source(dims, seed=53, parity="evenodd")
    L = lib.create_L("D", links)
    vi = lib.create_V("D", src)
    vo = lib.create_V("D", np.zeros_like(src))
    try:
        assert lib.set_wait_limit(0) == 0
        lib.dslash("D", L, vo, vi, "even")
        assert "timed out" in lib.last_error()
        assert lib.set_wait_limit(-1) == 0
        lib.dslash("D", L, vo, vi, "even")
        assert lib.last_error() == ""
        V = int(np.prod(dims))
        got = lib.extract_V("D", vo)[: 3 * V]
        assert rel_err(got, orc.asqtad_dslash(dims, links, src, "even", "D")[: 3 * V]) < 1e-13
    finally:
        lib.destroy_V("D", vi)
        lib.destroy_V("D", vo)
        lib.destroy_L("D", L)


def test_autotuner_times_the_tile_variant(gpu):
    dims = (16, 16, 16, 16)
    lib = gpu.use(dims)
    lib.set_dslash_variant(-1)
    links = fields(dims, seed=1001)
    src = synthetic.gaussian_source(dims, seed=54, parity="evenodd")
    for prec, name in (("F", "single"), ("D", "double")):
        L = lib.create_L(prec, links)
        vi = lib.create_V(prec, src)
        vo = lib.create_V(prec, np.zeros_like(src))
        lib.dslash(prec, L, vo, vi, "even")
        v, us = lib.tuning(name)
        assert v in (0, 1, 2, 3) and all(u > 0 for u in us), (name, v, us)
        for h in (vi, vo):
            lib.destroy_V(prec, h)
        lib.destroy_L(prec, L)
