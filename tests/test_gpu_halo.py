"""GPU: the domain-decomposed path on one GPU, in loopback.

QPHIX_B200_set_loopback_halo(1) sends every Dslash through the halo path of
a t-slab decomposition with the rank as its own t neighbour -- the send
buffers are the receive buffers, like the reference's ASSUME_MULTINODE
(ks_boundary.cpp:196-200, 250-256): the first and last three t-slices of
the input parity are packed into the ghost buffer, the interior sites
(3 <= t < Nt-3) run in one launch and the boundary sites, whose t
neighbours come from the ghost, in another; every reduction goes through
the split path (this GPU's totals, the sum over ranks, then a one-thread
finishing kernel).  Checked here:
  * the Dslash equals the oracle (1e-13 FP64, 1e-6 FP32) with and without
    the interior/boundary split (Nt = 8 and Nt = 4), and every inner-solve
    kernel gives bit-identical results through the halo and through the
    periodic wrap (the ghosts hold exact copies);
  * FP64 CG through the halo path takes the oracle's iteration count (to
    one iteration: only the order of one sum differs) and reaches the same
    solution; the relative-residue path uses the global volume;
  * mixed CG and mixed multi-shift reach the FP64 true residual.
"""
import numpy as np
import pytest

from conftest import fields, orc, rel_err, synthetic

pytestmark = pytest.mark.gpu


def _dslash(lib, dims, links, src, prec, parity):
    L = lib.create_L(prec, links)
    vi = lib.create_V(prec, src)
    vo = lib.create_V(prec, np.zeros_like(src))
    try:
        lib.dslash(prec, L, vo, vi, parity)
        assert lib.last_error() == "", lib.last_error()
        return lib.extract_V(prec, vo)
    finally:
        lib.destroy_V(prec, vi)
        lib.destroy_V(prec, vo)
        lib.destroy_L(prec, L)


@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (8, 8, 8, 4), (16, 8, 4, 12)])
@pytest.mark.parametrize("prec", ["D", "F"])
def test_loopback_dslash(gpu, dims, prec):
    lib = gpu.use(dims)
    links = fields(dims, seed=1001)
    src = synthetic.gaussian_source(dims, seed=41, parity="evenodd")
    V = int(np.prod(dims))
    assert lib.set_loopback_halo(True) == 0
    try:
        for parity in ("even", "odd"):
            got = _dslash(lib, dims, links, src, prec, parity)
            s = slice(0, 3 * V) if parity == "even" else slice(3 * V, 6 * V)
            want = orc.asqtad_dslash(dims, links, src, parity, "D")[s]
            assert rel_err(got[s], want) < (1e-13 if prec == "D" else 1e-6), (dims, prec, parity)
    finally:
        assert lib.set_loopback_halo(False) == 0


@pytest.mark.parametrize("storage", ["single", "single-r12", "single-r13", "half-links", "half"])
def test_loopback_inner_kernels_bit_identical(gpu, storage):
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims, seed=1001)
    src = synthetic.gaussian_source(dims, seed=42, parity="evenodd")

    def run():
        L = lib.create_L("D", links)
        vi = lib.create_V("D", src)
        vo = lib.create_V("D", np.zeros_like(src))
        try:
            outs = []
            for parity in ("even", "odd"):
                assert lib.dslash_inner(L, vo, vi, parity, storage) == 0, lib.last_error()
                outs.append(lib.extract_V("D", vo))
            return outs
        finally:
            lib.destroy_V("D", vi)
            lib.destroy_V("D", vo)
            lib.destroy_L("D", L)

    periodic = run()
    assert lib.set_loopback_halo(True) == 0
    try:
        halo = run()
    finally:
        lib.set_loopback_halo(False)
    for a, b in zip(periodic, halo):
        assert np.array_equal(a, b), storage


def _cg(lib, links, src, mass, inner="double", relresid=0.0, resid=1e-20):
    lib.set_inner_precision(inner)
    try:
        L = lib.create_L("D", links)
        b = lib.create_V("D", src, "even")
        x = lib.create_V("D", np.zeros_like(src), "even")
        it, info, res = lib.invert("D", L, x, b, mass, parity="even", max_iter=2000, nrestart=5, resid=resid,
                                   relresid=relresid)
        assert info.status == 0, lib.last_error()
        sol = lib.extract_V("D", x, "even")
        st = lib.last_stats()
        for h in (x, b):
            lib.destroy_V("D", h)
        lib.destroy_L("D", L)
        return res, sol, st
    finally:
        lib.set_inner_precision("double")


@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (8, 8, 8, 4)])
def test_loopback_fp64_cg(gpu, dims):
    lib = gpu.use(dims)
    links = fields(dims, seed=1001)
    src = synthetic.gaussian_source(dims, seed=2002, parity="even")
    V = int(np.prod(dims))
    ito, xo, reso = orc.invert(dims, links, src, 0.05, "even", "D", max_iter=2000, nrestart=5, resid=1e-20)
    assert lib.set_loopback_halo(True) == 0
    try:
        res, x, st = _cg(lib, links, src, 0.05)
    finally:
        lib.set_loopback_halo(False)
    assert abs(res.final_iter - reso.final_iter) <= 1, (res.final_iter, reso.final_iter)
    assert res.final_rsq < 1e-20
    assert rel_err(x[: 3 * V], xo[: 3 * V]) < 1e-10


def test_loopback_relresid(gpu):
    """relative_residue (ks_blas_utils_c.cpp:136-149) through the split
    reductions, with restarts: the oracle's stopping point and relative
    residue (the loopback path sums p.Ap in another order, so the last bits
    may differ)."""
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims, seed=1001)
    src = synthetic.gaussian_source(dims, seed=2002, parity="even")
    ito, xo, reso = orc.invert(dims, links, src, 0.05, "even", "D", 50, 8, 1e-16, relresid=1e-6)
    assert lib.set_loopback_halo(True) == 0
    lib.set_inner_precision("double")
    try:
        L = lib.create_L("D", links)
        b = lib.create_V("D", src, "even")
        x = lib.create_V("D", np.zeros_like(src), "even")
        it, info, res = lib.invert("D", L, x, b, 0.05, parity="even", max_iter=50, nrestart=8, resid=1e-16,
                                   relresid=1e-6)
        assert info.status == 0, lib.last_error()
        xs = lib.extract_V("D", x, "even")
        for h in (x, b):
            lib.destroy_V("D", h)
        lib.destroy_L("D", L)
    finally:
        lib.set_loopback_halo(False)
    assert abs(res.final_iter - reso.final_iter) <= 1 and res.final_restart == reso.final_restart
    if res.final_iter == reso.final_iter:
        assert abs(res.final_rel - reso.final_rel) <= 1e-6 * abs(reso.final_rel)
    assert rel_err(xs[: 3 * 4096], xo[: 3 * 4096]) < 1e-8


def test_loopback_mixed_cg_and_multishift(gpu):
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims, seed=1001)
    src = synthetic.gaussian_source(dims, seed=2002, parity="even")
    masses = np.sqrt(0.02 ** 2 + np.logspace(-3, 0, 4) / 4)
    assert lib.set_loopback_halo(True) == 0
    try:
        res, x, st = _cg(lib, links, src, 0.02, inner="single")
        assert orc.true_residual(dims, links, x, src, 0.02, "even") < 1.5e-20
        lib.set_inner_precision("single")
        L = lib.create_L("D", links)
        b = lib.create_V("D", src, "even")
        xs = [lib.create_V("D", np.zeros_like(src), "even") for _ in masses]
        it, info, rs = lib.invert_multi("D", L, xs, b, masses, parity="even", max_iter=2000, nrestart=5,
                                        resid=1e-20)
        assert info.status == 0, lib.last_error()
        for m, h in zip(masses, xs):
            assert orc.true_residual(dims, links, lib.extract_V("D", h, "even"), src, m, "even") < 1.5e-20
            lib.destroy_V("D", h)
        lib.destroy_V("D", b)
        lib.destroy_L("D", L)
    finally:
        lib.set_inner_precision("double")
        lib.set_loopback_halo(False)


def test_decomposition_needs_a_communicator(gpu):
    """machsize {1,1,1,2} without QPHIX_B200_comm_init is refused, and the
    communicator cannot be set up while the library is initialised."""
    lib = gpu.use((8, 8, 8, 8))
    uid = lib.comm_unique_id()
    assert len(uid) == 128
    assert lib.comm_init(uid, 2, 0) != 0 and "before QPHIX_init" in lib.last_error()
    lib.finalize()
    gpu.dims = None
    assert lib.init((8, 8, 8, 16), (1, 1, 1, 2), 0) != 0
    assert "communicator" in lib.last_error()
