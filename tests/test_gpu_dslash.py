"""GPU: the Dslash and the layout remap through the C ABI, against the oracle.

Tolerances (stated by the spec of this path): Dslash within 1e-13 relative
in FP64 and 1e-6 relative in FP32 (max-norm over the output, relative to
its max); layout round trips bit-exact.
"""
import numpy as np
import pytest

from conftest import fields, orc, rel_err, synthetic

pytestmark = pytest.mark.gpu

LATTICES = [(4, 4, 4, 4), (8, 4, 4, 8), (8, 8, 8, 8), (12, 8, 4, 4), (16, 8, 8, 4)]
TOL = {"D": 1e-13, "F": 1e-6}


def _dslash_both(lib, prec, L, src):
    vin = lib.create_V(prec, src)
    vout = lib.create_V(prec, np.zeros_like(src))
    assert vin and vout, lib.last_error()
    lib.dslash(prec, L, vout, vin, "even")
    lib.dslash(prec, L, vout, vin, "odd")
    out = lib.extract_V(prec, vout)
    lib.destroy_V(prec, vin)
    lib.destroy_V(prec, vout)
    return out


@pytest.mark.parametrize("dims", LATTICES)
@pytest.mark.parametrize("prec", ["D", "F"])
def test_dslash_matches_oracle(gpu, dims, prec):
    lib = gpu.use(dims)
    links = fields(dims, seed=11)
    src = synthetic.gaussian_source(dims, seed=22, parity="evenodd")
    L = lib.create_L(prec, links)
    assert L, lib.last_error()
    got = _dslash_both(lib, prec, L, src)
    lib.destroy_L(prec, L)
    want = orc.asqtad_dslash(dims, links, src, "even", "D") + orc.asqtad_dslash(dims, links, src, "odd", "D")
    assert rel_err(got, want) < TOL[prec]


@pytest.mark.parametrize("prec", ["D", "F"])
def test_dslash_ubench_fields_checksum(gpu, prec):
    """Analytic micro-benchmark fields of the reference (ubench_helper.h)."""
    dims = (8, 4, 4, 8)
    lib = gpu.use(dims)
    f = synthetic.ubench_fields(dims)
    links = {k: f[k] for k in ("fat", "lng", "fatback", "lngback")}
    L = lib.create_L(prec, links)
    got = _dslash_both(lib, prec, L, f["spinor"])
    lib.destroy_L(prec, L)
    want = orc.asqtad_dslash(dims, links, f["spinor"], "even") + orc.asqtad_dslash(dims, links, f["spinor"], "odd")
    assert rel_err(got, want) < TOL[prec]
    for par in (0, 1):
        cw = synthetic.ubench_checksum(dims, want, par)
        cg = synthetic.ubench_checksum(dims, got, par)
        assert abs(cw - cg) <= (1e-12 if prec == "D" else 1e-5) * abs(cw)


def test_dslash_single_parity_vectors(gpu):
    """out EVEN-only, in ODD-only handles (the API's parity bookkeeping)."""
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims, seed=11)
    src = synthetic.gaussian_source(dims, seed=22, parity="odd")
    L = lib.create_L("D", links)
    vin = lib.create_V("D", src, "odd")
    vout = lib.create_V("D", np.zeros_like(src), "even")
    lib.dslash("D", L, vout, vin, "even")
    got = lib.extract_V("D", vout, "even")
    want = orc.asqtad_dslash(dims, links, src, "even")
    V = int(np.prod(dims))
    assert rel_err(got[: V * 3], want[: V * 3]) < 1e-13
    # wrong parity combination is refused, not executed
    lib.dslash("D", L, vout, vin, "odd")
    assert "parities" in lib.last_error()
    for h in (vin, vout):
        lib.destroy_V("D", h)
    lib.destroy_L("D", L)


@pytest.mark.parametrize("prec", ["D", "F"])
def test_vector_round_trip_bit_exact(gpu, prec):
    dims = (8, 4, 8, 4)
    lib = gpu.use(dims)
    nt = np.float64 if prec == "D" else np.float32
    src = synthetic.gaussian_source(dims, seed=5, parity="evenodd").astype(nt)
    for eo in ("even", "odd", "evenodd"):
        h = lib.create_V(prec, src, eo)
        back = lib.extract_V(prec, h, eo)
        V = int(np.prod(dims))
        if eo in ("even", "evenodd"):
            assert np.array_equal(back[: V * 3], src[: V * 3])
        if eo in ("odd", "evenodd"):
            assert np.array_equal(back[V * 3:], src[V * 3:])
        lib.destroy_V(prec, h)


@pytest.mark.parametrize("prec", ["D", "F"])
def test_link_round_trip_bit_exact(gpu, prec):
    dims = (8, 4, 8, 4)
    lib = gpu.use(dims)
    nt = np.float64 if prec == "D" else np.float32
    links = {k: v.astype(nt) for k, v in fields(dims, seed=3).items()}
    L = lib.create_L(prec, links)
    fat, lng = lib.extract_L(prec, L)
    assert np.array_equal(fat, links["fat"])
    assert np.array_equal(lng, links["lng"])
    lib.destroy_L(prec, L)


def test_dslash_is_anti_hermitian_on_gpu(gpu):
    """<y, D_eo x> = -<D_oe y, x> with plain-adjoint backward links."""
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims, seed=7)
    x = synthetic.gaussian_source(dims, seed=1, parity="odd")
    y = synthetic.gaussian_source(dims, seed=2, parity="even")
    L = lib.create_L("D", links)
    hx, hy = lib.create_V("D", x), lib.create_V("D", y)
    dx, dy = lib.create_V("D", np.zeros_like(x)), lib.create_V("D", np.zeros_like(x))
    lib.dslash("D", L, dx, hx, "even")
    lib.dslash("D", L, dy, hy, "odd")
    Dx, Dy = lib.extract_V("D", dx), lib.extract_V("D", dy)
    cx = lambda v: v[0::2] + 1j * v[1::2]
    lhs = np.vdot(cx(y), cx(Dx))
    rhs = -np.vdot(cx(Dy), cx(x))
    assert abs(lhs - rhs) < 1e-11 * abs(lhs)
    for h in (hx, hy, dx, dy):
        lib.destroy_V("D", h)
    lib.destroy_L("D", L)


def test_dslash_timed_runs(gpu):
    dims = (16, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims, seed=11)
    src = synthetic.gaussian_source(dims, seed=22, parity="evenodd")
    L = lib.create_L("F", links)
    vin = lib.create_V("F", src)
    vout = lib.create_V("F", np.zeros_like(src))
    ms = lib.dslash_timed("F", L, vout, vin, "even", 5)
    assert ms > 0
    got = lib.extract_V("F", vout)
    want = orc.asqtad_dslash(dims, links, src, "even")
    V = int(np.prod(dims))
    assert rel_err(got[: V * 3], want[: V * 3]) < 1e-6
    for h in (vin, vout):
        lib.destroy_V("F", h)
    lib.destroy_L("F", L)


def test_dslash_fp32_vectors_16bit_links(gpu):
    """The HALF_LINKS inner operator (FP32 vectors with 16-bit fixed-point
    links) drives a mixed solve to the FP64 tolerance, and the autotuner
    has timed that vector/link pair."""
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = fields(dims, seed=11)
    src = synthetic.gaussian_source(dims, seed=22, parity="evenodd")
    L = lib.create_L("D", links)
    b = lib.create_V("D", src, "even")
    x = lib.create_V("D", np.zeros_like(src), "even")
    lib.set_inner_precision("half-links")
    try:
        it, info, res = lib.invert("D", L, x, b, 0.05, parity="even", max_iter=2000, nrestart=5, resid=1e-20)
        st = lib.last_stats()
    finally:
        lib.set_inner_precision("double")
    assert info.status == 0 and res.final_rsq < 1e-20
    v, us = lib.dslash_variant("half-links")
    assert v in (0, 1, 2) and min(us) > 0
    for h in (b, x):
        lib.destroy_V("D", h)
    lib.destroy_L("D", L)


@pytest.mark.parametrize("pinned", [False, True])
def test_large_round_trips_bit_exact(gpu, pinned):
    """Round trips large enough for the pinned-staging copies (16 MB and up,
    split across host threads): 24^3x48 colour vectors (32 MB) and 16^3x32
    links (75 MB per array), from pageable numpy arrays and from pinned ones
    (which are copied directly)."""
    import torch

    def host(a):
        if not pinned:
            return a
        t = torch.empty(a.shape, dtype=torch.float64).pin_memory()
        t.numpy()[...] = a
        return t.numpy()

    dims = (24, 24, 24, 48)
    lib = gpu.use(dims)
    src = host(np.random.default_rng(7).standard_normal(6 * int(np.prod(dims))))
    h = lib.create_V("D", src)
    back = lib.extract_V("D", h)
    lib.destroy_V("D", h)
    assert np.array_equal(back, src)

    dims = (16, 16, 16, 32)
    lib = gpu.use(dims)
    dev = "cuda" if torch.cuda.is_available() else None
    links = {k: host(v) for k, v in synthetic.asqtad_links(dims, seed=3, device=dev).items()}
    L = lib.create_L("D", links)
    fat, lng = lib.extract_L("D", L)
    lib.destroy_L("D", L)
    assert np.array_equal(fat, links["fat"]) and np.array_equal(lng, links["lng"])
