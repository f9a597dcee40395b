"""GPU: element-wise parity of every Dslash the mixed-precision solves run.

The timed solves apply the Dslash with FP32 links (18-real, or Naik links
stored as 12 or 13 reals with the third row rebuilt in the kernel) and
with 16-bit fixed-point links and vectors.  A mixed solve converges even
when its inner operator is off by 1e-4 (reliable updates hide it), so each
inner kernel is compared here, element by element, with the oracle's FP64
Dslash (qphix_ks_dslash, ks_long_dslash.cpp:564-668, restated in
oracle/qphix_oracle.c), through QPHIX_B200_D3_asqtad_dslash_inner /
_mdagm_inner on FP64 handles.

Tolerances (relative max-norm, max |got - want| / max |want|):
  * FP32 forms, compressed ones included: 1e-6, the FP32 Dslash tolerance;
  * 16-bit forms against the FP64 oracle: 6e-5 and the worst-case storage
    bound of fixedpoint.storage_bound (the measured storage error is
    2-3e-5; see fixedpoint.py);
  * 16-bit forms against the oracle applied to the emulated 16-bit inputs:
    2e-6 (FP32 arithmetic only), plus half an output quantum per component
    when the output is stored in 16 bits too.
"""
import numpy as np
import pytest
import torch

from conftest import fields, orc, rel_err, synthetic
from fixedpoint import naik_phased, quantize_links, quantize_vec, storage_bound

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-6
HALF_TOL = 6e-5
EMU_TOL = 2e-6
STORAGES = ("single", "single-r12", "single-r13", "half-links", "half")

_cache = {}


def _field(dims, kind):
    key = (dims, kind)
    if key not in _cache:
        if max(dims) > 16:
            dev = "cuda" if torch.cuda.is_available() else None
            base = synthetic.asqtad_links(dims, seed=1001, device=dev)
        elif kind == "hisq":
            base = fields(dims, seed=33, smear=True, eps_fat=0.2)
        else:
            base = fields(dims, seed=1001)
        _cache[key] = naik_phased(dims, base) if kind == "phased" else base
    return _cache[key]


def _half(dims, parity):
    V = int(np.prod(dims))
    return slice(0, 3 * V) if parity == "even" else slice(3 * V, 6 * V)


def _run_inner(lib, dims, links, src, parity, storage):
    L = lib.create_L("D", links)
    vin = lib.create_V("D", src)
    vout = lib.create_V("D", np.zeros_like(src))
    try:
        rc = lib.dslash_inner(L, vout, vin, parity, storage)
        got = lib.extract_V("D", vout) if rc == 0 else lib.last_error()
        return rc, got
    finally:
        lib.destroy_V("D", vin)
        lib.destroy_V("D", vout)
        lib.destroy_L("D", L)


def _check(dims, links, src, parity, storage, got):
    s = _half(dims, parity)
    want = orc.asqtad_dslash(dims, links, src, parity, "D")[s]
    err = rel_err(got[s], want)
    if storage.startswith("single"):
        assert err < FP32_TOL, (storage, parity, err)
        return err
    assert err < HALF_TOL and err < storage_bound(links, src, want), (storage, parity, err)
    # the kernel's own arithmetic, with the storage rounding emulated
    ql, _, _ = quantize_links(links)
    qin = quantize_vec(src)[0] if storage == "half" else src
    emu = orc.asqtad_dslash(dims, ql, qin, parity, "D")[s]
    diff = np.abs(got[s] - emu)
    slack = EMU_TOL * np.abs(emu).max()
    if storage == "half":
        # the output is stored in 16 bits: half a quantum of its site's norm
        m = np.abs(emu).reshape(-1, 6).max(axis=1)
        slack = slack + (0.5 / 32767.0) * np.repeat(m, 6) * (1 + 1e-5)
    assert np.all(diff <= slack), (storage, parity, float((diff - slack).max()))
    return err


@pytest.mark.parametrize("kind", ["asqtad", "hisq", "phased"])
@pytest.mark.parametrize("storage", STORAGES)
def test_inner_dslash_8x8x8x8(gpu, kind, storage):
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    links = _field(dims, kind)
    src = synthetic.gaussian_source(dims, seed=77, parity="evenodd")
    for parity in ("even", "odd"):
        rc, got = _run_inner(lib, dims, links, src, parity, storage)
        if storage == "single-r12" and kind == "phased":
            # U(3) Naik links have no single real ratio: the 12-real form is refused
            assert rc != 0 and "12-real" in got, got
            continue
        assert rc == 0, lib.last_error()
        _check(dims, links, src, parity, storage, got)


@pytest.mark.parametrize("storage", STORAGES)
def test_inner_dslash_24x24x24x48(gpu, storage):
    """The headline lattice and link recipe (the timed solve runs
    single-r12)."""
    dims = (24, 24, 24, 48)
    lib = gpu.use(dims)
    links = _field(dims, "asqtad")
    src = synthetic.gaussian_source(dims, seed=78, parity="evenodd")
    rc, got = _run_inner(lib, dims, links, src, "even", storage)
    assert rc == 0, lib.last_error()
    _check(dims, links, src, "even", storage, got)


def test_inner_dslash_13_real_24x24x24x48(gpu):
    """13-real Naik links at full size: U(1)-phased Naik links."""
    dims = (24, 24, 24, 48)
    lib = gpu.use(dims)
    links = naik_phased(dims, _field(dims, "asqtad"))
    src = synthetic.gaussian_source(dims, seed=79, parity="evenodd")
    rc, got = _run_inner(lib, dims, links, src, "odd", "single-r13")
    assert rc == 0, lib.last_error()
    _check(dims, links, src, "odd", "single-r13", got)
    rc, _ = _run_inner(lib, dims, links, src, "odd", "single-r12")
    assert rc != 0


@pytest.mark.parametrize("storage", STORAGES)
def test_inner_mdagm_8x8x8x8(gpu, storage):
    """The inner CG's two kernels (K1, then K2 with the M^dag M epilogue and
    the p.Mp reduction) against 4m^2 v - D D v and its dot product."""
    dims = (8, 8, 8, 8)
    mass = 0.03
    lib = gpu.use(dims)
    links = _field(dims, "hisq" if storage == "single-r13" else "asqtad")
    src = synthetic.gaussian_source(dims, seed=80, parity="evenodd")
    L = lib.create_L("D", links)
    vin = lib.create_V("D", src)
    vout = lib.create_V("D", np.zeros_like(src))
    try:
        for parity in ("even", "odd"):
            rc, dot = lib.mdagm_inner(L, vout, vin, mass, parity, storage)
            assert rc == 0, lib.last_error()
            got = lib.extract_V("D", vout)
            s = _half(dims, parity)
            other = "odd" if parity == "even" else "even"
            v = np.zeros_like(src)
            v[s] = src[s]
            t = orc.asqtad_dslash(dims, links, v, other, "D")
            dd = orc.asqtad_dslash(dims, links, t, parity, "D")[s]
            want = dd - 4 * mass * mass * src[s]  # the reference's ttt = D D p - 4 m^2 p
            tol = 2 * FP32_TOL if storage.startswith("single") else 2 * HALF_TOL
            assert rel_err(got[s], want) < tol, (storage, parity)
            wdot = float(src[s] @ want)
            assert abs(dot - wdot) < (1e-6 if storage.startswith("single") else 1e-4) * abs(wdot)
    finally:
        lib.destroy_V("D", vin)
        lib.destroy_V("D", vout)
        lib.destroy_L("D", L)


BATCH_LATS = [(8, 8, 8, 8), (12, 12, 12, 12), (16, 8, 8, 8)]


@pytest.mark.parametrize("prec,g", [("single", 4), ("single", 2), ("single", 1), ("double", 0)])
def test_batched_dslash(gpu, prec, g):
    """The batched solver's Dslash kernels (k_bdslash_s with 4, 2 or 1
    systems per thread, k_bdslash_d) on 3 lattices with segments of 8, 3
    and 2 systems (3 systems always run 3 per thread), every system against
    the oracle."""
    lib = gpu.use(BATCH_LATS[0])
    lat_links = [fields(d, seed=1001 + i) for i, d in enumerate(BATCH_LATS)]
    B = lib.batch_create_L(list(zip(BATCH_LATS, lat_links)))
    assert B, lib.last_error()
    try:
        counts = [8, 3, 2]
        systems = []
        for l, n in enumerate(counts):
            for r in range(n):
                systems.append((l, 0.02 + 0.01 * r,
                                synthetic.gaussian_source(BATCH_LATS[l], seed=500 + 10 * l + r, parity="evenodd")))
        tol = FP32_TOL if prec == "single" else 1e-13
        for parity in ("even", "odd"):
            rc, outs = lib.batch_dslash(B, systems, parity=parity, op=0, prec=prec, rhs_per_thread=g)
            assert rc == 0, lib.last_error()
            for (l, m, src), got in zip(systems, outs):
                dims = BATCH_LATS[l]
                s = _half(dims, parity)
                want = orc.asqtad_dslash(dims, lat_links[l], src, parity, "D")[s]
                assert rel_err(got[s], want) < tol, (prec, g, parity, l)
                other = _half(dims, "odd" if parity == "even" else "even")
                assert not np.any(got[other]), "the other parity must be left untouched"
            if prec == "single":
                rc, outs = lib.batch_dslash(B, systems, parity=parity, op=1, prec=prec, rhs_per_thread=g)
                assert rc == 0, lib.last_error()
                for (l, m, src), got in zip(systems, outs):
                    dims = BATCH_LATS[l]
                    s = _half(dims, parity)
                    other = "odd" if parity == "even" else "even"
                    v = np.zeros_like(src)
                    v[s] = src[s]
                    dd = orc.asqtad_dslash(dims, lat_links[l],
                                           orc.asqtad_dslash(dims, lat_links[l], v, other, "D"), parity, "D")[s]
                    want = 4 * m * m * src[s] - dd
                    assert rel_err(got[s], want) < 2 * FP32_TOL, (g, parity, l)
    finally:
        lib.batch_destroy_L(B)


def test_batched_dslash_refuses_bad_arguments(gpu):
    lib = gpu.use(BATCH_LATS[0])
    B = lib.batch_create_L([(BATCH_LATS[0], fields(BATCH_LATS[0], seed=1001))])
    try:
        src = synthetic.gaussian_source(BATCH_LATS[0], seed=1, parity="evenodd")
        assert lib.batch_dslash(B, [(0, 0.1, src)], op=1, prec="double")[0] != 0
        assert lib.batch_dslash(B, [(1, 0.1, src)])[0] != 0
        assert lib.batch_dslash(B, [(0, 0.1, src)], rhs_per_thread=3)[0] != 0
    finally:
        lib.batch_destroy_L(B)
