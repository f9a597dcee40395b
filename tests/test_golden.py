"""Golden fixtures produced by the reference itself (tests/golden/make_golden.py
runs the reference host code, oracle/_ref).  CPU tests pin the C oracle to
them; GPU tests pin the product library to them.  Neither needs the
reference sources at run time."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import ROOT, fields, orc, synthetic

GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "golden.json")))["cases"]


def weights(n, seed=77):
    return np.random.Generator(np.random.PCG64(seed)).standard_normal(n)


def wsum(v):
    v = np.asarray(v, dtype=np.float64)
    return float(np.dot(v, weights(v.size)))


def _close(a, b, rel):
    return abs(a - b) <= rel * max(abs(b), 1e-300)


def _dslash_cases():
    return [k for k in GOLD if k.startswith("dslash_")]


# ------------------------------------------------------------------ oracle --
@pytest.mark.parametrize("key", _dslash_cases())
def test_oracle_dslash_golden(key):
    g = GOLD[key]
    dims = tuple(g["dims"])
    links = fields(dims, seed=g["link_seed"])
    src = synthetic.gaussian_source(dims, seed=g["src_seed"], parity="evenodd")
    prec = key[-1]
    out = orc.asqtad_dslash(dims, links, src, "even", prec) + orc.asqtad_dslash(dims, links, src, "odd", prec)
    assert _close(wsum(out), g["wsum"], 1e-12 if prec == "D" else 1e-5)


def test_oracle_dslash_full_vector_golden():
    want = np.load(os.path.join(ROOT, "tests", "golden", "dslash_4x4x4x4.npz"))["out"]
    dims = (4, 4, 4, 4)
    links = fields(dims, seed=11)
    src = synthetic.gaussian_source(dims, seed=22, parity="evenodd")
    got = orc.asqtad_dslash(dims, links, src, "even") + orc.asqtad_dslash(dims, links, src, "odd")
    assert np.abs(got - want).max() <= 1e-14 * np.abs(want).max()


def test_oracle_ubench_golden():
    g = GOLD["ubench_8x4x4x8_D"]
    dims = tuple(g["dims"])
    f = synthetic.ubench_fields(dims)
    links = {k: f[k] for k in ("fat", "lng", "fatback", "lngback")}
    out = orc.asqtad_dslash(dims, links, f["spinor"], "even") + orc.asqtad_dslash(dims, links, f["spinor"], "odd")
    assert _close(synthetic.ubench_checksum(dims, out, 0), g["checksum_even"], 1e-12)
    assert _close(synthetic.ubench_checksum(dims, out, 1), g["checksum_odd"], 1e-12)


@pytest.mark.parametrize("parity", ["even", "odd", "evenodd"])
def test_oracle_cg_golden(parity):
    g = GOLD[f"cg_8x8x8x8_D_{parity}"]
    dims = tuple(g["dims"])
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    it, x, res = orc.invert(dims, links, src, g["mass"], parity, "D", g["max"], g["nrestart"], g["resid"])
    assert (it, res.final_iter, res.final_restart) == (g["return"], g["final_iter"], g["final_restart"])
    assert _close(wsum(x), g["wsum"], 1e-9)


def test_oracle_cg_relresid_golden():
    g = GOLD["cg_8x8x8x8_D_even_relresid"]
    dims = tuple(g["dims"])
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    it, x, res = orc.invert(dims, links, src, g["mass"], "even", "D", g["max"], g["nrestart"], g["resid"],
                            relresid=g["relresid"])
    assert (it, res.final_iter, res.final_restart) == (g["return"], g["final_iter"], g["final_restart"])
    assert _close(res.final_rel, g["final_rel"], 1e-6)


@pytest.mark.parametrize("parity", ["even", "evenodd"])
def test_oracle_multishift_golden(parity):
    g = GOLD[f"multishift_8x8x8x8_D_{parity}"]
    dims = tuple(g["dims"])
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    it, xs, res, info = orc.invert_multi(dims, links, src, g["masses"], parity, "D", g["max"], g["nrestart"],
                                         g["resid"])
    assert it == g["return"]
    assert [r.final_iter for r in res] == g["final_iter"]
    assert info.final_flop == g["final_flop"]
    for x, w in zip(xs, g["wsum"]):
        assert _close(wsum(x), w, 1e-9)


@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (8, 4, 8, 4), (12, 8, 4, 4)])
def test_oracle_neighbour_table_golden(dims):
    tab, _ = orc.neigh_table(dims)
    real = orc.padded_index(dims, np.arange(int(np.prod(dims)) // 2))
    sel = np.ascontiguousarray(tab[:, real]).astype(np.uint32)
    assert hashlib.sha256(sel.tobytes()).hexdigest() == GOLD["neigh_" + "x".join(map(str, dims))]["sha256"]


# ---------------------------------------------------------------- product --
@pytest.mark.gpu
@pytest.mark.parametrize("key", _dslash_cases())
def test_gpu_dslash_golden(gpu, key):
    g = GOLD[key]
    dims = tuple(g["dims"])
    prec = key[-1]
    lib = gpu.use(dims)
    links = fields(dims, seed=g["link_seed"])
    src = synthetic.gaussian_source(dims, seed=g["src_seed"], parity="evenodd")
    L = lib.create_L(prec, links)
    vin = lib.create_V(prec, src)
    vout = lib.create_V(prec, np.zeros_like(src))
    lib.dslash(prec, L, vout, vin, "even")
    lib.dslash(prec, L, vout, vin, "odd")
    out = lib.extract_V(prec, vout)
    for h in (vin, vout):
        lib.destroy_V(prec, h)
    lib.destroy_L(prec, L)
    assert _close(wsum(out), g["wsum"], 1e-12 if prec == "D" else 1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("parity", ["even", "odd", "evenodd"])
def test_gpu_cg_golden(gpu, parity):
    g = GOLD[f"cg_8x8x8x8_D_{parity}"]
    dims = tuple(g["dims"])
    lib = gpu.use(dims)
    lib.set_inner_precision("double")
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    L = lib.create_L("D", links)
    b = lib.create_V("D", src, parity)
    x = lib.create_V("D", np.zeros_like(src), parity)
    it, info, res = lib.invert("D", L, x, b, g["mass"], parity=parity, max_iter=g["max"], nrestart=g["nrestart"],
                               resid=g["resid"])
    xs = lib.extract_V("D", x, parity)
    for h in (b, x):
        lib.destroy_V("D", h)
    lib.destroy_L("D", L)
    assert (it, res.final_iter, res.final_restart) == (g["return"], g["final_iter"], g["final_restart"])
    assert info.final_flop == g["final_flop"]
    assert _close(wsum(xs), g["wsum"], 1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("parity", ["even", "evenodd"])
def test_gpu_multishift_golden(gpu, parity):
    g = GOLD[f"multishift_8x8x8x8_D_{parity}"]
    dims = tuple(g["dims"])
    lib = gpu.use(dims)
    lib.set_inner_precision("double")
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    L = lib.create_L("D", links)
    b = lib.create_V("D", src, parity)
    outs = [lib.create_V("D", np.zeros_like(src), parity) for _ in g["masses"]]
    it, info, res = lib.invert_multi("D", L, outs, b, g["masses"], parity=parity, max_iter=g["max"],
                                     nrestart=g["nrestart"], resid=g["resid"])
    xs = [lib.extract_V("D", o, parity) for o in outs]
    for h in outs + [b]:
        lib.destroy_V("D", h)
    lib.destroy_L("D", L)
    assert it == g["return"]
    assert [r.final_iter for r in res] == g["final_iter"]
    assert info.final_flop == g["final_flop"]
    for x, w in zip(xs, g["wsum"]):
        assert _close(wsum(x), w, 1e-9)
