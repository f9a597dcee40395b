"""CPU: pin the plain-C oracle against the reference's own host code.

The reference has no tests and no golden data.  Its layout remap, neighbour
tables, OpenMP site loop, CG (ks_d_congrad_fn.cpp) and multi-shift CG
(ks_multicg_offset.cpp) compile here (oracle/_ref); only the generated
per-site kernel is restated.  These tests check that the independent C
restatement (oracle/qphix_oracle.c) reproduces that code: the same Dslash,
the same iteration counts and solutions, the same EVENODD behaviour, the
same flop accounting, and bit-identical neighbour tables.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import fields, orc, rel_err, synthetic

import np_oracle as npo

DIMS = [(4, 4, 4, 4), (8, 4, 4, 8), (8, 8, 8, 8)]


@pytest.fixture(scope="module")
def ref(ref_lib):
    return ref_lib


def _ref_dslash(ref, dims, links, src, prec):
    ref.init(dims)
    L = ref.create_L(prec, links)
    vin = ref.create_V(prec, src)
    vout = ref.create_V(prec, np.zeros_like(src))
    ref.dslash(prec, L, vout, vin, "even")
    ref.dslash(prec, L, vout, vin, "odd")
    out = ref.extract_V(prec, vout)
    ref.destroy_V(prec, vin)
    ref.destroy_V(prec, vout)
    ref.destroy_L(prec, L)
    ref.finalize()
    return out


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("prec,tol", [("D", 1e-14), ("F", 2e-6)])
def test_dslash_oracle_matches_reference_host_code(ref, dims, prec, tol):
    links = fields(dims, seed=11)
    src = synthetic.gaussian_source(dims, seed=22, parity="evenodd")
    want = _ref_dslash(ref, dims, links, src, prec)
    got = orc.asqtad_dslash(dims, links, src, "even", prec) + orc.asqtad_dslash(dims, links, src, "odd", prec)
    assert rel_err(got, want) < tol


@pytest.mark.parametrize("dims", DIMS[:2])
def test_dslash_oracle_matches_numpy(dims):
    links = fields(dims, seed=11)
    src = synthetic.gaussian_source(dims, seed=22, parity="evenodd")
    lat = npo.Lat(dims)
    lk = npo.Links(lat, links)
    psi = npo.vec_from_raw(lat, src)
    want = npo.vec_to_raw(lat, npo.dslash_eo(lk, psi, 0) + npo.dslash_eo(lk, psi, 1))
    got = orc.asqtad_dslash(dims, links, src, "even") + orc.asqtad_dslash(dims, links, src, "odd")
    assert rel_err(got, want) < 1e-14


def test_ubench_fixture_checksums(ref):
    """The reference micro-benchmark's analytic fields (ubench_helper.h:256-364)
    through the reference host code and the oracle: equal weighted checksums
    (ubench_helper.h:451-487) of D applied to the analytic spinor."""
    dims = (8, 4, 4, 8)
    f = synthetic.ubench_fields(dims)
    links = {k: f[k] for k in ("fat", "lng", "fatback", "lngback")}
    want = _ref_dslash(ref, dims, links, f["spinor"], "D")
    got = orc.asqtad_dslash(dims, links, f["spinor"], "even") + orc.asqtad_dslash(dims, links, f["spinor"], "odd")
    for par in (0, 1):
        cw = synthetic.ubench_checksum(dims, want, par)
        cg = synthetic.ubench_checksum(dims, got, par)
        assert abs(cw - cg) <= 1e-12 * abs(cw)


def test_neighbour_table_restatement_bit_exact(ref):
    """NeighTable of init_ks_dslash_imp (qphix_misc.cpp:46-230), read out of the
    reference library after QPHIX_init, equals the restated table."""
    for dims in [(4, 4, 4, 4), (8, 4, 8, 4), (12, 8, 4, 4)]:
        ref.init(dims)
        nt_ptr = C.c_void_p.in_dll(ref.lib, "NeighTableF").value
        pxyz = C.c_int.in_dll(ref.lib, "Pxyzf").value
        vt = C.c_int.in_dll(ref.lib, "Vtf").value
        half = pxyz * vt
        arr = np.ctypeslib.as_array((C.c_uint * (2 * half * 16)).from_address(nt_ptr)).reshape(2, half, 16).copy()
        bt_ptr = C.c_void_p.in_dll(ref.lib, "BoundTableF").value
        bnd = np.ctypeslib.as_array((C.c_ubyte * (2 * half * 4)).from_address(bt_ptr)).reshape(2, half, 4).copy()
        ref.finalize()
        mine, mbnd = orc.neigh_table(dims)
        V = int(np.prod(dims))
        real = orc.padded_index(dims, np.arange(V // 2))
        assert np.array_equal(arr[:, real], mine[:, real])
        assert np.array_equal(bnd[:, real], mbnd[:, real])


@pytest.mark.parametrize("parity", ["even", "odd", "evenodd"])
def test_cg_fp64_same_iterations_and_solution(ref, parity):
    dims = (8, 8, 8, 8)
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    ref.init(dims)
    L = ref.create_L("D", links)
    b = ref.create_V("D", src, parity)
    x = ref.create_V("D", np.zeros_like(src), parity)
    it, info, res = ref.invert("D", L, x, b, 0.05, parity=parity, max_iter=1000, nrestart=5, resid=1e-20)
    xr = ref.extract_V("D", x, parity)
    for h in (b, x):
        ref.destroy_V("D", h)
    ref.destroy_L("D", L)
    ref.finalize()
    ito, xo, reso = orc.invert(dims, links, src, 0.05, parity, "D", 1000, 5, 1e-20)
    assert ito == it
    assert reso.final_iter == res.final_iter
    assert reso.final_restart == res.final_restart
    assert rel_err(xo, xr) < 1e-10
    assert reso.final_rsq < 1e-20 and res.final_rsq < 1e-20


def test_cg_relresid_path(ref):
    """relresid > 0 exercises relative_residue (ks_blas_utils_c.cpp:136-149)."""
    dims = (8, 8, 8, 8)
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    ref.init(dims)
    L = ref.create_L("D", links)
    b = ref.create_V("D", src, "even")
    x = ref.create_V("D", np.zeros_like(src), "even")
    it, info, res = ref.invert("D", L, x, b, 0.05, parity="even", max_iter=50, nrestart=8, resid=1e-16,
                               relresid=1e-6)
    xr = ref.extract_V("D", x, "even")
    ref.destroy_V("D", b)
    ref.destroy_V("D", x)
    ref.destroy_L("D", L)
    ref.finalize()
    ito, xo, reso = orc.invert(dims, links, src, 0.05, "even", "D", 50, 8, 1e-16, relresid=1e-6)
    assert (ito, reso.final_iter, reso.final_restart) == (it, res.final_iter, res.final_restart)
    # r is ~1e-9 of b at this point: its rounding (FMA contraction, sum order) is ~1e-7 of r
    assert abs(reso.final_rel - res.final_rel) <= 1e-6 * abs(res.final_rel)
    assert rel_err(xo, xr) < 1e-10


def test_cg_fp32_close(ref):
    dims = (8, 8, 8, 8)
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    ref.init(dims)
    L = ref.create_L("F", links)
    b = ref.create_V("F", src, "even")
    x = ref.create_V("F", np.zeros_like(src), "even")
    it, info, res = ref.invert("F", L, x, b, 0.05, parity="even", max_iter=1000, nrestart=5, resid=1e-12)
    xr = ref.extract_V("F", x, "even")
    ref.destroy_V("F", b)
    ref.destroy_V("F", x)
    ref.destroy_L("F", L)
    ref.finalize()
    ito, xo, reso = orc.invert(dims, links, src, 0.05, "even", "F", 1000, 5, 1e-12)
    # FP32 reductions are summed in a different order (OpenMP teams vs serial)
    assert abs(reso.final_iter - res.final_iter) <= 3
    assert rel_err(xo, xr) < 5e-6


@pytest.mark.parametrize("parity", ["even", "evenodd"])
def test_multishift_fp64_same_iterations_and_solutions(ref, parity):
    dims = (8, 8, 8, 8)
    links = fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    sig = np.logspace(-3, 0, 5)
    masses = np.sqrt(0.05 ** 2 + sig / 4)
    masses = np.concatenate([masses[2:], masses[:2]])  # lowest mass not first
    ref.init(dims)
    L = ref.create_L("D", links)
    b = ref.create_V("D", src, parity)
    outs = [ref.create_V("D", np.zeros_like(src), parity) for _ in masses]
    it, info, res = ref.invert_multi("D", L, outs, b, masses, parity=parity, max_iter=1000, nrestart=5, resid=1e-20)
    xr = [ref.extract_V("D", o, parity) for o in outs]
    for h in outs + [b]:
        ref.destroy_V("D", h)
    ref.destroy_L("D", L)
    ref.finalize()
    ito, xo, reso, info_o = orc.invert_multi(dims, links, src, masses, parity, "D", 1000, 5, 1e-20)
    assert ito == it
    assert [r.final_iter for r in reso] == [r.final_iter for r in res]
    assert info_o.final_flop == info.final_flop
    for a, b_ in zip(xo, xr):
        assert rel_err(a, b_) < 1e-10
