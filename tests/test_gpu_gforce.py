"""GPU: the Symanzik one-loop gauge force (QPHIX_{D3,F3}_symanzik_1loop_gauge_force)
and its gauge-field / momentum objects, through the C ABI, against the FP64
host oracle (oracle/gauge_force_oracle.py, itself checked against finite
differences of the action in tests/test_gauge_force_oracle.py).

  * create/extract of G and F round-trip the raw arrays bit for bit, and F
    keeps only the parities it was created with;
  * one call adds eps F_mu(x) to the momenta of the links of one
    checkerboard (the objects' parity; EVENODD works on EVEN, as in the
    reference) and leaves the other checkerboard and the gauge field alone:
    FP64 within 1e-12 and FP32 within 1e-5 of the oracle, relative to the
    largest momentum entry, on 8^4 and a non-cubic 4x8x4x12 lattice;
  * two calls with eps1 and eps2 equal one with eps1 + eps2; mismatched
    parities and NULL arguments return QPHIX_FAIL.
"""
import numpy as np
import pytest

from conftest import synthetic

import gauge_force_oracle as G

pytestmark = pytest.mark.gpu

COEFFS = {"plaquette": 1.0, "rectangle": -0.0545, "parallelogram": -0.0123}


def _fields(dims, seed=7):
    lat = synthetic.Lattice(dims)
    U = G.random_su3_lex(dims, seed, 0.5)
    A = G.random_algebra_lex(dims, seed + 1)
    return lat, U, A, synthetic._to_raw_links(lat, U), synthetic._to_raw_links(lat, A)


def _lex(dims, raw):
    return synthetic.links_raw_to_lex(dims, raw)


@pytest.mark.parametrize("prec", ["D", "F"])
def test_gauge_and_momentum_round_trips(gpu, prec):
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    lat, U, A, Uraw, Araw = _fields(dims)
    nt = np.float64 if prec == "D" else np.float32
    g = lib.create_G(prec, Uraw)
    assert g, lib.last_error()
    assert np.array_equal(lib.extract_G(prec, g), Uraw.astype(nt))
    lib.destroy_G(prec, g)
    half = lat.V * 36
    for eo in ("even", "odd", "evenodd"):
        f = lib.create_F(prec, Araw, eo)
        assert f, lib.last_error()
        out = lib.extract_F(prec, f, "evenodd")
        want = Araw.astype(nt).copy()
        if eo == "even":
            want[half:] = 0
        if eo == "odd":
            want[:half] = 0
        assert np.array_equal(out, want), eo
        lib.destroy_F(prec, f)


@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (4, 8, 4, 12)])
@pytest.mark.parametrize("prec,tol", [("D", 1e-12), ("F", 1e-5)])
@pytest.mark.parametrize("parity", ["even", "odd", "evenodd"])
def test_gauge_force_matches_oracle(gpu, dims, prec, tol, parity):
    lib = gpu.use(dims)
    lat, U, A, Uraw, Araw = _fields(dims)
    eps = 0.0375
    g = lib.create_G(prec, Uraw, parity)
    f = lib.create_F(prec, Araw, "evenodd")
    try:
        info = lib.gauge_force(prec, g, f, COEFFS, eps) if parity != "odd" else None
        if parity == "odd":
            # the objects' parities must agree (gauge_force_imp.cpp:142)
            info = lib.gauge_force(prec, g, f, COEFFS, eps)
            assert info.status != 0 and "parities differ" in lib.last_error()
            lib.destroy_F(prec, f)
            f = lib.create_F(prec, Araw, "odd")
            info = lib.gauge_force(prec, g, f, COEFFS, eps)
        assert info.status == 0, lib.last_error()
        assert info.final_flop > 0
        got = _lex(dims, lib.extract_F(prec, f, "evenodd"))
        Ug = lib.extract_G(prec, g)
    finally:
        lib.destroy_G(prec, g)
        lib.destroy_F(prec, f)
    P = "odd" if parity == "odd" else "even"
    mask = G.parity_mask(dims, P)
    want = G.momentum_update(U, A, COEFFS, eps, mask)
    if parity == "odd":
        # created with ODD only: the even momenta were never loaded
        want = want * mask[..., None, None, None]
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= tol * scale, float(np.abs(got - want).max() / scale)
    # the gauge field is not changed by the force
    assert np.array_equal(Ug, Uraw.astype(Ug.dtype))


def test_gauge_force_is_linear_in_eps(gpu):
    dims = (8, 8, 8, 8)
    lib = gpu.use(dims)
    lat, U, A, Uraw, Araw = _fields(dims, seed=11)
    g = lib.create_G("D", Uraw)
    f1 = lib.create_F("D", Araw)
    f2 = lib.create_F("D", Araw)
    try:
        for e in (0.01, 0.025):
            assert lib.gauge_force("D", g, f1, COEFFS, e).status == 0
        assert lib.gauge_force("D", g, f2, COEFFS, 0.035).status == 0
        a, b = lib.extract_F("D", f1), lib.extract_F("D", f2)
    finally:
        lib.destroy_G("D", g)
        lib.destroy_F("D", f1)
        lib.destroy_F("D", f2)
    assert np.abs(a - b).max() <= 1e-14 * np.abs(b).max()


def test_gauge_force_rejects_null_arguments(gpu):
    lib = gpu.use((8, 8, 8, 8))
    lat, U, A, Uraw, Araw = _fields((8, 8, 8, 8))
    g = lib.create_G("D", Uraw)
    try:
        assert lib.gauge_force("D", g, None, COEFFS, 0.1).status != 0
        assert lib.lib.QPHIX_D3_create_F_from_raw(None, 2) is None
        assert "NULL" in lib.last_error()
    finally:
        lib.destroy_G("D", g)
