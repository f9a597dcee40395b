"""CPU: the FP64 host fermion force (oracle/force_oracle.py) against central
finite differences of S = phi^dag (4m^2 - D D)^{-1} phi, with the backward
links rebuilt from the perturbed forward links, on both solve parities; and
the same force from the reference's own CG and Dslash (oracle/_ref)."""
import numpy as np
import pytest

from conftest import capi, synthetic

import force_oracle
import np_oracle as O

DIMS = (4, 4, 4, 8)
MASS = 0.2


def _random_su3_algebra(rng, shape):
    a = rng.standard_normal(shape + (3, 3)) + 1j * rng.standard_normal(shape + (3, 3))
    T = 0.5 * (a + np.conj(np.swapaxes(a, -1, -2)))
    tr = np.trace(T, axis1=-2, axis2=-1) / 3.0
    return T - tr[..., None, None] * np.eye(3)


def _action(lat, fat, lng, phi, parity):
    L = O.Links.__new__(O.Links)
    L.lat = lat
    L.fat, L.lng = fat, lng
    L.fatback = np.stack([np.roll(fat[..., mu, :, :], 1, axis=3 - mu) for mu in range(4)], axis=-3)
    L.lngback = np.stack([np.roll(lng[..., mu, :, :], 3, axis=3 - mu) for mu in range(4)], axis=-3)
    x, _ = O.cg(L, phi, MASS, parity, rel_tol=1e-14)
    return O.dot(phi, x).real, x, L


@pytest.mark.parametrize("parity", ["even", "odd"])
def test_host_force_matches_finite_differences(parity):
    P = 0 if parity == "even" else 1
    lat = O.Lat(DIMS)
    links = synthetic.asqtad_links(DIMS, seed=31)
    fat, lng = O.links_from_raw(lat, links["fat"]), O.links_from_raw(lat, links["lng"])
    rng = np.random.default_rng(3003)
    phi = rng.standard_normal(lat.shape + (3,)) + 1j * rng.standard_normal(lat.shape + (3,))
    phi = np.where((lat.parity == P)[..., None], phi, 0)
    S0, x, L = _action(lat, fat, lng, phi, P)
    y = O.dslash_eo(L, x, 1 - P)
    gf, gl = force_oracle.host_force(DIMS, O.vec_to_raw(lat, x), O.vec_to_raw(lat, y), parity)
    h = 1e-5
    for trial in range(4):
        Tf = _random_su3_algebra(rng, lat.shape + (4,))
        Tl = _random_su3_algebra(rng, lat.shape + (4,))
        dfat, dlng = 1j * Tf @ fat, 1j * Tl @ lng
        Sp = _action(lat, fat + h * dfat, lng + h * dlng, phi, P)[0]
        Sm = _action(lat, fat - h * dfat, lng - h * dlng, phi, P)[0]
        fd = (Sp - Sm) / (2 * h)
        draw_f = _links_raw(lat, dfat)
        draw_l = _links_raw(lat, dlng)
        an = float(np.dot(gf, draw_f) + np.dot(gl, draw_l))
        assert abs(fd - an) <= 1e-6 * abs(an), (trial, fd, an)


def _links_raw(lat, U):
    raw = np.empty((lat.V, 4, 3, 3, 2))
    flat = U.reshape(lat.V, 4, 3, 3)
    raw[lat.raw_of_lex, ..., 0] = flat.real
    raw[lat.raw_of_lex, ..., 1] = flat.imag
    return raw.reshape(-1)


def test_host_force_from_reference_solver(ref_lib):
    """x from the reference's CG and y from its Dslash give the force the
    numpy oracle's x and y give."""
    lat = O.Lat(DIMS)
    links = synthetic.asqtad_links(DIMS, seed=31)
    src = synthetic.gaussian_source(DIMS, seed=2002, parity="even")
    lib = ref_lib
    assert lib.init(DIMS) == 0
    try:
        L = lib.create_L("D", links)
        b = lib.create_V("D", src, "even")
        x = lib.create_V("D", np.zeros_like(src), "even")
        lib.invert("D", L, x, b, MASS, parity="even", max_iter=2000, nrestart=5, resid=1e-28)
        xr = lib.extract_V("D", x, "even")
        # the reference's asqtad_dslash accepts only EVENODD vectors: its
        # parity check uses QPHIX_OPP_PAR(p) = p ^ 11 (qphix_int.h:102)
        xf = lib.create_V("D", xr)
        y = lib.create_V("D", np.zeros_like(src))
        lib.dslash("D", L, y, xf, "odd")
        yr = lib.extract_V("D", y)
        for h in (b, x, xf, y):
            lib.destroy_V("D", h)
        lib.destroy_L("D", L)
    finally:
        lib.finalize()
    gf, gl = force_oracle.host_force(DIMS, xr, yr, "even")
    Ln = O.Links(lat, links)
    phi = O.vec_from_raw(lat, src)
    phi = np.where((lat.parity == 0)[..., None], phi, 0)
    xn, _ = O.cg(Ln, phi, MASS, 0, rel_tol=1e-14)
    yn = O.dslash_eo(Ln, xn, 1)
    gf2, gl2 = force_oracle.host_force(DIMS, O.vec_to_raw(lat, xn), O.vec_to_raw(lat, yn), "even")
    scale = max(np.abs(gf2).max(), np.abs(gl2).max())
    assert np.abs(gf - gf2).max() < 1e-9 * scale
    assert np.abs(gl - gl2).max() < 1e-9 * scale
