"""ORACLE / TEST INFRASTRUCTURE ONLY -- independent FP64 numpy restatement.

A second oracle that shares no code and no index arithmetic with the C
restatement (qphix_oracle.c) or with the reference host code: fields live on
plain 4-D arrays ``[t, z, y, x]`` and every shift is an ``np.roll``.  It
restates the asqtad/HISQ stencil that the reference's site loop
(ks_long_dslash.cpp:564-668) applies through its per-site kernel
(ks_dslash_complete_specialization.cpp:338-378, body absent):

    (D psi)(x) = sum_mu [ F_mu(x) psi(x+mu)   - B_mu(x)^dag psi(x-mu)  ]
               + sum_mu [ L_mu(x) psi(x+3mu)  - LB_mu(x)^dag psi(x-3mu) ]

with F, L, B, LB the caller's ``fat``, ``lng``, ``fatback``, ``lngback``
arrays (raw MILC layout, see ``synthetic.py``).  The even-odd operator of
``QPHIX_*_asqtad_dslash`` (qphix_f3.cpp:1233-1245) is D restricted to an
output parity with the input taken from the other parity.

Used to cross-check the C oracle and the reference host code, and for the
algebraic identities (anti-Hermiticity, gauge covariance, free-field
spectrum) that pin the stencil semantics.
"""
from __future__ import annotations

import numpy as np


class Lat:
    def __init__(self, dims):
        self.nx, self.ny, self.nz, self.nt = (int(d) for d in dims)
        self.nxh = self.nx // 2
        self.V = self.nx * self.ny * self.nz * self.nt
        self.Vh = self.V // 2
        t, z, y, x = np.meshgrid(np.arange(self.nt), np.arange(self.nz),
                                 np.arange(self.ny), np.arange(self.nx), indexing="ij")
        self.parity = (x + y + z + t) & 1
        par = self.parity
        self.raw_of_lex = ((((t * self.nz + z) * self.ny + y) * self.nxh + x // 2)
                           + par * self.Vh).reshape(-1)
        self.shape = (self.nt, self.nz, self.ny, self.nx)


def links_from_raw(lat, raw):
    a = np.asarray(raw, dtype=np.float64).reshape(lat.V, 4, 3, 3, 2)
    c = a[..., 0] + 1j * a[..., 1]
    return c[lat.raw_of_lex].reshape(lat.shape + (4, 3, 3))


def vec_from_raw(lat, raw):
    a = np.asarray(raw, dtype=np.float64).reshape(lat.V, 3, 2)
    c = a[..., 0] + 1j * a[..., 1]
    return c[lat.raw_of_lex].reshape(lat.shape + (3,))


def vec_to_raw(lat, v):
    out = np.empty((lat.V, 3, 2))
    flat = v.reshape(lat.V, 3)
    out[lat.raw_of_lex, :, 0] = flat.real
    out[lat.raw_of_lex, :, 1] = flat.imag
    return out.reshape(-1)


def _sh(a, mu, k):
    return np.roll(a, -k, axis=3 - mu)


def _mv(U, v):
    return np.einsum("...ij,...j->...i", U, v)


def _amv(U, v):
    return np.einsum("...ji,...j->...i", U.conj(), v)


class Links:
    def __init__(self, lat, raw):
        self.lat = lat
        self.fat = links_from_raw(lat, raw["fat"])
        self.lng = links_from_raw(lat, raw["lng"])
        self.fatback = links_from_raw(lat, raw["fatback"])
        self.lngback = links_from_raw(lat, raw["lngback"])


def dslash_full(links, psi):
    """D psi on the whole lattice (complex (T,Z,Y,X,3))."""
    out = np.zeros_like(psi)
    for mu in range(4):
        out += _mv(links.fat[..., mu, :, :], _sh(psi, mu, 1))
        out -= _amv(links.fatback[..., mu, :, :], _sh(psi, mu, -1))
        out += _mv(links.lng[..., mu, :, :], _sh(psi, mu, 3))
        out -= _amv(links.lngback[..., mu, :, :], _sh(psi, mu, -3))
    return out


def dslash_eo(links, psi, out_parity):
    """Output on ``out_parity`` (0 even, 1 odd) from the other parity of psi."""
    lat = links.lat
    src = np.where((lat.parity == 1 - out_parity)[..., None], psi, 0)
    out = dslash_full(links, src)
    return np.where((lat.parity == out_parity)[..., None], out, 0)


def mdagm(links, psi, mass, parity):
    """(4 m^2 - D_{p,1-p} D_{1-p,p}) psi on parity p (Hermitian, positive)."""
    t = dslash_eo(links, psi, 1 - parity)
    t = dslash_eo(links, t, parity)
    return 4.0 * mass * mass * psi - t


def dot(a, b):
    return complex(np.vdot(a.reshape(-1), b.reshape(-1)))


def cg(links, b, mass, parity, rel_tol=1e-12, maxiter=100000):
    """Textbook FP64 CG on parity ``parity``; returns (x, iterations)."""
    x = np.zeros_like(b)
    r = b.copy()
    p = r.copy()
    rr = dot(r, r).real
    bb = rr
    it = 0
    while rr > rel_tol ** 2 * bb and it < maxiter:
        Ap = mdagm(links, p, mass, parity)
        a = rr / dot(p, Ap).real
        x += a * p
        r -= a * Ap
        rr_new = dot(r, r).real
        p = r + (rr_new / rr) * p
        rr = rr_new
        it += 1
    return x, it


def random_gauge_transform(lat, rng):
    """Random SU(3) field g(x) (T,Z,Y,X,3,3) via QR of complex Gaussians."""
    a = rng.standard_normal(lat.shape + (3, 3)) + 1j * rng.standard_normal(lat.shape + (3, 3))
    q, r = np.linalg.qr(a)
    d = np.diagonal(r, axis1=-2, axis2=-1)
    q = q * (d / np.abs(d))[..., None, :]
    det = np.linalg.det(q)
    q[..., :, 0] /= det[..., None] ** 1.0  # det(q)=e^{i phi}; divide one column
    return q


def gauge_transform_links(links, g):
    """U_mu(x) -> g(x) U_mu(x) g(x+k mu)^dag for each stored link family."""
    lat = links.lat
    gd = np.conj(np.swapaxes(g, -1, -2))
    out = Links.__new__(Links)
    out.lat = lat
    out.fat = np.empty_like(links.fat)
    out.lng = np.empty_like(links.lng)
    out.fatback = np.empty_like(links.fatback)
    out.lngback = np.empty_like(links.lngback)
    for mu in range(4):
        out.fat[..., mu, :, :] = g @ links.fat[..., mu, :, :] @ _sh(gd, mu, 1)
        out.lng[..., mu, :, :] = g @ links.lng[..., mu, :, :] @ _sh(gd, mu, 3)
        # backward slot at x holds U_mu(x - k mu): transforms with g(x-k mu), g(x)^dag
        out.fatback[..., mu, :, :] = _sh(g, mu, -1) @ links.fatback[..., mu, :, :] @ gd
        out.lngback[..., mu, :, :] = _sh(g, mu, -3) @ links.lngback[..., mu, :, :] @ gd
    return out


def links_to_raw(links):
    lat = links.lat

    def conv(U):
        flat = U.reshape(lat.V, 4, 3, 3)
        out = np.empty((lat.V, 4, 3, 3, 2))
        out[lat.raw_of_lex, ..., 0] = flat.real
        out[lat.raw_of_lex, ..., 1] = flat.imag
        return out.reshape(-1)

    return {"fat": conv(links.fat), "lng": conv(links.lng),
            "fatback": conv(links.fatback), "lngback": conv(links.lngback)}
