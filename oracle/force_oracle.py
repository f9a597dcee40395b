"""ORACLE / TEST INFRASTRUCTURE ONLY -- FP64 host fermion force.

Gradient of S = phi^dag (4m^2 - D_pq D_qp)^{-1} phi with respect to the raw
fat and Naik link arrays, from the solution x (parity p) and y = D_qp x
(parity q), both raw MILC colour vectors computed by the reference's own CG
and Dslash (ks_d_congrad_fn.cpp, ks_long_dslash.cpp through oracle/_ref) or
by the numpy oracle.  Restated from the derivative of the stencil
(np_oracle.dslash_full): a link U_mu(z) enters D forward at z and, through
the backward array the caller derives from it, adjoint at z + hop mu, so

    dS = 2 s(z) Re tr[dU W(z+hop mu) W(z)^dag],

W = x on p, y on q, s = +1 on p, -1 on q.  Returned per raw entry:
dS/dRe U_ab = 2 s Re M_ab, dS/dIm U_ab = -2 s Im M_ab, M_ab = conj(W_a(z))
W_b(z+hop mu).  Plain 4-D numpy arrays, np.roll shifts; no shared code with
the CUDA kernel.
"""
from __future__ import annotations

import numpy as np

import np_oracle as O


def host_force(dims, x_raw, y_raw, parity="even"):
    """(grad_fat, grad_lng) raw arrays (V*72 reals each)."""
    lat = O.Lat(dims)
    P = 0 if parity == "even" else 1
    W = O.vec_from_raw(lat, np.asarray(x_raw) * _parity_mask(lat, P)) + \
        O.vec_from_raw(lat, np.asarray(y_raw) * _parity_mask(lat, 1 - P))
    s = np.where(lat.parity == P, 2.0, -2.0)[..., None, None]
    out = []
    for hop in (1, 3):
        G = np.empty(lat.shape + (4, 3, 3), dtype=np.complex128)
        for mu in range(4):
            Wn = O._sh(W, mu, hop)
            M = np.einsum("...a,...b->...ab", W.conj(), Wn)
            G[..., mu, :, :] = s * (M.real - 1j * M.imag)
        out.append(_links_to_raw(lat, G))
    return out[0], out[1]


def _parity_mask(lat, P):
    m = np.zeros(lat.V * 6)
    m[P * lat.Vh * 6:(P + 1) * lat.Vh * 6] = 1.0
    return m


def _links_to_raw(lat, G):
    """complex (T,Z,Y,X,4,3,3) with re = dS/dRe, im = dS/dIm -> raw reals."""
    raw = np.empty((lat.V, 4, 3, 3, 2))
    flat = G.reshape(lat.V, 4, 3, 3)
    raw[lat.raw_of_lex, ..., 0] = flat.real
    raw[lat.raw_of_lex, ..., 1] = flat.imag
    return raw.reshape(-1)
