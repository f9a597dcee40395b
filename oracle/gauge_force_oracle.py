"""ORACLE / TEST INFRASTRUCTURE ONLY -- FP64 host Symanzik one-loop gauge
action and gauge force.

QPHIX_*_symanzik_1loop_gauge_force (gauge_force_imp.cpp:136-199) hands the
gauge field, the momenta, coeffs->plaquette / rectangle / parallelogram and
eps to per-site bodies (gforce_imp_body, update_mg_body) that live in the
unvendored milc-qphix-codegen, so the arithmetic is restated here from the
one-loop Symanzik action as MILC defines it (imp_gauge_force: the momentum
of each link moves by eps times the traceless anti-Hermitian part of the
link times its staples, eps carrying beta/3):

    S(U) = -1/3 sum_x [ c_p sum(plaquettes) + c_r sum(1x2 rectangles)
                        + c_g sum(parallelograms) ] Re tr U_loop

over every geometric loop once: plaquettes [mu, nu, -mu, -nu], rectangles
[mu, mu, nu, -mu, -mu, -nu] and the six-link parallelograms
[a, b, c, -a, -b, -c] through three different axes.  The force on the
link U_mu(x) is

    F_mu(x) = TA( U_mu(x) sum_loops c_loop S_loop ),
    TA(M) = (M - M^dag)/2 - tr(M - M^dag)/6,

S_loop the product of the other links of a loop that contains U_mu(x),
taken from x + mu around back to x (6 plaquettes, 18 rectangles and 24
parallelograms per link; `staple_paths`).  For a traceless anti-Hermitian
direction X on every link, d/dh S(exp(h X) U) = -1/3 sum Re tr(X F): the
tests check this identity by central differences.  The momentum update of
the entry point is A_mu(x) <- A_mu(x) + eps F_mu(x) on the links of one
parity of sites.

Plain 4-D numpy arrays (T, Z, Y, X, 4, 3, 3) with np.roll shifts; no code
shared with the CUDA kernel.
"""
from __future__ import annotations

import itertools

import numpy as np

# step = (axis, sign); axes x, y, z, t = 0..3


def staple_paths(mu):
    """{type: [paths]} of the staples of a forward link mu: each path is the
    list of steps from x + mu back to x."""
    others = [d for d in range(4) if d != mu]
    plaq, rect, para = [], [], []
    for nu in others:
        for s in (1, -1):
            plaq.append([(nu, s), (mu, -1), (nu, -s)])
            rect.append([(mu, 1), (nu, s), (mu, -1), (mu, -1), (nu, -s)])
            rect.append([(nu, s), (mu, -1), (mu, -1), (nu, -s), (mu, 1)])
            rect.append([(nu, s), (nu, s), (mu, -1), (nu, -s), (nu, -s)])
    for nu, rho in itertools.permutations(others, 2):
        for s in (1, -1):
            for r in (1, -1):
                para.append([(nu, s), (rho, r), (mu, -1), (nu, -s), (rho, -r)])
    return {"plaquette": plaq, "rectangle": rect, "parallelogram": para}


def _link(U, d, off):
    """U_d(x + off) for every x: the field rolled by -off."""
    return np.roll(U[..., d, :, :], shift=tuple(-o for o in (off[3], off[2], off[1], off[0])), axis=(0, 1, 2, 3))


def _adj(M):
    return np.conj(np.swapaxes(M, -1, -2))


def path_product(U, path, start):
    """Product of the links along `path` from x + start, for every x."""
    off = list(start)
    M = None
    for d, s in path:
        if s > 0:
            L = _link(U, d, off)
            off[d] += 1
        else:
            off[d] -= 1
            L = _adj(_link(U, d, off))
        M = L if M is None else M @ L
    return M


def staple_sums(U, coeffs):
    """sum_loops c_loop S_loop for every link: (T,Z,Y,X,4,3,3)."""
    out = np.zeros_like(U)
    for mu in range(4):
        start = [0, 0, 0, 0]
        start[mu] = 1
        for kind, paths in staple_paths(mu).items():
            c = coeffs[kind]
            if c == 0.0:
                continue
            for p in paths:
                out[..., mu, :, :] += c * path_product(U, p, start)
    return out


def ta(M):
    A = 0.5 * (M - _adj(M))
    tr = np.trace(A, axis1=-2, axis2=-1)
    return A - (tr / 3.0)[..., None, None] * np.eye(3)


def gauge_force(U, coeffs):
    """F_mu(x) = TA(U_mu(x) sum c S) for every link, (T,Z,Y,X,4,3,3)."""
    return ta(U @ staple_sums(U, coeffs))


def loops_per_site():
    """Every closed path of each type starting at a site, with the number of
    times each geometric loop occurs among them."""
    plaq, rect, para = [], [], []
    signed = [(a, s) for a in range(4) for s in (1, -1)]
    for (a, sa), (b, sb) in itertools.product(signed, signed):
        if a == b:
            continue
        plaq.append([(a, sa), (b, sb), (a, -sa), (b, -sb)])
        rect.append([(a, sa), (a, sa), (b, sb), (a, -sa), (a, -sa), (b, -sb)])
    for (a, sa), (b, sb), (c, sc) in itertools.product(signed, signed, signed):
        if len({a, b, c}) < 3:
            continue
        para.append([(a, sa), (b, sb), (c, sc), (a, -sa), (b, -sb), (c, -sc)])
    # plaquette: 4 corners x 2 orientations; rectangle: 2 corners x 2
    # orientations start with the long side; parallelogram: 6 x 2
    return {"plaquette": (plaq, 8), "rectangle": (rect, 4), "parallelogram": (para, 12)}


def action(U, coeffs):
    """S(U) = -1/3 sum c Re tr U_loop over every geometric loop once."""
    S = 0.0
    for kind, (paths, mult) in loops_per_site().items():
        c = coeffs[kind]
        if c == 0.0:
            continue
        tot = 0.0
        for p in paths:
            tot += np.trace(path_product(U, p, [0, 0, 0, 0]), axis1=-2, axis2=-1).real.sum()
        S += -c * tot / (3.0 * mult)
    return float(S)


def momentum_update(U, A, coeffs, eps, parity_mask):
    """A + eps F on the links of the sites where parity_mask is true."""
    F = gauge_force(U, coeffs)
    return A + eps * F * parity_mask[..., None, None, None]


def random_su3_lex(dims, seed, eps=0.5):
    """Random SU(3) links exp(i eps H), (T,Z,Y,X,4,3,3)."""
    nx, ny, nz, nt = dims
    rng = np.random.default_rng(seed)
    shape = (nt, nz, ny, nx, 4)
    a = rng.standard_normal(shape + (3, 3)) + 1j * rng.standard_normal(shape + (3, 3))
    H = 0.5 * (a + _adj(a))
    H = H - (np.trace(H, axis1=-2, axis2=-1) / 3.0)[..., None, None] * np.eye(3)
    w, v = np.linalg.eigh(H)
    return (v * np.exp(1j * eps * w)[..., None, :]) @ _adj(v)


def random_algebra_lex(dims, seed):
    """Random traceless anti-Hermitian field, (T,Z,Y,X,4,3,3)."""
    nx, ny, nz, nt = dims
    rng = np.random.default_rng(seed)
    shape = (nt, nz, ny, nx, 4, 3, 3)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    return ta(a)


def expm_ah(X):
    """exp(X) of anti-Hermitian matrices."""
    w, v = np.linalg.eigh(-1j * X)
    return (v * np.exp(1j * w)[..., None, :]) @ _adj(v)


def parity_mask(dims, parity):
    """1 on the sites of `parity` ('even' / 'odd'), (T,Z,Y,X)."""
    nx, ny, nz, nt = dims
    t, z, y, x = np.meshgrid(np.arange(nt), np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    p = (x + y + z + t) & 1
    return (p == (0 if parity == "even" else 1)).astype(np.float64)
