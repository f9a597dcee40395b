"""CPU: the identities the compressed Naik links rely on (csrc/recon.cu).

For a Naik link N = c U with c real and U unitary, the third row follows from
the first two: row2(N) = lambda conj(row0(N) x row1(N)) with lambda = det(U)/c.
For U in SU(3), lambda = 1/c is real (12-real storage: a sign and one
magnitude per field); for U in U(3) it is a complex number per link (13-real).
A matrix with a non-unitary part has no such lambda."""
import numpy as np


def _random_u3(rng, n, su3):
    z = rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))
    q, r = np.linalg.qr(z)
    q = q * (np.diagonal(r, axis1=1, axis2=2) / np.abs(np.diagonal(r, axis1=1, axis2=2)))[:, None, :]
    if su3:
        q = q / np.linalg.det(q)[:, None, None] ** (1.0 / 3.0)
    return q


def _ratio(n):
    """least-squares lambda and relative residual of row2 = lambda conj(row0 x row1)"""
    c = np.conj(np.cross(n[:, 0, :], n[:, 1, :]))
    lam = np.sum(np.conj(c) * n[:, 2, :], axis=1) / np.sum(np.abs(c) ** 2, axis=1)
    res = np.linalg.norm(n[:, 2, :] - lam[:, None] * c, axis=1) / np.linalg.norm(n[:, 2, :], axis=1)
    return lam, res


def test_su3_naik_links_have_one_real_ratio():
    rng = np.random.default_rng(1)
    coef = -1.0 / 24.0
    sign = rng.choice([-1.0, 1.0], size=64)
    n = coef * sign[:, None, None] * _random_u3(rng, 64, su3=True)
    lam, res = _ratio(n)
    assert np.max(res) < 1e-13
    assert np.max(np.abs(lam.imag)) < 1e-12 * np.max(np.abs(lam))
    assert np.allclose(np.abs(lam), 24.0, rtol=1e-12)
    assert np.array_equal(np.sign(lam.real), np.sign(coef * sign))


def test_u3_naik_links_have_a_complex_ratio_per_link():
    rng = np.random.default_rng(2)
    u = _random_u3(rng, 64, su3=False)
    scale = 0.04 * (1.0 + 0.1 * rng.random(64))
    n = scale[:, None, None] * u
    lam, res = _ratio(n)
    assert np.max(res) < 1e-13
    assert np.allclose(lam, np.linalg.det(u) / scale, rtol=1e-12)


def test_non_unitary_links_have_no_ratio():
    rng = np.random.default_rng(3)
    n = _random_u3(rng, 64, su3=True) / 24.0
    n = n + 1e-3 / 24.0 * (rng.standard_normal(n.shape) + 1j * rng.standard_normal(n.shape))
    _, res = _ratio(n)
    assert np.min(res) > 1e-6
