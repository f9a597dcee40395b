"""CPU: algebraic identities that pin the stencil semantics independently of
any implementation (the reference's per-site kernel is absent, so these are
what fix its meaning): anti-Hermiticity of D, Hermiticity and positivity of
4m^2 - D_eo D_oe, gauge covariance, and the free-field spectrum."""
import numpy as np
import pytest

from conftest import fields, orc, synthetic

import np_oracle as npo


def cx(v):
    return v[0::2] + 1j * v[1::2]


@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (8, 4, 8, 4)])
def test_dslash_anti_hermitian(dims):
    links = fields(dims, seed=5)
    x = synthetic.gaussian_source(dims, seed=1, parity="odd")
    y = synthetic.gaussian_source(dims, seed=2, parity="even")
    Dx = orc.asqtad_dslash(dims, links, x, "even")
    Dy = orc.asqtad_dslash(dims, links, y, "odd")
    lhs = np.vdot(cx(y), cx(Dx))
    rhs = -np.vdot(cx(Dy), cx(x))
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)


def test_mdagm_hermitian_positive():
    dims = (8, 4, 4, 8)
    links = fields(dims, seed=5)
    m = 0.05
    V = int(np.prod(dims))

    def M(v):
        t = orc.asqtad_dslash(dims, links, v, "odd")
        t = orc.asqtad_dslash(dims, links, t, "even")
        out = 4 * m * m * v - t
        out[V * 3:] = 0
        return out

    x = synthetic.gaussian_source(dims, seed=1, parity="even")
    y = synthetic.gaussian_source(dims, seed=2, parity="even")
    a = np.vdot(cx(y), cx(M(x)))
    b = np.conj(np.vdot(cx(x), cx(M(y))))
    assert abs(a - b) < 1e-12 * abs(a)
    q = np.vdot(cx(x), cx(M(x)))
    assert abs(q.imag) < 1e-12 * abs(q) and q.real > 4 * m * m * np.vdot(cx(x), cx(x)).real


def test_gauge_covariance():
    """D[U^g] (g psi) = g (D[U] psi) for a random SU(3) transformation g."""
    dims = (8, 4, 4, 8)
    lat = npo.Lat(dims)
    raw = fields(dims, seed=5)
    links = npo.Links(lat, raw)
    g = npo.random_gauge_transform(lat, np.random.Generator(np.random.PCG64(9)))
    raw_g = npo.links_to_raw(npo.gauge_transform_links(links, g))
    psi_raw = synthetic.gaussian_source(dims, seed=3, parity="evenodd")
    psi = npo.vec_from_raw(lat, psi_raw)
    gpsi = npo.vec_to_raw(lat, np.einsum("...ij,...j->...i", g, psi))
    lhs = orc.asqtad_dslash(dims, raw_g, gpsi, "even") + orc.asqtad_dslash(dims, raw_g, gpsi, "odd")
    d = orc.asqtad_dslash(dims, raw, psi_raw, "even") + orc.asqtad_dslash(dims, raw, psi_raw, "odd")
    rhs = npo.vec_to_raw(lat, np.einsum("...ij,...j->...i", g, npo.vec_from_raw(lat, d)))
    assert np.abs(lhs - rhs).max() < 1e-12 * np.abs(rhs).max()


@pytest.mark.parametrize("n", [(1, 0, 0, 0), (1, 2, 0, 1), (3, 1, 2, 3)])
def test_free_field_plane_wave_spectrum(n):
    """Unit links with staggered phases: D_eo D_oe on an even-site plane wave
    e^{ipx} multiplies it by -4 sum_mu (sin p_mu + c3 sin 3p_mu)^2, c3 = -1/24."""
    dims = (8, 8, 8, 8)
    links = synthetic.unit_links(dims)
    lat = synthetic.Lattice(dims)
    x, y, z, t = lat.raw_coords()
    p = [2 * np.pi * n[i] / dims[i] for i in range(4)]
    phase = np.exp(1j * (p[0] * x + p[1] * y + p[2] * z + p[3] * t))
    colour = np.array([1.0, 0.5 - 0.2j, -0.3j])
    w = phase[:, None] * colour[None, :]
    w[lat.Vh:] = 0  # even sites only
    raw = np.stack([w.real, w.imag], axis=-1).reshape(-1)
    t1 = orc.asqtad_dslash(dims, links, raw, "odd")
    t2 = orc.asqtad_dslash(dims, links, t1, "even")
    c3 = synthetic.NAIK
    lam = -4 * sum((np.sin(q) + c3 * np.sin(3 * q)) ** 2 for q in p)
    assert np.abs(t2 - lam * raw).max() < 1e-12 * max(1.0, abs(lam))


def test_cg_solution_satisfies_system_numpy():
    """The C oracle's CG solution solves the system as applied by the
    independent numpy stencil."""
    dims = (8, 4, 4, 8)
    links = fields(dims, seed=5)
    src = synthetic.gaussian_source(dims, seed=4, parity="even")
    _, x, _ = orc.invert(dims, links, src, 0.05, "even", "D", 1000, 5, 1e-24)
    lat = npo.Lat(dims)
    lk = npo.Links(lat, links)
    Mx = npo.mdagm(lk, npo.vec_from_raw(lat, x), 0.05, 0)
    b = npo.vec_from_raw(lat, src)
    assert np.linalg.norm(Mx - b) < 1e-11 * np.linalg.norm(b)
