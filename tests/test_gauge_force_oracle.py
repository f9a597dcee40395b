"""CPU: the restated Symanzik one-loop gauge force (oracle/gauge_force_oracle.py).

The reference's gauge-force arithmetic lives in the unvendored
milc-qphix-codegen, so the oracle is pinned by identities of its own
definition rather than by reference outputs:
  * the force is the derivative of the action: for a random traceless
    anti-Hermitian X on every link, central differences of
    S(exp(h X) U) equal -1/3 sum Re tr(X F), for each loop type alone
    (which also pins the loop enumeration of the staples against the loop
    counting of the action);
  * the action is gauge invariant and the force gauge covariant
    (F_mu(x) -> g(x) F_mu(x) g(x)^dag);
  * on unit links every staple is the identity, so the force vanishes.
"""
import numpy as np
import pytest

import gauge_force_oracle as G

DIMS = (4, 4, 4, 4)
KINDS = ("plaquette", "rectangle", "parallelogram")


def _only(kind):
    return {k: (1.0 if k == kind else 0.0) for k in KINDS}


@pytest.mark.parametrize("kind", KINDS)
def test_force_is_the_derivative_of_the_action(kind):
    U = G.random_su3_lex(DIMS, 1, 0.6)
    X = G.random_algebra_lex(DIMS, 2)
    co = _only(kind)
    F = G.gauge_force(U, co)
    an = -np.sum(np.trace(X @ F, axis1=-2, axis2=-1).real) / 3.0
    h = 1e-4
    fd = (G.action(G.expm_ah(h * X) @ U, co) - G.action(G.expm_ah(-h * X) @ U, co)) / (2 * h)
    assert abs(fd - an) <= 1e-6 * abs(an)


def test_staple_counts():
    for mu in range(4):
        p = G.staple_paths(mu)
        assert [len(p[k]) for k in KINDS] == [6, 18, 24]
        for kind in KINDS:
            for path in p[kind]:
                off = [0, 0, 0, 0]
                off[mu] = 1
                for d, s in path:
                    off[d] += s
                assert off == [0, 0, 0, 0], (mu, kind, path)  # closes at x


def test_gauge_invariance_and_covariance():
    U = G.random_su3_lex(DIMS, 3, 0.5)
    g = G.random_su3_lex(DIMS, 4, 1.0)[..., 0, :, :]  # one SU(3) matrix per site
    Ug = np.empty_like(U)
    for mu in range(4):
        off = [0, 0, 0, 0]
        off[mu] = 1
        gn = np.roll(g, shift=tuple(-o for o in (off[3], off[2], off[1], off[0])), axis=(0, 1, 2, 3))
        Ug[..., mu, :, :] = g @ U[..., mu, :, :] @ np.conj(np.swapaxes(gn, -1, -2))
    co = {"plaquette": 1.0, "rectangle": -0.07, "parallelogram": -0.02}
    assert abs(G.action(Ug, co) - G.action(U, co)) <= 1e-11 * abs(G.action(U, co))
    F, Fg = G.gauge_force(U, co), G.gauge_force(Ug, co)
    want = g[..., None, :, :] @ F @ np.conj(np.swapaxes(g, -1, -2))[..., None, :, :]
    assert np.abs(Fg - want).max() <= 1e-12 * np.abs(F).max()


def test_unit_links_give_no_force():
    U = np.broadcast_to(np.eye(3, dtype=np.complex128), (4, 4, 4, 4, 4, 3, 3)).copy()
    co = {"plaquette": 1.0, "rectangle": -0.07, "parallelogram": -0.02}
    assert np.abs(G.gauge_force(U, co)).max() == 0.0
