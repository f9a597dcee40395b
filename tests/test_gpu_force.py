"""GPU: the fermion force QPHIX_B200_{D3,F3}_asqtad_force through the C ABI.

The force is the gradient of S = phi^dag (4m^2 - D_eo D_oe)^{-1} phi with
respect to the raw fat and Naik link arrays (backward links derived from the
forward ones).  Checked three ways:
  * against the FP64 host force (oracle/force_oracle.py) built from the same
    solution and the oracle's Dslash: 1e-12 relative (FP64), 1e-5 (FP32);
  * through a torch.autograd.Function (test harness only) whose backward
    calls the C ABI, against central finite differences (h = 1e-5) of S along
    random su(3) perturbations dU = i T U of all links: 1e-6 relative;
  * the multi-solution form equals the weighted sum of single calls.
"""
import numpy as np
import pytest
import torch

from conftest import fields, orc, synthetic

import force_oracle

pytestmark = pytest.mark.gpu

DIMS = (8, 8, 8, 8)
MASS = 0.05
RESID = 1e-24


def _solve(lib, links, src, prec="D", mass=MASS):
    L = lib.create_L(prec, links)
    b = lib.create_V(prec, src, "even")
    x = lib.create_V(prec, np.zeros_like(src), "even")
    lib.set_inner_precision("double")
    it, info, res = lib.invert(prec, L, x, b, mass, parity="even", max_iter=4000, nrestart=5,
                               resid=RESID if prec == "D" else 1e-12)
    assert info.status == 0, lib.last_error()
    lib.destroy_V(prec, b)
    return L, x


def _host(links, x_raw, parity="even"):
    other = "odd" if parity == "even" else "even"
    y = orc.asqtad_dslash(DIMS, links, x_raw, other, "D")
    return force_oracle.host_force(DIMS, x_raw, y, parity)


@pytest.mark.parametrize("prec,tol", [("D", 1e-12), ("F", 1e-5)])
def test_force_matches_host_force(gpu, prec, tol):
    lib = gpu.use(DIMS)
    links = fields(DIMS, seed=41)
    src = synthetic.gaussian_source(DIMS, seed=3003, parity="even")
    L, x = _solve(lib, links, src)
    x_raw = lib.extract_V("D", x, "even")
    lib.destroy_V("D", x)
    lib.destroy_L("D", L)
    hf, hl = _host(links, x_raw)
    Lp = lib.create_L(prec, links)
    xp = lib.create_V(prec, x_raw, "even")
    gf, gl = lib.force(prec, Lp, [xp], [1.0], "even")
    lib.destroy_V(prec, xp)
    lib.destroy_L(prec, Lp)
    scale = max(np.abs(hf).max(), np.abs(hl).max())
    assert np.abs(gf - hf).max() <= tol * scale
    assert np.abs(gl - hl).max() <= tol * scale


def test_force_odd_parity_matches_host_force(gpu):
    lib = gpu.use(DIMS)
    links = fields(DIMS, seed=41)
    x_raw = synthetic.gaussian_source(DIMS, seed=77, parity="odd")
    L = lib.create_L("D", links)
    x = lib.create_V("D", x_raw, "odd")
    gf, gl = lib.force("D", L, [x], [1.0], "odd")
    lib.destroy_V("D", x)
    lib.destroy_L("D", L)
    hf, hl = _host(links, x_raw, "odd")
    scale = max(np.abs(hf).max(), np.abs(hl).max())
    assert np.abs(gf - hf).max() <= 1e-12 * scale
    assert np.abs(gl - hl).max() <= 1e-12 * scale


def test_force_sums_solutions(gpu):
    """RHMC form: sum_k coef_k grad(x_k) in one call."""
    lib = gpu.use(DIMS)
    links = fields(DIMS, seed=41)
    L = lib.create_L("D", links)
    xs_raw = [synthetic.gaussian_source(DIMS, seed=90 + k, parity="even") for k in range(3)]
    xs = [lib.create_V("D", r, "even") for r in xs_raw]
    coef = [0.5, -1.25, 2.0]
    gf, gl = lib.force("D", L, xs, coef, "even")
    sf, sl = np.zeros_like(gf), np.zeros_like(gl)
    for c, x in zip(coef, xs):
        f1, l1 = lib.force("D", L, [x], [1.0], "even")
        sf += c * f1
        sl += c * l1
    for x in xs:
        lib.destroy_V("D", x)
    lib.destroy_L("D", L)
    assert np.abs(gf - sf).max() <= 1e-13 * np.abs(sf).max()
    assert np.abs(gl - sl).max() <= 1e-13 * np.abs(sl).max()


def test_force_rejects_bad_arguments(gpu):
    lib = gpu.use(DIMS)
    links = fields(DIMS, seed=41)
    L = lib.create_L("D", links)
    x = lib.create_V("D", synthetic.gaussian_source(DIMS, seed=1, parity="even"), "even")
    with pytest.raises(RuntimeError, match="parity must be EVEN or ODD"):
        lib.force("D", L, [x], [1.0], "evenodd")
    with pytest.raises(RuntimeError, match="lacks the parity"):
        lib.force("D", L, [x], [1.0], "odd")
    lib.destroy_V("D", x)
    lib.destroy_L("D", L)


class AsqtadAction(torch.autograd.Function):
    """S(fat, lng) = phi^dag (4m^2 - D_eo D_oe)^{-1} phi through the C ABI;
    backward returns the fermion force.  Backward links are rebuilt from the
    forward arrays, as MILC does."""

    @staticmethod
    def forward(ctx, fat, lng, lib, phi, mass):
        f, l = fat.detach().numpy(), lng.detach().numpy()
        links = {"fat": f, "lng": l, "fatback": synthetic.backlinks_raw(DIMS, f, 1),
                 "lngback": synthetic.backlinks_raw(DIMS, l, 3)}
        L, x = _solve(lib, links, phi, mass=mass)
        x_raw = lib.extract_V("D", x, "even")
        gf, gl = lib.force("D", L, [x], [1.0], "even")
        lib.destroy_V("D", x)
        lib.destroy_L("D", L)
        ctx.save_for_backward(torch.from_numpy(gf), torch.from_numpy(gl))
        V = int(np.prod(DIMS))
        return torch.tensor(float(np.dot(phi[: 3 * V], x_raw[: 3 * V])), dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        gf, gl = ctx.saved_tensors
        return g * gf, g * gl, None, None, None


def _su3_direction(rng, raw):
    """dU = i T U, T a random traceless Hermitian field, as raw reals."""
    U = synthetic.links_raw_to_lex(DIMS, raw)
    a = rng.standard_normal(U.shape) + 1j * rng.standard_normal(U.shape)
    T = 0.5 * (a + np.conj(np.swapaxes(a, -1, -2)))
    T = T - (np.trace(T, axis1=-2, axis2=-1) / 3.0)[..., None, None] * np.eye(3)
    return synthetic._to_raw_links(synthetic.Lattice(DIMS), 1j * T @ U)


def test_force_autograd_matches_finite_differences(gpu):
    lib = gpu.use(DIMS)
    links = fields(DIMS, seed=41)
    phi = synthetic.gaussian_source(DIMS, seed=3003, parity="even")
    fat = torch.tensor(links["fat"], requires_grad=True)
    lng = torch.tensor(links["lng"], requires_grad=True)
    S = AsqtadAction.apply(fat, lng, lib, phi, MASS)
    S.backward()
    rng = np.random.default_rng(3003)
    h = 1e-5
    worst = 0.0
    for _ in range(8):
        df, dl = _su3_direction(rng, links["fat"]), _su3_direction(rng, links["lng"])
        with torch.no_grad():
            Sp = AsqtadAction.apply(torch.tensor(links["fat"] + h * df), torch.tensor(links["lng"] + h * dl),
                                    lib, phi, MASS)
            Sm = AsqtadAction.apply(torch.tensor(links["fat"] - h * df), torch.tensor(links["lng"] - h * dl),
                                    lib, phi, MASS)
        fd = float(Sp - Sm) / (2 * h)
        an = float(fat.grad.numpy() @ df + lng.grad.numpy() @ dl)
        worst = max(worst, abs(fd - an) / abs(an))
    assert worst < 1e-6, worst
