"""GPU: the benchmark configurations at their stated sizes, checked against
the oracle (oracle/qphix_oracle.c: Dslash, true residuals, small CGs) rather
than against the library itself.

  * 24^3x48, the headline lattice: the FP64 (D3) and FP32 (F3) Dslash of the
    reference API element-wise against the oracle (1e-13, 1e-6).
  * Config 3, 32^3x64: HISQ-shaped links (smeared eps = 0.2 fat links, eps =
    0.3 Naik links), m = 0.0012, 12 RHMC shifts sigma log-spaced 1e-5 .. 1
    (masses sqrt(m^2 + sigma/4)).  Mixed multi-shift (FP32 inner with 12-real
    Naik links, FP64 solutions): every shift's true residual, recomputed by
    the oracle, below 1e-20 (squared, relative); solutions within 5e-8 of the
    FP64 multi-shift's (both at |r|/|b| < 1e-10: they differ by up to the
    condition number times that, 1.1e-8 for the lightest shifts); the sloppy
    recurrence's iteration count within 2 % of the FP64 recurrence's.
  * Config 4: 16 Gaussian right-hand sides on 24^3x48 plus two lattices each
    of 8^4, 12^4, 16^3x32 and 20^3x40, m = 0.02, in one batched solve: every
    system's oracle true residual below 1e-20 and its solution within 1e-8 of
    that system's FP64 CG (the library's reference-flow CG, which the small
    lattices also check against the oracle's CG).
  * Config 5: the fermion force on 16^3x32, m = 0.05, eps = 0.3 links, FP64
    and FP32.  The FP64 force against the host force built from the oracle's
    Dslash (1e-12 of its largest entry), the FP32 force within 1e-5 of it,
    and central finite differences (h = 1e-5) of S = phi^dag M^-1 phi along
    32 random su(3) directions dU = i T U of all fat and Naik links.  The
    criterion is |FD - grad S . dU| <= 1e-6 |grad S| |dU| for every
    direction: normalised by the norms, because a direction nearly
    orthogonal to the gradient has a tiny grad S . dU and its relative error
    measures only the finite-difference truncation.
"""
import numpy as np
import pytest
import torch

from conftest import orc, rel_err, synthetic

import force_oracle

pytestmark = pytest.mark.gpu

RESID = 1e-20
_DEV = "cuda" if torch.cuda.is_available() else None


def _links(dims, **kw):
    return synthetic.asqtad_links(dims, seed=1001, device=_DEV if max(dims) > 16 else None, **kw)


def _half(V, parity):
    return slice(0, 3 * V) if parity == "even" else slice(3 * V, 6 * V)


def test_headline_lattice_dslash_fp64_fp32(gpu):
    dims = (24, 24, 24, 48)
    V = int(np.prod(dims))
    lib = gpu.use(dims)
    links = _links(dims)
    src = synthetic.gaussian_source(dims, seed=61, parity="evenodd")
    for prec, tol in (("D", 1e-13), ("F", 1e-6)):
        L = lib.create_L(prec, links)
        vi = lib.create_V(prec, src)
        vo = lib.create_V(prec, np.zeros_like(src))
        for parity in ("even", "odd"):
            lib.dslash(prec, L, vo, vi, parity)
            got = lib.extract_V(prec, vo)
            s = _half(V, parity)
            want = orc.asqtad_dslash(dims, links, src, parity, "D")[s]
            assert rel_err(got[s], want) < tol, (prec, parity)
        for h in (vi, vo):
            lib.destroy_V(prec, h)
        lib.destroy_L(prec, L)


def test_config3_mixed_multishift_32x32x32x64(gpu):
    dims = (32, 32, 32, 64)
    V = int(np.prod(dims))
    mass = 0.0012
    masses = np.sqrt(mass ** 2 + np.logspace(-5, 0, 12) / 4)
    lib = gpu.use(dims)
    links = _links(dims, eps_fat=0.2, eps_long=0.3, smear=True)
    src = synthetic.gaussian_source(dims, seed=2002, parity="even")
    L = lib.create_L("D", links)
    b = lib.create_V("D", src, "even")

    def multi(inner):
        lib.set_inner_precision(inner)
        xs = [lib.create_V("D", np.zeros_like(src), "even") for _ in masses]
        it, info, res = lib.invert_multi("D", L, xs, b, masses, parity="even", max_iter=20000, nrestart=5,
                                         resid=RESID)
        assert info.status == 0, lib.last_error()
        st = lib.last_stats()
        sols = [lib.extract_V("D", x, "even") for x in xs]
        for x in xs:
            lib.destroy_V("D", x)
        return it, st, res, sols

    lib.set_reliable_delta(0.2)
    lib.set_link_compression(True)
    try:
        it64, st64, res64, x64 = multi("double")
        itm, stm, resm, xm = multi("single")
        assert stm.links_compressed == 1
    finally:
        lib.set_inner_precision("double")
        lib.set_link_compression(False)
        lib.destroy_V("D", b)
        lib.destroy_L("D", L)
    e = slice(0, 3 * V)
    for k, m in enumerate(masses):
        assert orc.true_residual(dims, links, xm[k], src, m, "even") < 1.5 * RESID, k
        # two solutions with |r|/|b| < 1e-10 differ by up to the condition
        # number times that; the light shifts here differ by ~1e-8
        assert rel_err(xm[k][e], x64[k][e]) < 5e-8, k
    # both calls return the iterations of the shifted recurrence (the mixed
    # one before its per-shift refinements)
    assert abs(itm - it64) <= 0.02 * it64, (itm, it64)


BATCH_BIG = (24, 24, 24, 48)
BATCH_SMALL = [(8, 8, 8, 8), (12, 12, 12, 12), (16, 16, 16, 32), (20, 20, 20, 40)]


def test_config4_batch_16rhs_and_8_lattices(gpu):
    mass = 0.02
    lats = [BATCH_BIG] + [d for d in BATCH_SMALL for _ in range(2)]
    lib = gpu.use(BATCH_BIG)
    links = [synthetic.asqtad_links(d, seed=1001 + i, device=_DEV) for i, d in enumerate(lats)]
    systems = [(0, mass, synthetic.gaussian_source(BATCH_BIG, seed=2002 + r, parity="even")) for r in range(16)]
    systems += [(l, mass, synthetic.gaussian_source(lats[l], seed=2102 + l, parity="even"))
                for l in range(1, len(lats))]
    B = lib.batch_create_L(list(zip(lats, links)))
    assert B, lib.last_error()
    try:
        it, info, res, xs = lib.batch_invert(B, systems, max_iter=20000, nrestart=5, resid=RESID)
        assert info.status == 0, lib.last_error()
    finally:
        lib.batch_destroy_L(B)
    lib.set_inner_precision("double")
    for l, dims in enumerate(lats):
        V = int(np.prod(dims))
        mine = [k for k, s in enumerate(systems) if s[0] == l]
        gpu.use(dims)
        L = lib.create_L("D", links[l])
        for k in mine:
            src = systems[k][2]
            assert orc.true_residual(dims, links[l], xs[k], src, mass, "even") < 1.5 * RESID, (l, k)
            b = lib.create_V("D", src, "even")
            x = lib.create_V("D", np.zeros_like(src), "even")
            _, inf, r1 = lib.invert("D", L, x, b, mass, parity="even", max_iter=20000, nrestart=5, resid=RESID)
            assert inf.status == 0, lib.last_error()
            x64 = lib.extract_V("D", x, "even")
            assert rel_err(xs[k][: 3 * V], x64[: 3 * V]) < 1e-8, (l, k)
            if max(dims) <= 12:
                _, xo, ro = orc.invert(dims, links[l], src, mass, "even", "D", max_iter=20000, nrestart=5,
                                       resid=RESID)
                assert r1.final_iter == ro.final_iter and rel_err(x64[: 3 * V], xo[: 3 * V]) < 1e-10
            lib.destroy_V("D", b)
            lib.destroy_V("D", x)
        lib.destroy_L("D", L)


def test_config5_force_16x16x16x32(gpu):
    dims = (16, 16, 16, 32)
    mass = 0.05
    V = int(np.prod(dims))
    lat = synthetic.Lattice(dims)
    lib = gpu.use(dims)
    lib.set_inner_precision("double")
    links = synthetic.asqtad_links(dims, seed=1001)
    phi = synthetic.gaussian_source(dims, seed=2002, parity="even")

    def action(fat, lng, force=False):
        lk = {"fat": fat, "lng": lng, "fatback": synthetic.backlinks_raw(dims, fat, 1),
              "lngback": synthetic.backlinks_raw(dims, lng, 3)}
        L = lib.create_L("D", lk)
        b = lib.create_V("D", phi, "even")
        x = lib.create_V("D", np.zeros_like(phi), "even")
        _, info, _ = lib.invert("D", L, x, b, mass, parity="even", max_iter=20000, nrestart=5, resid=1e-26)
        assert info.status == 0, lib.last_error()
        xr = lib.extract_V("D", x, "even")
        out = [float(phi[: 3 * V] @ xr[: 3 * V])]
        if force:
            out += list(lib.force("D", L, [x], [1.0], "even"))
            Lf = lib.create_L("F", lk)
            xf = lib.create_V("F", xr, "even")
            out += list(lib.force("F", Lf, [xf], [1.0], "even"))
            lib.destroy_V("F", xf)
            lib.destroy_L("F", Lf)
            out.append(xr)
        for h in (b, x):
            lib.destroy_V("D", h)
        lib.destroy_L("D", L)
        return out

    S0, gf, gl, ff, fl, xr = action(links["fat"], links["lng"], force=True)
    y = orc.asqtad_dslash(dims, links, xr, "odd", "D")
    hf, hl = force_oracle.host_force(dims, xr, y, "even")
    scale = max(np.abs(hf).max(), np.abs(hl).max())
    assert max(np.abs(gf - hf).max(), np.abs(gl - hl).max()) <= 1e-12 * scale
    assert max(np.abs(ff - hf).max(), np.abs(fl - hl).max()) <= 1e-5 * scale
    gnorm = float(np.sqrt(gf @ gf + gl @ gl))
    rng = np.random.default_rng(3003)
    h = 1e-5
    worst = 0.0
    for _ in range(32):
        dirs = []
        for key in ("fat", "lng"):
            U = synthetic.links_raw_to_lex(dims, links[key])
            a = rng.standard_normal(U.shape) + 1j * rng.standard_normal(U.shape)
            T = 0.5 * (a + np.conj(np.swapaxes(a, -1, -2)))
            T = T - (np.trace(T, axis1=-2, axis2=-1) / 3.0)[..., None, None] * np.eye(3)
            dirs.append(synthetic._to_raw_links(lat, 1j * T @ U))
        Sp = action(links["fat"] + h * dirs[0], links["lng"] + h * dirs[1])[0]
        Sm = action(links["fat"] - h * dirs[0], links["lng"] - h * dirs[1])[0]
        fd = (Sp - Sm) / (2 * h)
        an = float(gf @ dirs[0] + gl @ dirs[1])
        dnorm = float(np.sqrt(dirs[0] @ dirs[0] + dirs[1] @ dirs[1]))
        worst = max(worst, abs(fd - an) / (gnorm * dnorm))
    assert worst <= 1e-6, worst
