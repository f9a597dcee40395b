"""GPU: size-independent properties at the benchmark sizes.

The oracle finishes in seconds only on small lattices, so at 24^3x48 (the
mixed-precision workload) and 32^3x64 (the multi-shift workload) the tests
check properties that hold at any size, with the FP64 operator applied
through QPHIX_D3_asqtad_dslash as the independent check:
  * every inner precision reaches |b - M x|^2 / |b|^2 < 1e-20, the FP64 true
    residual recomputed here, the solutions agree with the FP64 CG's, and the
    16-bit inner solves take at most 30% more iterations than the FP32 one;
  * D is anti-Hermitian (<y, D_eo x> = -<D_oe y, x>) and M = 4m^2 - D D is
    Hermitian and positive, in FP64, on the full 32^3x64 lattice.
"""
import numpy as np
import pytest
import torch

from conftest import rel_err, synthetic

pytestmark = pytest.mark.gpu

RESID = 1e-20


def _fields(dims, smear=False, eps_fat=0.3):
    dev = "cuda" if torch.cuda.is_available() else None
    return synthetic.asqtad_links(dims, seed=1001, eps_fat=eps_fat, smear=smear, device=dev)


def _apply_dd(lib, L, v_raw, parity):
    """D_{p,q} D_{q,p} v on parity p, FP64, through the C ABI."""
    other = "odd" if parity == "even" else "even"
    h = lib.create_V("D", v_raw)
    t = lib.create_V("D", np.zeros_like(v_raw))
    o = lib.create_V("D", np.zeros_like(v_raw))
    lib.dslash("D", L, t, h, other)
    lib.dslash("D", L, o, t, parity)
    out = lib.extract_V("D", o)
    for x in (h, t, o):
        lib.destroy_V("D", x)
    return out


def _true_rsq(lib, L, x, b, mass, V):
    e = slice(0, 3 * V)
    full = np.zeros(6 * V)
    full[e] = x[e]
    dd = _apply_dd(lib, L, full, "even")[e]
    r = b[e] - (4 * mass * mass * x[e] - dd)
    return float(r @ r / (b[e] @ b[e]))


def test_mixed_cg_24x24x24x48_every_inner_precision(gpu):
    dims = (24, 24, 24, 48)
    mass = 0.01
    V = int(np.prod(dims))
    lib = gpu.use(dims)
    links = _fields(dims)
    src = synthetic.gaussian_source(dims, seed=2002, parity="even")
    L = lib.create_L("D", links)
    b = lib.create_V("D", src, "even")
    sols, iters = {}, {}
    try:
        for inner in ("double", "single", "half-links", "half"):
            lib.set_inner_precision(inner)
            x = lib.create_V("D", np.zeros_like(src), "even")
            it, info, res = lib.invert("D", L, x, b, mass, parity="even", max_iter=20000, nrestart=5, resid=RESID)
            assert info.status == 0, lib.last_error()
            iters[inner] = lib.last_stats().iterations
            sols[inner] = lib.extract_V("D", x, "even")
            lib.destroy_V("D", x)
            assert _true_rsq(lib, L, sols[inner], src, mass, V) < 1.5 * RESID, inner
    finally:
        lib.set_inner_precision("double")
        lib.destroy_V("D", b)
        lib.destroy_L("D", L)
    for inner in ("single", "half-links", "half"):
        assert rel_err(sols[inner][: 3 * V], sols["double"][: 3 * V]) < 1e-7, inner
    # 16-bit storage perturbs the operator by ~3e-5: a few more iterations
    # than FP32 (927 against 806 here), not twice as many
    for inner in ("half-links", "half"):
        assert iters[inner] <= 1.3 * iters["single"], (inner, iters)


def test_operator_identities_32x32x32x64(gpu):
    dims = (32, 32, 32, 64)
    V = int(np.prod(dims))
    lib = gpu.use(dims)
    links = _fields(dims, smear=True, eps_fat=0.2)
    L = lib.create_L("D", links)
    try:
        x = synthetic.gaussian_source(dims, seed=11, parity="odd")
        y = synthetic.gaussian_source(dims, seed=12, parity="even")
        hx, hy = lib.create_V("D", x), lib.create_V("D", y)
        dx, dy = lib.create_V("D", np.zeros_like(x)), lib.create_V("D", np.zeros_like(x))
        lib.dslash("D", L, dx, hx, "even")
        lib.dslash("D", L, dy, hy, "odd")
        Dx, Dy = lib.extract_V("D", dx), lib.extract_V("D", dy)
        for h in (hx, hy, dx, dy):
            lib.destroy_V("D", h)
        cx = lambda v: v[0::2] + 1j * v[1::2]  # noqa: E731
        lhs = np.vdot(cx(y), cx(Dx))
        rhs = -np.vdot(cx(Dy), cx(x))
        assert abs(lhs - rhs) < 1e-10 * abs(lhs)
        # M = 4m^2 - D_eo D_oe: <u, M v> = <M u, v> and <v, M v> >= 4 m^2 |v|^2
        m = 0.0012
        u = synthetic.gaussian_source(dims, seed=13, parity="even")
        v = synthetic.gaussian_source(dims, seed=14, parity="even")
        e = slice(0, 3 * V)
        Mu = 4 * m * m * u - _apply_dd(lib, L, u, "even")
        Mv = 4 * m * m * v - _apply_dd(lib, L, v, "even")
        a, c = np.vdot(cx(u[e]), cx(Mv[e])), np.vdot(cx(Mu[e]), cx(v[e]))
        assert abs(a - c) < 1e-10 * abs(a)
        vMv = np.vdot(cx(v[e]), cx(Mv[e]))
        assert abs(vMv.imag) < 1e-10 * abs(vMv) and vMv.real >= 4 * m * m * float(v[e] @ v[e])
    finally:
        lib.destroy_L("D", L)
