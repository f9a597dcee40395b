"""GPU: FP32 inner solves with 12-real and 13-real Naik links
(QPHIX_B200_set_link_compression).

The rebuilt third rows make the FP32 operator equal to the 18-real one up to
FP32 rounding, so a mixed-precision solve with compression must take the same
number of inner iterations to within a few and reach the same FP64 true
residual (checked by the oracle).  SU(3) Naik links times one real factor
are 12-real; U(3) links times a real factor per link are 13-real; a Naik
field with a non-unitary part must be detected and solved with 18-real
links.
"""
import numpy as np
import pytest

from conftest import fields, orc, synthetic

pytestmark = pytest.mark.gpu

DIMS = (8, 8, 8, 8)
RESID = 1e-20


def _solve(lib, links, src, mass, compress, multi=None):
    lib.set_link_compression(compress)
    lib.set_inner_precision("single")
    try:
        L = lib.create_L("D", links)
        b = lib.create_V("D", src, "even")
        if multi is None:
            x = lib.create_V("D", np.zeros_like(src), "even")
            it, info, res = lib.invert("D", L, x, b, mass, parity="even", max_iter=4000, nrestart=5, resid=RESID)
            st = lib.last_stats()
            sols = [lib.extract_V("D", x, "even")]
            lib.destroy_V("D", x)
        else:
            xs = [lib.create_V("D", np.zeros_like(src), "even") for _ in multi]
            it, info, res = lib.invert_multi("D", L, xs, b, multi, parity="even", max_iter=4000, nrestart=5,
                                             resid=RESID)
            st = lib.last_stats()
            sols = [lib.extract_V("D", x, "even") for x in xs]
            for x in xs:
                lib.destroy_V("D", x)
        assert info.status == 0, lib.last_error()
        lib.destroy_V("D", b)
        lib.destroy_L("D", L)
    finally:
        lib.set_link_compression(False)
        lib.set_inner_precision("double")
    return st, sols


@pytest.mark.parametrize("smear", [False, True])
def test_compressed_naik_links_solve(gpu, smear):
    lib = gpu.use(DIMS)
    links = fields(DIMS, seed=21, smear=smear, eps_fat=0.2 if smear else 0.3)
    src = synthetic.gaussian_source(DIMS, seed=2002, parity="even")
    st0, (x0,) = _solve(lib, links, src, 0.03, False)
    st1, (x1,) = _solve(lib, links, src, 0.03, True)
    assert st0.links_compressed == 0 and st1.links_compressed == 1
    # the two FP32 operators differ by rounding: the reliable-update schedule,
    # and with it the inner iteration count, can move by a few per cent
    assert abs(st1.iterations - st0.iterations) <= max(20, st0.iterations // 20)
    assert orc.true_residual(DIMS, links, x1, src, 0.03, "even") < 1.5 * RESID


@pytest.mark.parametrize("mode", [1, 2])
def test_compressed_multishift(gpu, mode):
    """Mixed multi-shift with 12-real (SU(3) Naik links) and 13-real (U(3)
    Naik links) inner Dslash: every shift reaches the FP64 tolerance."""
    lib = gpu.use(DIMS)
    links = fields(DIMS, seed=21)
    if mode == 2:
        links = _naik_variant(links, "phase")
    src = synthetic.gaussian_source(DIMS, seed=2002, parity="even")
    masses = np.sqrt(0.02 ** 2 + np.logspace(-3, 0, 4) / 4)
    st, xs = _solve(lib, links, src, None, True, multi=masses)
    assert st.links_compressed == mode
    for m, x in zip(masses, xs):
        assert orc.true_residual(DIMS, links, x, src, m, "even") < 1.5 * RESID


def _naik_variant(links, how, seed=5):
    """Naik links of `links` changed per link: 'phase' multiplies each by a
    random U(1) phase (U(3) times the Naik factor, the HISQ form), 'scale' by
    a random real factor per site, 'noise' adds a small non-unitary part."""
    dims = DIMS
    V = int(np.prod(dims))
    rng = np.random.default_rng(seed)
    lng = links["lng"].reshape(V, 4, 9, 2)
    z = lng[..., 0] + 1j * lng[..., 1]
    if how == "phase":
        z = z * np.exp(1j * rng.uniform(-np.pi, np.pi, (V, 4)))[:, :, None]
    elif how == "scale":
        z = z * (1.0 + 0.1 * rng.random(V))[:, None, None]
    else:
        z = z + 1e-3 * np.abs(z).max() * (rng.standard_normal(z.shape) + 1j * rng.standard_normal(z.shape))
    out = dict(links)
    out["lng"] = np.stack([z.real, z.imag], axis=-1).reshape(-1)
    out["lngback"] = synthetic.backlinks_raw(dims, out["lng"], 3)
    return out


@pytest.mark.parametrize("how", ["phase", "scale"])
def test_u3_naik_links_13_real(gpu, how):
    """Naik links that are U(3) times a real factor per link (a random phase
    per link, or a factor that varies by site) are not 12-real but are
    13-real: one complex ratio per link rebuilds the third row exactly.  The
    compressed FP32 solve matches the 18-real one."""
    lib = gpu.use(DIMS)
    links = _naik_variant(fields(DIMS, seed=21), how)
    src = synthetic.gaussian_source(DIMS, seed=2002, parity="even")
    st0, (x0,) = _solve(lib, links, src, 0.03, False)
    st1, (x1,) = _solve(lib, links, src, 0.03, True)
    assert st0.links_compressed == 0 and st1.links_compressed == 2
    assert abs(st1.iterations - st0.iterations) <= max(20, st0.iterations // 20)
    assert orc.true_residual(DIMS, links, x1, src, 0.03, "even") < 1.5 * RESID


def test_non_unitary_naik_links_keep_18_reals(gpu):
    """Naik links with a non-unitary part have no ratio that rebuilds their
    third row: the check refuses them and the solve runs with 18-real links."""
    lib = gpu.use(DIMS)
    links = _naik_variant(fields(DIMS, seed=21), "noise")
    src = synthetic.gaussian_source(DIMS, seed=2002, parity="even")
    st, (x,) = _solve(lib, links, src, 0.03, True)
    assert st.links_compressed == 0
    assert orc.true_residual(DIMS, links, x, src, 0.03, "even") < 1.5 * RESID


def test_link_compression_from_environment(gpu, monkeypatch):
    """QPHIX_GPU_LINK_COMPRESSION=1 turns compression on at QPHIX_init (for
    MILC builds that call only the reference API); without it the library
    starts with 18-real links."""
    lib = gpu.use(DIMS)
    links = fields(DIMS, seed=21)
    src = synthetic.gaussian_source(DIMS, seed=2002, parity="even")

    def solve_stats():
        lib.set_inner_precision("single")
        try:
            L = lib.create_L("D", links)
            b = lib.create_V("D", src, "even")
            x = lib.create_V("D", np.zeros_like(src), "even")
            it, info, res = lib.invert("D", L, x, b, 0.03, parity="even", max_iter=4000, nrestart=5, resid=RESID)
            assert info.status == 0, lib.last_error()
            st = lib.last_stats()
            for h in (x, b):
                lib.destroy_V("D", h)
            lib.destroy_L("D", L)
        finally:
            lib.set_inner_precision("double")
        return st

    try:
        monkeypatch.setenv("QPHIX_GPU_LINK_COMPRESSION", "1")
        lib.finalize()
        assert lib.init(DIMS) == 0
        assert solve_stats().links_compressed == 1
        monkeypatch.delenv("QPHIX_GPU_LINK_COMPRESSION")
        lib.finalize()
        assert lib.init(DIMS) == 0
        assert solve_stats().links_compressed == 0
    finally:
        lib.set_link_compression(False)
