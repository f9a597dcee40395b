"""GPU: batched solves (QPHIX_B200_D3_batch_invert) through the C ABI.

Several lattices of different sizes, several right-hand sides per lattice
(segments of 6 + 1, 2 and 1 systems: register groups of G = 3, 2 and 1),
different masses, one device run.  Every
system must reach its FP64 true-residual tolerance as measured by the oracle,
agree with the oracle's FP64 CG solution, and be bit-reproducible run to run.
The oracle here is the plain-C restatement (oracle/qphix_oracle.c, built as
oracle/_build/liboracle.so); it is tied to the reference's own host code by
the CPU pin tests (tests/test_oracle_pin.py, tests/test_golden.py), not
called here.
"""
import os

import numpy as np
import pytest

from conftest import fields, orc, rel_err, synthetic

pytestmark = pytest.mark.gpu

LATS = [(8, 8, 8, 8), (8, 4, 4, 8), (12, 8, 4, 4)]
RESID = 1e-20


def _systems():
    """(lattice, mass, source): 7 systems on lattice 0, 2 on 1, 1 on 2."""
    sys = []
    for k, m in enumerate([0.05, 0.07, 0.05, 0.1, 0.06, 0.2, 0.08]):
        sys.append((0, m, synthetic.gaussian_source(LATS[0], seed=500 + k, parity="even")))
    for k, m in enumerate([0.05, 0.03]):
        sys.append((1, m, synthetic.gaussian_source(LATS[1], seed=600 + k, parity="even")))
    sys.append((2, 0.04, synthetic.gaussian_source(LATS[2], seed=700, parity="even")))
    return sys


def _links(l):
    return fields(LATS[l], seed=1001 + l)


@pytest.fixture(scope="module")
def batch(gpu):
    lib = gpu.use((4, 4, 4, 4))
    B = lib.batch_create_L([(d, _links(i)) for i, d in enumerate(LATS)])
    assert B, lib.last_error()
    yield lib, B
    lib.batch_destroy_L(B)


def _check_solutions(systems, res, xs):
    for (l, m, src), r, x in zip(systems, res, xs):
        dims = LATS[l]
        assert r.final_rsq <= RESID
        assert orc.true_residual(dims, _links(l), x, src, m, "even") < 1.5 * RESID
        V = int(np.prod(dims))
        assert not np.any(x[V * 3:]), "odd sites of an even solve must be untouched"


@pytest.mark.parametrize("graphs", ["1", "0"])
def test_batch_every_system_converges(batch, graphs):
    lib, B = batch
    systems = _systems()
    old = os.environ.get("QPHIX_B200_GRAPHS")
    os.environ["QPHIX_B200_GRAPHS"] = graphs
    try:
        it, info, res, xs = lib.batch_invert(B, systems, max_iter=4000, resid=RESID)
    finally:
        if old is None:
            del os.environ["QPHIX_B200_GRAPHS"]
        else:
            os.environ["QPHIX_B200_GRAPHS"] = old
    assert info.status == 0, lib.last_error()
    assert it == max(r.final_iter for r in res) > 0
    assert all(r.final_restart >= 1 for r in res)
    _check_solutions(systems, res, xs)


def test_batch_matches_fp64_cg_and_is_reproducible(batch):
    lib, B = batch
    systems = _systems()
    _, _, res1, xs1 = lib.batch_invert(B, systems, max_iter=4000, resid=RESID)
    _, _, res2, xs2 = lib.batch_invert(B, systems, max_iter=4000, resid=RESID)
    for a, b in zip(xs1, xs2):
        assert np.array_equal(a, b)
    assert [r.final_iter for r in res1] == [r.final_iter for r in res2]
    for (l, m, src), x in list(zip(systems, xs1))[::3]:
        dims = LATS[l]
        _, xo, _ = orc.invert(dims, _links(l), src, m, "even", "D", 4000, 5, RESID)
        V = int(np.prod(dims))
        assert rel_err(x[: V * 3], xo[: V * 3]) < 1e-8


def test_batch_initial_guess_and_zero_source(batch):
    lib, B = batch
    systems = _systems()[:3]
    _, _, res, xs = lib.batch_invert(B, systems, max_iter=4000, resid=RESID)
    # restarted from their solutions the systems converge at the first true residual
    warm = [(l, m, s, x) for (l, m, s), x in zip(systems, xs)]
    it, _, res2, xs2 = lib.batch_invert(B, warm, max_iter=4000, resid=1e-18)
    assert it == 0 and all(r.final_iter == 0 for r in res2)
    for a, b in zip(xs, xs2):
        assert np.array_equal(a, b)
    # a zero source gives x = 0 without iterating; the other systems still solve
    zsys = [(0, 0.05, np.zeros_like(systems[0][2]))] + systems[1:]
    _, info, res3, xs3 = lib.batch_invert(B, zsys, max_iter=4000, resid=RESID)
    assert info.status == 0
    assert res3[0].final_iter == 0 and not np.any(xs3[0])
    _check_solutions(zsys[1:], res3[1:], xs3[1:])


def test_batch_iteration_cap(batch):
    lib, B = batch
    systems = _systems()
    it, info, res, xs = lib.batch_invert(B, systems, max_iter=10, nrestart=2, resid=1e-30)
    assert info.status == 0
    assert it == 20
    for (l, m, src), r, x in zip(systems, res, xs):
        tr = orc.true_residual(LATS[l], _links(l), x, src, m, "even")
        assert r.final_rsq > 1e-30
        assert abs(tr - r.final_rsq) <= 1e-6 * tr


def test_batch_rejects_bad_arguments(batch):
    lib, B = batch
    src = synthetic.gaussian_source(LATS[0], seed=1, parity="even")
    _, info, _, _ = lib.batch_invert(B, [(0, 0.1, src)], parity="evenodd")
    assert info.status != 0 and "parity" in lib.last_error()
    _, info, _, _ = lib.batch_invert(B, [(5, 0.1, src)])
    assert info.status != 0 and "lattice index" in lib.last_error()
    _, info, _, _ = lib.batch_invert(B, [(0, 0.1, src)] * 65)
    assert info.status != 0 and "nsys" in lib.last_error()
    bad = lib.batch_create_L([((6, 4, 4, 4), _links(1))])
    assert not bad and "Nx/2 must be even" in lib.last_error()


def test_batch_dslash_tuner(batch):
    """16 systems on one lattice: the tuner picks 4, 2 or 1 systems per
    thread for the FP32 batched Dslash; forcing another choice gives the same
    solutions to the solve tolerance."""
    lib, B = batch
    systems = [(0, 0.04 + 0.01 * (k % 5), synthetic.gaussian_source(LATS[0], seed=900 + k, parity="even"))
               for k in range(16)]
    _, info, res, xs = lib.batch_invert(B, systems, max_iter=4000, resid=RESID)
    assert info.status == 0, lib.last_error()
    g = lib.last_stats().batch_rhs_per_thread
    assert g in (1, 2, 4)
    _check_solutions(systems, res, xs)
    other = 2 if g != 2 else 1
    old = os.environ.get("QPHIX_B200_BATCH_G")
    os.environ["QPHIX_B200_BATCH_G"] = str(other)
    try:
        _, info2, _, xs2 = lib.batch_invert(B, systems, max_iter=4000, resid=RESID)
        assert lib.last_stats().batch_rhs_per_thread == other
    finally:
        if old is None:
            del os.environ["QPHIX_B200_BATCH_G"]
        else:
            os.environ["QPHIX_B200_BATCH_G"] = old
    assert info2.status == 0
    V = int(np.prod(LATS[0]))
    for a, b in zip(xs, xs2):
        assert rel_err(a[: V * 3], b[: V * 3]) < 1e-8
