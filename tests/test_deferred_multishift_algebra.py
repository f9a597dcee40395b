"""CPU: the algebra of the mixed multi-shift's deferred shift updates.

The FP32 sloppy recurrence of the mixed multi-shift (csrc/solvers.cu
MsDeferred; csrc/blas.cu k_ms_defer, k_ms_coef, k_ms_flush) does not update
the shifted solutions and directions every iteration.  It stores the base
residual r(t) of every iteration of a segment and the scalars each shift
would use, x += b_t p(t) and p(t+1) = z_t r(t) + a_t p(t), and at the end of
the segment applies the expansion
    x += GX p(0) + sum_u CX[u] r(u),   p(m) = P p(0) + sum_u D[u] r(u),
with P = prod_t a_t, GX = sum_t b_t P_t, D[u] = z_u prod_{t>u} a_t and
CX[u] = sum_{t>u} b_t D_t[u].  k_ms_coef computes each column u of D and CX
from the entries t >= u only.  This test restates that computation in numpy
and checks it against explicit updates of a multi-shift CG in the reference's
notation (ks_multicg_offset.cpp:475-498, 587-598, 142-184) on a small SPD
matrix, across segment boundaries, including a shift that stops updating
mid-segment.
"""
import numpy as np


def column_coefficients(entries, m):
    """k_ms_coef's per-column recurrence: entries[t] = (b, a, z, upd) of one
    shift; returns GX, P, CX[0..m), D[0..m)."""
    CX = np.zeros(m)
    D = np.zeros(m)
    for u in range(m):
        d = cx = 0.0
        for t in range(u, m):
            b, a, z, upd = entries[t]
            if t == u:
                if upd & 2:
                    d = z
            else:
                if upd & 1:
                    cx += b * d
                if upd & 2:
                    d *= a
        CX[u], D[u] = cx, d
    P, GX = 1.0, 0.0
    for b, a, z, upd in entries[:m]:
        if upd & 1:
            GX += b * P
        if upd & 2:
            P *= a
    return GX, P, CX, D


def multishift_history(A, b, shifts_abs, iters, stop_at=None):
    """Reference-notation multi-shift CG with explicit updates; returns the
    final x, p and per-iteration (scalars, residual) history.  stop_at[k]:
    iteration after which shift k is no longer updated (its x is updated in
    that iteration, its p not)."""
    n, N = len(shifts_abs), len(b)
    jl = 0
    sh = shifts_abs - shifts_abs[jl]
    x = np.zeros((n, N))
    p = np.tile(b, (n, 1))
    r = b.copy()
    zeta_i = np.ones(n); zeta_im1 = np.ones(n); zeta_ip1 = np.ones(n)
    beta_i = np.zeros(n); beta_im1 = -np.ones(n); alpha = np.zeros(n)
    rsq = r @ r
    hist, rs = [], []
    first = True
    for it in range(1, iters + 1):
        ttt = -(A + shifts_abs[jl] * np.eye(N)) @ p[jl]
        pkp = p[jl] @ ttt
        if not first:
            beta_im1, zeta_im1, zeta_i = beta_i.copy(), zeta_i.copy(), zeta_ip1.copy()
        first = False
        beta_i = beta_i.copy(); zeta_ip1 = zeta_ip1.copy()
        beta_i[jl] = -rsq / pkp
        zeta_ip1[jl] = 1.0
        for k in range(n):
            if k == jl:
                continue
            z = zeta_i[k] * zeta_im1[k] * beta_im1[jl]
            c1 = beta_i[jl] * alpha[jl] * (zeta_im1[k] - zeta_i[k])
            c2 = zeta_im1[k] * beta_im1[jl] * (1.0 + sh[k] * beta_i[jl])
            zeta_ip1[k] = z / (c1 + c2)
            beta_i[k] = beta_i[jl] * zeta_ip1[k] / zeta_i[k]
        r = r + beta_i[jl] * ttt
        oldrsq, rsq = rsq, r @ r
        alpha = alpha.copy()
        alpha[jl] = rsq / oldrsq
        for k in range(n):
            if k != jl:
                alpha[k] = alpha[jl] * zeta_ip1[k] * beta_i[k] / (zeta_i[k] * beta_i[jl])
        entries = []
        for k in range(n):
            done = stop_at is not None and stop_at[k] is not None
            upd = 0 if done and it > stop_at[k] else (1 | (0 if done and it == stop_at[k] else 2))
            entries.append((beta_i[k], alpha[k], zeta_ip1[k], upd))
            if upd & 1:
                x[k] = x[k] + beta_i[k] * p[k]
            if upd & 2:
                p[k] = zeta_ip1[k] * r + alpha[k] * p[k]
        hist.append(entries)
        rs.append(r.copy())
    return x, p, hist, rs


def test_deferred_expansion_matches_explicit_updates():
    rng = np.random.default_rng(3)
    N = 48
    Q, _ = np.linalg.qr(rng.standard_normal((N, N)))
    A = Q @ np.diag(np.logspace(-3, 0, N)) @ Q.T
    b = rng.standard_normal(N)
    shifts = np.array([0.0, 2e-3, 1e-2, 0.1, 0.6])
    iters = 36
    stop_at = [None, None, None, 20, 11]  # heavy shifts stop mid-segment
    x_ref, p_ref, hist, rs = multishift_history(A, b, shifts, iters, stop_at)
    n = len(shifts)
    bounds = [0, 5, 6, 19, 36]  # segments of 5, 1, 13 and 17 iterations
    x = np.zeros((n, N))
    p = np.tile(b, (n, 1))
    for s0, s1 in zip(bounds[:-1], bounds[1:]):
        m = s1 - s0
        H = np.array(rs[s0:s1])
        for k in range(n):
            GX, P, CX, D = column_coefficients([hist[t][k] for t in range(s0, s1)], m)
            x[k] = x[k] + GX * p[k] + CX @ H
            p[k] = P * p[k] + D @ H
    for k in range(n):
        assert np.abs(x[k] - x_ref[k]).max() <= 1e-13 * np.abs(x_ref[k]).max(), k
        if stop_at[k] is None:
            assert np.abs(p[k] - p_ref[k]).max() <= 1e-13 * np.abs(p_ref[k]).max(), k
