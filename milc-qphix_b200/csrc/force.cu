// Fermion force: the gradient of S = phi^dag (4m^2 - D_pq D_qp)^{-1} phi with
// respect to the fat and Naik links (no counterpart in the reference, whose
// force entry points are the gauge force, gauge_force_imp.cpp).
//
// With x = (4m^2 - D_pq D_qp)^{-1} phi on parity p and y = D_qp x on the
// other parity q, dS = x^dag dD_pq y - y^dag dD_qp x (D is anti-Hermitian).
// A link U = F_mu(z) (or L_mu(z), hop h = 1 or 3) enters D forward at z and,
// through the backward link the caller derives from it, adjoint at z + h mu;
// both uses combine into
//     dS = 2 s(z) Re tr[ dU W(z+h mu) W(z)^dag ],
// W = x on parity p and y on parity q, s = +1 on p and -1 on q.  The kernel
// writes the gradient with respect to the real and imaginary parts of every
// raw link entry (the layout of QPHIX_*_asqtad_create_L_from_raw's fat and
// lng arrays):
//     dS/dRe U_ab = 2 s Re M_ab,   dS/dIm U_ab = -2 s Im M_ab,
//     M_ab = conj(W(z)_a) W(z+h mu)_b.
// D x is recomputed from x with the Dslash rather than kept from the solve.
// The kernel is a pure outer product: 2 x 18 reals written per (site,
// direction) against 3 colour vectors read, so it is bound by the writes.
#include <string>
#include <vector>

#include "context.h"
#include "device_common.cuh"

namespace qb {

// One block covers 64 consecutive raw sites x 4 directions, whose gradient
// entries are one contiguous run of 256 x 18 reals per link family.  The
// outer products go through shared memory so that the block writes that run
// with coalesced stores (a thread's own 18 reals are 144 bytes apart from its
// neighbour's).  ACC = false: the first solution writes the gradient; true:
// later ones add to it.
template <typename R, bool ACC>
__global__ void __launch_bounds__(kBlock) k_force(R *gfat, R *glng, VecView<R> x, VecView<R> y, Geom g, int P,
                                                  R coef)
{
    __shared__ R stage[kBlock * 18];
    const long long n = 8LL * g.vh;  // (raw site, direction) pairs
    const long long t0 = (long long)blockIdx.x * kBlock;
    const long long t = t0 + threadIdx.x;
    R w[6], wn[2][6];
    R sc = 0;
    if (t < n) {
        const int i = (int)(t >> 2), mu = (int)(t & 3);
        const int p = i >= g.vh ? 1 : 0;
        const int j = i - p * g.vh;
        const SiteCoords s = decode(g, p, j);
        const VecView<R> &here = (p == P) ? x : y;
        const VecView<R> &there = (p == P) ? y : x;
        here.load(j, w);
        there.load(neighbor(g, s, 2 * mu + 1), wn[0]);
        there.load(neighbor(g, s, 8 + 2 * mu + 1), wn[1]);
        sc = (p == P ? R(2) : R(-2)) * coef;
    }
    const long long nout = (n - t0 < kBlock ? n - t0 : kBlock) * 18;  // reals this block writes
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        if (t < n) {
            R *o = stage + threadIdx.x * 18;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    o[6 * a + 2 * b] = sc * (w[2 * a] * wn[h][2 * b] + w[2 * a + 1] * wn[h][2 * b + 1]);
                    o[6 * a + 2 * b + 1] = -sc * (w[2 * a] * wn[h][2 * b + 1] - w[2 * a + 1] * wn[h][2 * b]);
                }
            }
        }
        __syncthreads();
        R *dst = (h == 0 ? gfat : glng) + t0 * 18;
        for (int e = threadIdx.x; e < nout; e += kBlock) {
            if (ACC) dst[e] += stage[e];
            else dst[e] = stage[e];
        }
        __syncthreads();
    }
}

template <typename Real> struct ForceApi;
template <> struct ForceApi<double> {
    using FL = QPHIX_D3_FermionLinksAsqtad;
    using CV = QPHIX_D3_ColorVector;
    static constexpr Prec prec = Prec::Double;
};
template <> struct ForceApi<float> {
    using FL = QPHIX_F3_FermionLinksAsqtad;
    using CV = QPHIX_F3_ColorVector;
    static constexpr Prec prec = Prec::Single;
};

template <typename Real>
static void force_impl(typename ForceApi<Real>::FL *H, int n, const Real *coef, typename ForceApi<Real>::CV **x,
                       QPHIX_evenodd_t parity, Real *grad_fat, Real *grad_lng)
{
    Context &c = ctx();
    if (!c.initialized) throw Error("asqtad_force: QPhiX library used before QPHIX_init");
    if (!H || !coef || !x || !grad_fat || !grad_lng) throw Error("asqtad_force: NULL argument");
    if (n < 1) throw Error("asqtad_force: n must be at least 1");
    if (parity != QPHIX_EVEN && parity != QPHIX_ODD) throw Error("asqtad_force: parity must be EVEN or ODD");
    // the outer products need the t neighbours of the slab's boundary sites
    if (c.halo.on && c.halo.nranks > 1) throw Error("asqtad_force: not available with several ranks");
    const int P = parity == QPHIX_EVEN ? 0 : 1;
    for (int k = 0; k < n; ++k)
        if (!x[k] || !(x[k]->parity & parity)) throw Error("asqtad_force: solution vector lacks the parity");
    const Launch L = c.launch();
    const size_t nraw = (size_t)2 * c.g.vh * 72;
    Real *g = static_cast<Real *>(dev_alloc(2 * nraw * sizeof(Real)));
    VecBlock y = alloc_vec(ForceApi<Real>::prec);
    try {
        QB_CUDA(cudaEventRecord(c.ev_solve[0], c.stream));
        const int grid = (int)((8LL * c.g.vh + kBlock - 1) / kBlock);
        for (int k = 0; k < n; ++k) {
            const VecBlock xb = x[k]->blk[P];
            dslash(ForceApi<Real>::prec, L, y, xb, H->links, 1 - P);  // y = D_qp x
            const VecView<Real> xv = view<Real>(xb, c.g.vh), yv = view<Real>(y, c.g.vh);
            if (k == 0) k_force<Real, false><<<grid, kBlock, 0, c.stream>>>(g, g + nraw, xv, yv, c.g, P, coef[k]);
            else k_force<Real, true><<<grid, kBlock, 0, c.stream>>>(g, g + nraw, xv, yv, c.g, P, coef[k]);
        }
        QB_CUDA(cudaGetLastError());
        QB_CUDA(cudaEventRecord(c.ev_solve[1], c.stream));
        d2h_copy(grad_fat, g, nraw * sizeof(Real));
        d2h_copy(grad_lng, g + nraw, nraw * sizeof(Real));
        sync_check();
        float ms = 0.f;
        QB_CUDA(cudaEventElapsedTime(&ms, c.ev_solve[0], c.ev_solve[1]));
        c.stats = Stats{};
        c.stats.solve_ms = ms;
    } catch (...) {
        free_vec(y);
        dev_free(g);
        throw;
    }
    free_vec(y);
    dev_free(g);
}

}  // namespace qb

namespace {
template <typename F>
QPHIX_status_t force_guarded(F f)
{
    try {
        f();
        qb::ctx().last_error.clear();
        return QPHIX_SUCCESS;
    } catch (const qb::Error &e) {
        qb::ctx().last_error = e.what();
        return e.status;
    } catch (const std::exception &e) {
        qb::ctx().last_error = e.what();
        return QPHIX_FAIL;
    }
}
}  // namespace

#pragma GCC visibility push(default)
extern "C" {

QPHIX_status_t QPHIX_B200_D3_asqtad_force(QPHIX_D3_FermionLinksAsqtad *L, int n, const double *coef,
                                          QPHIX_D3_ColorVector **x, QPHIX_evenodd_t parity, double *grad_fat,
                                          double *grad_lng)
{
    return force_guarded([&] { qb::force_impl<double>(L, n, coef, x, parity, grad_fat, grad_lng); });
}

QPHIX_status_t QPHIX_B200_F3_asqtad_force(QPHIX_F3_FermionLinksAsqtad *L, int n, const float *coef,
                                          QPHIX_F3_ColorVector **x, QPHIX_evenodd_t parity, float *grad_fat,
                                          float *grad_lng)
{
    return force_guarded([&] { qb::force_impl<float>(L, n, coef, x, parity, grad_fat, grad_lng); });
}

}  // extern "C"
#pragma GCC visibility pop
