// Even-odd asqtad/HISQ Dslash on one parity block (K1) and its fused
// M^dag M epilogue (K2).
//
// Reference path: qphix_ks_dslash (ks_long_dslash.cpp:564-668) loops over
// the output sites of parity cb, gathers 8 one-hop and 8 three-hop neighbour
// vectors through NeighTable and calls the generated per-site kernel
// ks_long_dslash_vec_noinline (ks_dslash_complete_specialization.cpp:338-378,
// body absent from the reference).  Here one thread owns one output site:
//   out(x) = sum_mu F_mu(x) psi(x+mu)  - B_mu(x)^dag  psi(x-mu)
//          + sum_mu L_mu(x) psi(x+3mu) - LB_mu(x)^dag psi(x-3mu)
// The 16 links are streamed from the site-major link block; neighbour
// indices are computed in registers (periodic wrap replaces the single-node
// halo, ks_boundary.cpp:66-89); the 16 gathered vectors mostly hit L2.
//
// Roofline: 1146 flop per site against >= 1200 B (FP32, 18-real links):
// memory bound on HBM.
#include "device_common.cuh"

namespace qb {

template <typename S>
struct DslashArgs {
    VecView<S> out;
    VecView<S> in;
    LinkView<S> links;
    Geom g;
    int cb;
};

template <typename S, typename A>
__device__ __forceinline__ void dslash_site(const DslashArgs<S> &a, int j, A acc[6])
{
    const SiteCoords s = decode(a.g, a.cb, j);
#pragma unroll
    for (int i = 0; i < 6; ++i) acc[i] = A(0);
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
        A u[18], v[6];
        // fat link, forward:  F_dir(x) psi(x + dir)
        a.in.load(neighbor(a.g, s, 2 * dir + 1), v);
        a.links.load(0 * 4 + dir, j, u);
        mv_add(acc, u, v);
        // fat link, backward: -B_dir(x)^dag psi(x - dir)
        a.in.load(neighbor(a.g, s, 2 * dir), v);
        a.links.load(1 * 4 + dir, j, u);
        mv_adj_sub(acc, u, v);
        // Naik link, forward:  L_dir(x) psi(x + 3 dir)
        a.in.load(neighbor(a.g, s, 8 + 2 * dir + 1), v);
        a.links.load(2 * 4 + dir, j, u);
        mv_add(acc, u, v);
        // Naik link, backward: -LB_dir(x)^dag psi(x - 3 dir)
        a.in.load(neighbor(a.g, s, 8 + 2 * dir), v);
        a.links.load(3 * 4 + dir, j, u);
        mv_adj_sub(acc, u, v);
    }
}

template <typename S>
__global__ void __launch_bounds__(kBlock) k_dslash(DslashArgs<S> a, const SolverState *st, int gate)
{
    using A = typename Acc<S>::type;
    if (st && gated_off(st, gate)) return;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= a.g.vh) return;
    A acc[6];
    dslash_site<S, A>(a, j, acc);
    a.out.store(j, acc);
}

// ttt = D tmp + m4 * p ;  pkp = sum p . ttt  (calc_pkp, ks_d_congrad_fn.cpp:159-171;
// ks_multicg_offset.cpp:107-122), then the scalar step of the solver.
template <typename S>
__global__ void __launch_bounds__(kBlock)
k_dslash_mdagm(DslashArgs<S> a, VecView<S> pv, double m4, SolverState *st, double *partials,
               int gate, int mode)
{
    using A = typename Acc<S>::type;
    if (gated_off(st, gate)) return;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    double dot[1] = {0.0};
    if (j < a.g.vh) {
        A acc[6], p[6];
        dslash_site<S, A>(a, j, acc);
        pv.load_cg(j, p);
        const A m = (A)m4;
#pragma unroll
        for (int i = 0; i < 6; ++i) acc[i] = acc[i] + m * p[i];
        // the product is formed from the stored (rounded) value, as the
        // reference reads ttt back from memory; store() leaves it in acc
        a.out.store(j, acc);
#pragma unroll
        for (int i = 0; i < 6; ++i) dot[0] += (double)(p[i] * acc[i]);
    }
    grid_reduce<1>(dot, partials, &st->counter, [&](const double *tot) {
        st->pkp = tot[0];
        st->iteration += 1;
        if (mode == 0) {
            st->a = round_to(-st->rsq / tot[0], st->prec_single);
        } else {
            // multi-shift scalar recurrences (ks_multicg_offset.cpp:475-496);
            // the values of the previous iteration are scrolled first
            // (:617-622), which the reference does at the end of that iteration
            const int single = st->prec_single;
            const int jl = st->j_low;
            if (!st->first_iter) {
                for (int k = 0; k < st->num_now; ++k) {
                    st->beta_im1[k] = st->beta_i[k];
                    st->zeta_im1[k] = st->zeta_i[k];
                    st->zeta_i[k] = st->zeta_ip1[k];
                }
            }
            st->first_iter = 0;
            st->beta_i[jl] = round_to(-st->rsq / tot[0], single);
            st->zeta_ip1[jl] = 1.0;
            int nn = st->num_now;
            for (int k = 0; k < nn; ++k) {
                if (k == jl) continue;
                double z = round_to(round_to(st->zeta_i[k] * st->zeta_im1[k], single) * st->beta_im1[jl], single);
                const double c1 = round_to(round_to(st->beta_i[jl] * st->alpha[jl], single) *
                                               round_to(st->zeta_im1[k] - st->zeta_i[k], single), single);
                const double c2 = round_to(round_to(st->zeta_im1[k] * st->beta_im1[jl], single) *
                                               (1.0 + round_to(st->shifts[k] * st->beta_i[jl], single)), single);
                const double den = round_to(c1 + c2, single);
                if (den != 0.0) z = round_to(z / den, single);
                else { z = 0.0; st->finished[k] = 1; }
                st->zeta_ip1[k] = z;
                if (st->zeta_i[k] != 0.0)
                    st->beta_i[k] = round_to(round_to(st->beta_i[jl] * z, single) / st->zeta_i[k], single);
                else { st->zeta_ip1[k] = 0.0; st->beta_i[k] = 0.0; st->finished[k] = 1; }
                if (st->finished[k] == 1 && k == nn - 1 && k > jl) nn--;
            }
            st->num_now = nn;
        }
    });
}

template <typename S>
static DslashArgs<S> make_args(const Launch &L, VecBlock out, VecBlock in, const LinkSet &ls, int cb)
{
    DslashArgs<S> a;
    a.out = view<S>(out, L.g->vh);
    a.in = view<S>(in, L.g->vh);
    if constexpr (std::is_same<S, __half>::value) {
        a.links = LinkView<__half>{static_cast<const short2 *>(ls.blk[cb]), L.g->vh,
                                   ls.link_max[0] / 32767.0f, ls.link_max[1] / 32767.0f};
    } else {
        a.links = LinkView<S>{static_cast<const cx_t<S> *>(ls.blk[cb]), L.g->vh};
    }
    a.g = *L.g;
    a.cb = cb;
    return a;
}

template <typename S>
static void launch_dslash(const Launch &L, VecBlock out, VecBlock in, const LinkSet &ls, int cb,
                          const SolverState *st, int gate)
{
    auto a = make_args<S>(L, out, in, ls, cb);
    k_dslash<S><<<grid_for(L.g->vh), kBlock, 0, L.stream>>>(a, st, gate);
}

void dslash(Prec p, const Launch &L, VecBlock out, VecBlock in, const LinkSet &ls, int cb)
{
    switch (p) {
    case Prec::Double: launch_dslash<double>(L, out, in, ls, cb, nullptr, -1); break;
    case Prec::Single: launch_dslash<float>(L, out, in, ls, cb, nullptr, -1); break;
    case Prec::Half: launch_dslash<__half>(L, out, in, ls, cb, nullptr, -1); break;
    }
}

void dslash_gated(Prec p, const Launch &L, VecBlock out, VecBlock in, const LinkSet &ls, int cb,
                  SolverState *st, int gate)
{
    switch (p) {
    case Prec::Double: launch_dslash<double>(L, out, in, ls, cb, st, gate); break;
    case Prec::Single: launch_dslash<float>(L, out, in, ls, cb, st, gate); break;
    case Prec::Half: launch_dslash<__half>(L, out, in, ls, cb, st, gate); break;
    }
}

template <typename S>
static void launch_mdagm(const Launch &L, VecBlock ttt, VecBlock tmp, const LinkSet &ls,
                         VecBlock pv, double m4, int cb, SolverState *st, double *partials,
                         int gate, int mode)
{
    auto a = make_args<S>(L, ttt, tmp, ls, cb);
    k_dslash_mdagm<S><<<grid_for(L.g->vh), kBlock, 0, L.stream>>>(a, view<S>(pv, L.g->vh), m4, st,
                                                                   partials, gate, mode);
}

void dslash_mdagm_dot(Prec p, const Launch &L, VecBlock ttt, VecBlock tmp, const LinkSet &ls,
                      VecBlock pv, double m4, int cb, SolverState *st, double *partials, int gate,
                      int mode)
{
    switch (p) {
    case Prec::Double: launch_mdagm<double>(L, ttt, tmp, ls, pv, m4, cb, st, partials, gate, mode); break;
    case Prec::Single: launch_mdagm<float>(L, ttt, tmp, ls, pv, m4, cb, st, partials, gate, mode); break;
    case Prec::Half: launch_mdagm<__half>(L, ttt, tmp, ls, pv, m4, cb, st, partials, gate, mode); break;
    }
}

}  // namespace qb
