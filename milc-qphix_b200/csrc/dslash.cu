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
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

#include "device_common.cuh"
#include "halo.h"
#include "tunecache.h"

namespace qb {

// SV: storage type of the colour vectors, SL: storage type of the links
// (double, float or the 16-bit formats tagged __half)
template <typename SV, typename SL>
struct DslashArgs {
    VecView<SV> out;
    VecView<SV> in;
    LinkView<SL> links;
    Geom g;
    int cb;
    // domain decomposition: the input parity's t-slices -3..-1 and Nt..Nt+2
    // of the neighbouring slabs (component stride 3 * g.st, index
    // slice * g.st + face site)
    VecView<SV> gback, gfwd;
};

// Where the Dslash gathers neighbour k of output site s from:
//  * NbGlobal: the input block, every neighbour inside the lattice with
//    periodic wrap;
//  * NbHalo: the same, except that the t direction does not wrap: t - 1,
//    t - 3 below 0 and t + 1, t + 3 at or beyond Nt come from the ghost
//    slices of the neighbouring slabs (domain decomposition);
//  * NbTile: nine (z, t) planes of the input staged in shared memory (the
//    TMA tile variant, k_dslash_tile).
// A z or t hop keeps xh (the parity flip and the odd hop cancel in
// x = 2 xh + ((y+z+t+cb) & 1)).
struct NbGlobal {
    template <typename SV, typename SL, typename A>
    __device__ __forceinline__ void load(const DslashArgs<SV, SL> &a, const SiteCoords &s, int k, A v[6]) const
    {
        a.in.load(neighbor(a.g, s, k), v);
    }
};

struct NbHalo {
    template <typename SV, typename SL, typename A>
    __device__ __forceinline__ void load(const DslashArgs<SV, SL> &a, const SiteCoords &s, int k, A v[6]) const
    {
        if (((k & 7) >> 1) == 3) {
            const int hop = k < 8 ? 1 : 3;
            const int t = s.t + ((k & 1) ? hop : -hop);
            const int face = s.z * a.g.sz + s.y * a.g.sy + s.xh;
            if (t < 0) a.gback.load((t + 3) * a.g.st + face, v);
            else if (t >= a.g.nt) a.gfwd.load((t - a.g.nt) * a.g.st + face, v);
            else a.in.load(t * a.g.st + face, v);
            return;
        }
        a.in.load(neighbor(a.g, s, k), v);
    }
};

// Nine planes of np = Nxh*Ny sites in shared memory, each [3][np] complex:
// slot 0 the output plane's own (z, t), 1/2 z -/+ 1, 3/4 z -/+ 3, 5/6 t -/+ 1,
// 7/8 t -/+ 3.  x and y neighbours stay in slot 0 (their block index minus
// the plane's first index p0); z and t neighbours keep (xh, y).
template <typename SV>
struct NbTile {
    const cx_t<SV> *base;
    int np, p0;
    template <typename SL, typename A>
    __device__ __forceinline__ void load(const DslashArgs<SV, SL> &a, const SiteCoords &s, int k, A v[6]) const
    {
        const int d = (k & 7) >> 1;
        int slot, idx;
        if (d < 2) {
            slot = 0;
            idx = neighbor(a.g, s, k) - p0;
        } else {
            slot = 1 + (d - 2) * 4 + (k >= 8 ? 2 : 0) + (k & 1);
            idx = s.y * a.g.sy + s.xh;
        }
        const cx_t<SV> *q = base + (size_t)slot * 3 * np + idx;
        const cx_t<SV> x0 = q[0], x1 = q[np], x2 = q[2 * np];
        v[0] = x0.x; v[1] = x0.y; v[2] = x1.x; v[3] = x1.y; v[4] = x2.x; v[5] = x2.y;
    }
};

// Neighbour k of output site s: one hop 2*d (backward) / 2*d+1 (forward),
// three hops 8+2*d / 9+2*d (the reference's NeighTable order).
template <typename SV, typename SL, typename A, typename NB = NbGlobal>
__device__ __forceinline__ void dslash_site(const DslashArgs<SV, SL> &a, int j, A acc[6], const NB &nb = NB{})
{
    const SiteCoords s = decode(a.g, a.cb, j);
#pragma unroll
    for (int i = 0; i < 6; ++i) acc[i] = A(0);
    if constexpr (std::is_same<SL, double>::value) {
        // FP64: one matrix and its neighbour per batch (192 bytes in flight)
#pragma unroll
        for (int d = 0; d < 4; ++d) {
#pragma unroll
            for (int sl = 0; sl < 4; ++sl) {
                const int k = (sl < 2 ? 0 : 8) + 2 * d + (sl & 1 ? 0 : 1);
                A u[18], v[6];
                nb.load(a, s, k, v);
                a.links.load_mat(d, sl, j, u);
                if (sl & 1) mv_adj_sub(acc, u, v);
                else mv_add(acc, u, v);
            }
        }
    } else if constexpr (std::is_same<SL, float>::value || std::is_same<SL, Recon12>::value ||
                         std::is_same<SL, Recon13>::value) {
        // FP32: eight stages, the forward/backward pair of fat (h = 0) and of
        // Naik (h = 1) links of each direction: 9 x 16 bytes, or 6 x 16 bytes
        // for compressed Naik links whose third rows are rebuilt from the
        // site's sign bits (12-real) or the links' complex ratios (13-real,
        // one more 16-byte load per direction).  Software-pipelined: the loads
        // of stage i + 1 are issued before the arithmetic of stage i, so every
        // thread keeps one stage of links and neighbours in flight.
        constexpr bool RN = !std::is_same<SL, float>::value;
        unsigned bits = 0;
        if constexpr (RN) bits = a.links.fetch_aux(j);
        float4 c[2][9];
        float4 lam[2];
        A v[2][2][6];
        auto issue = [&](int st, int b) {
            const int d = st >> 1, h = st & 1;
            nb.load(a, s, 8 * h + 2 * d + 1, v[b][0]);
            nb.load(a, s, 8 * h + 2 * d, v[b][1]);
            if constexpr (RN) {
                if (h) {
                    a.links.fetch_naik(d, j, c[b]);
                    if constexpr (LinkView<SL>::has_lam) lam[b] = a.links.fetch_lam(d, j);
                } else {
                    a.links.fetch_fat(d, j, c[b]);
                }
            } else {
                a.links.fetch_pair(d, h, j, c[b]);
            }
        };
        issue(0, 0);
#pragma unroll
        for (int st = 0; st < 8; ++st) {
            const int b = st & 1;
            if (st + 1 < 8) issue(st + 1, b ^ 1);
            A u[36];
            if (RN && (st & 1)) {
                if constexpr (RN) a.links.naik_from(c[b], st >> 1, bits, lam[b], u, u + 18);
            } else {
#pragma unroll
                for (int k = 0; k < 9; ++k) {
                    u[4 * k] = c[b][k].x; u[4 * k + 1] = c[b][k].y;
                    u[4 * k + 2] = c[b][k].z; u[4 * k + 3] = c[b][k].w;
                }
            }
            mv_add(acc, u, v[b][0]);
            mv_adj_sub(acc, u + 18, v[b][1]);
        }
    } else {
        // 16-bit links: the four matrices of a direction, 9 x 16 bytes + 4
        // neighbours per stage, pipelined over the directions like FP32.
        // All fat links share one fixed-point range and all Naik links
        // another, so the fat and Naik terms are summed from the unscaled
        // integers and each sum is scaled once at the end.
        int4 raw[2][9];
        A v[2][4][6];
        A accl[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) accl[i] = A(0);
        auto issue = [&](int d, int b) {
#pragma unroll
            for (int sl = 0; sl < 4; ++sl)
                nb.load(a, s, (sl < 2 ? 0 : 8) + 2 * d + (sl & 1 ? 0 : 1), v[b][sl]);
            a.links.load_quad(d, j, raw[b]);
        };
        issue(0, 0);
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const int b = d & 1;
            if (d + 1 < 4) issue(d + 1, b ^ 1);
#pragma unroll
            for (int sl = 0; sl < 4; ++sl) {
                A u[18];
                a.links.unpack_q(raw[b], sl, u);
                A *t = sl < 2 ? acc : accl;
                if (sl & 1) mv_adj_sub(t, u, v[b][sl]);
                else mv_add(t, u, v[b][sl]);
            }
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) acc[i] = acc[i] * a.links.scale_fat + accl[i] * a.links.scale_long;
    }
}

// blocks of 256 per SM the register allocation must allow.  The pipelined
// kernels keep one stage in flight in 80 registers at 3 blocks/SM.
// 24^3x48 mixed solves: 12-real 100.7 ms (4 blocks: 107.8 ms); 18-real
// 113.9 ms (1 block at 241 registers: 116.7 ms); 16-bit links 93.6 ms (1
// block: 118.1 ms; 4 blocks at 64 registers, no spills in K1: 93.0 against
// 88.0 ms, K2 49.8 against 44.9 us); 16-bit vectors and links 88.7 ms (4
// blocks at 64 registers: 93.0 ms)
template <typename SV, typename SL> struct MinBlocks { static constexpr int value = 1; };
template <> struct MinBlocks<float, float> { static constexpr int value = 3; };
template <> struct MinBlocks<float, Recon12> { static constexpr int value = 3; };
template <> struct MinBlocks<float, Recon13> { static constexpr int value = 3; };
template <> struct MinBlocks<float, __half> { static constexpr int value = 3; };
template <> struct MinBlocks<__half, __half> { static constexpr int value = 3; };

// Scalar step after p.(M^dag M p) is known, run by one warp of the last
// block of the reduction: CG (mode 0) a = -rsq/pkp in lane 0; multi-shift
// (mode 1) the shift recurrences, lane k handling shifts k, k + 32, ...
// (each shift's arithmetic is the sequential one, so the results do not
// depend on the lane split; one thread walking the shifts through device
// memory took ~10 us per iteration at 12 shifts).
// A zero or non-finite p.(M p) is a breakdown (M is positive definite for
// m > 0; the reference divides by it unchecked, ks_d_congrad_fn.cpp:511):
// the step is set to zero, st->error = 2 and the update kernel that follows
// ends the device run, so the host returns QPHIX_FAIL.
struct FinMdagm {
    SolverState *st;
    int mode;
    static constexpr bool kWarp = true;
    __device__ void operator()(const double *t, int lane) const
    {
        const double pkp = t[0];
        int done = 0;
        if (lane == 0) {
            st->pkp = pkp;
            st->iteration += 1;
            if (!(pkp != 0.0) || !isfinite(pkp)) {
                st->error = 2;
                st->a = 0.0;
                done = 1;
            } else if (mode == 0) {
                st->a = round_to(-st->rsq / pkp, st->prec_single);
                done = 1;
            }
        }
        if (__shfl_sync(0xffffffffu, done, 0)) return;
        // multi-shift scalar recurrences (ks_multicg_offset.cpp:475-496);
        // the values of the previous iteration are scrolled first
        // (:617-622), which the reference does at the end of that iteration
        const int single = st->prec_single;
        const int jl = st->j_low;
        const int nn = st->num_now;
        if (!st->first_iter) {
            for (int k = lane; k < nn; k += 32) {
                st->beta_im1[k] = st->beta_i[k];
                st->zeta_im1[k] = st->zeta_i[k];
                st->zeta_i[k] = st->zeta_ip1[k];
            }
        }
        __syncwarp();
        if (lane == 0) {
            st->first_iter = 0;
            st->beta_i[jl] = round_to(-st->rsq / pkp, single);
            st->zeta_ip1[jl] = 1.0;
        }
        __syncwarp();
        const double b_jl = st->beta_i[jl], a_jl = st->alpha[jl], bm1_jl = st->beta_im1[jl];
        for (int k = lane; k < nn; k += 32) {
            if (k == jl) continue;
            const double zi = st->zeta_i[k], zim1 = st->zeta_im1[k];
            double z = round_to(round_to(zi * zim1, single) * bm1_jl, single);
            const double c1 = round_to(round_to(b_jl * a_jl, single) * round_to(zim1 - zi, single), single);
            const double c2 =
                round_to(round_to(zim1 * bm1_jl, single) * (1.0 + round_to(st->shifts[k] * b_jl, single)), single);
            const double den = round_to(c1 + c2, single);
            if (den != 0.0) z = round_to(z / den, single);
            else { z = 0.0; st->finished[k] = 1; }
            st->zeta_ip1[k] = z;
            if (zi != 0.0)
                st->beta_i[k] = round_to(round_to(b_jl * z, single) / zi, single);
            else { st->zeta_ip1[k] = 0.0; st->beta_i[k] = 0.0; st->finished[k] = 1; }
        }
        __syncwarp();
        // the last active shift leaves the recurrence once it has finished
        if (lane == 0 && nn - 1 > jl && st->finished[nn - 1] == 1) st->num_now = nn - 1;
    }
};

template <typename SV, typename SL>
__global__ void __launch_bounds__(kBlock, MinBlocks<SV, SL>::value) k_dslash(DslashArgs<SV, SL> a, const SolverState *st, int gate)
{
    using A = typename Acc<SV>::type;
    if (st && gated_off(st, gate)) return;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < a.g.vh; j += gridDim.x * blockDim.x) {
        A acc[6];
        dslash_site<SV, SL, A>(a, j, acc);
        a.out.store(j, acc);
    }
}

// ttt = D tmp + m4 * p ;  pkp = sum p . ttt  (calc_pkp, ks_d_congrad_fn.cpp:159-171;
// ks_multicg_offset.cpp:107-122), then the scalar step of the solver.
template <typename SV, typename SL>
__global__ void __launch_bounds__(kBlock, MinBlocks<SV, SL>::value)
k_dslash_mdagm(DslashArgs<SV, SL> a, VecView<SV> pv, double m4, SolverState *st, double *partials,
               int gate, int mode)
{
    using A = typename Acc<SV>::type;
    if (gated_off(st, gate)) return;
    double dot[1] = {0.0};
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < a.g.vh; j += gridDim.x * blockDim.x) {
        A acc[6], p[6];
        dslash_site<SV, SL, A>(a, j, acc);
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
    grid_reduce<1>(dot, partials, &st->counter, FinMdagm{st, mode});
}

// ---------------------------------------------------------------------------
// Domain-decomposed Dslash (halo.h): sites of a range of t-slices, the t
// neighbours beyond the slab read from the ghost slices.  Site i of the
// launch is j = i + off_a for i < split, else i + off_b, so one launch
// covers the interior (3 <= t < Nt-3) or both boundary bands (t < 3 and
// t >= Nt-3).  With pv set the M^dag M epilogue out = D in + m4 pv is
// applied (its dot product is reduced by k_dd_dot).
// ---------------------------------------------------------------------------
struct SiteRange {
    int n, split, off_a, off_b;
    __device__ __forceinline__ int site(int i) const { return i < split ? i + off_a : i + off_b; }
};

template <typename SV, typename SL>
__global__ void __launch_bounds__(kBlock, MinBlocks<SV, SL>::value)
k_dslash_dd(DslashArgs<SV, SL> a, SiteRange r, VecView<SV> pv, double m4, const SolverState *st, int gate)
{
    using A = typename Acc<SV>::type;
    if (st && gated_off(st, gate)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < r.n; i += gridDim.x * blockDim.x) {
        const int j = r.site(i);
        A acc[6];
        dslash_site<SV, SL, A>(a, j, acc, NbHalo{});
        if (pv.p) {
            A p[6];
            pv.load_cg(j, p);
            const A m = (A)m4;
#pragma unroll
            for (int k = 0; k < 6; ++k) acc[k] = acc[k] + m * p[k];
        }
        a.out.store(j, acc);
    }
}

// Copies the first and the last three t-slices of a parity block into the
// send buffers (the neighbours' forward and backward ghosts), element by
// element in the storage format (E: double2 / float2 per component, int4
// per 16-bit site; C components).
template <typename E, int C>
__global__ void __launch_bounds__(kBlock)
k_halo_pack(const E *in, E *sback, E *sfwd, int vh, int st, int nt, const SolverState *state, int gate)
{
    if (state && gated_off(state, gate)) return;
    const int n = 3 * st;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int c = 0; c < C; ++c) {
        sback[(size_t)c * n + i] = in[(size_t)c * vh + i];
        sfwd[(size_t)c * n + i] = in[(size_t)c * vh + (size_t)(nt - 3) * st + i];
    }
}

struct FinNothing {
    __device__ void operator()(const double *) const {}
};

// p . ttt of this GPU into st->dd_red[0] (the reduction of the fused kernel
// K2, which the halo path does not fuse), products formed as K2 forms them
template <typename SV>
__global__ void __launch_bounds__(kBlock)
k_dd_dot(VecView<SV> p, VecView<SV> t, SolverState *st, double *partials, int gate)
{
    using A = typename Acc<SV>::type;
    if (gated_off(st, gate)) return;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    double s[1] = {0.0};
    if (j < p.vh) {
        A a[6], b[6];
        p.load_cg(j, a);
        t.load_cg(j, b);
#pragma unroll
        for (int k = 0; k < 6; ++k) s[0] += (double)(a[k] * b[k]);
    }
    grid_reduce<1>(s, partials, &st->counter, FinNothing{}, st);
}

// ---------------------------------------------------------------------------
// TMA-pipelined Dslash.  A persistent CTA owns tiles of T consecutive output
// sites; for each tile it visits the 4 directions in turn.  The link chunks
// of one (tile, direction) -- C runs of T x 16 contiguous bytes in the link
// block -- are brought into shared memory by cp.async.bulk copies issued by
// one thread and completing on an mbarrier; NS such stages are in flight, so
// HBM streaming no longer depends on how many loads a thread keeps in
// registers.  Neighbour vectors are gathered from L2/L1 as in the plain
// kernel.  Every mbarrier wait is bounded: on a timeout the CTA records the
// failure in *err and stops.
// ---------------------------------------------------------------------------
template <typename S> struct TmaCfg;
template <> struct TmaCfg<double> { static constexpr int C = 36, T = 128, NS = 2; };
template <> struct TmaCfg<float> { static constexpr int C = 18, T = 128, NS = 3; };
template <> struct TmaCfg<__half> { static constexpr int C = 9, T = 128, NS = 4; };

constexpr unsigned kDefaultWaitPolls = 1u << 22;  // far longer than any copy takes
constexpr unsigned kDrainPolls = 1u << 22;
// poll limit of the pipeline's waits (QPHIX_B200_set_wait_limit)
static unsigned g_wait_limit = kDefaultWaitPolls;

template <typename S>
constexpr size_t tma_smem_bytes()
{
    return (size_t)TmaCfg<S>::NS * TmaCfg<S>::C * TmaCfg<S>::T * 16 + TmaCfg<S>::NS * sizeof(uint64_t);
}

// contribution of direction d from the staged chunks (chunk q of this
// thread's site at ch[q*T])
template <typename SV, typename SL, typename A>
__device__ __forceinline__ void tma_direction(const DslashArgs<SV, SL> &a, const SiteCoords &s, int d,
                                              const uint4 *ch, A acc[6])
{
    constexpr int T = TmaCfg<SL>::T;
    A v[4][6];
#pragma unroll
    for (int sl = 0; sl < 4; ++sl)
        a.in.load(neighbor(a.g, s, (sl < 2 ? 0 : 8) + 2 * d + (sl & 1 ? 0 : 1)), v[sl]);
    if constexpr (std::is_same<SL, double>::value) {
        const double2 *c2 = reinterpret_cast<const double2 *>(ch);
#pragma unroll
        for (int sl = 0; sl < 4; ++sl) {
            A u[18];
#pragma unroll
            for (int e = 0; e < 9; ++e) {
                const double2 z = c2[(9 * sl + e) * T];
                u[2 * e] = z.x; u[2 * e + 1] = z.y;
            }
            if (sl & 1) mv_adj_sub(acc, u, v[sl]);
            else mv_add(acc, u, v[sl]);
        }
    } else if constexpr (std::is_same<SL, float>::value) {
        const float4 *c4 = reinterpret_cast<const float4 *>(ch);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            A u[36];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                const float4 z = c4[(9 * h + c) * T];
                u[4 * c] = z.x; u[4 * c + 1] = z.y; u[4 * c + 2] = z.z; u[4 * c + 3] = z.w;
            }
            mv_add(acc, u, v[2 * h]);
            mv_adj_sub(acc, u + 18, v[2 * h + 1]);
        }
    } else {
        const int4 *c4 = reinterpret_cast<const int4 *>(ch);
        int4 raw[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) raw[c] = c4[c * T];
#pragma unroll
        for (int sl = 0; sl < 4; ++sl) {
            A u[18];
            a.links.unpack_q(raw, sl, u);
            const A sc = sl < 2 ? a.links.scale_fat : a.links.scale_long;
#pragma unroll
            for (int e = 0; e < 18; ++e) u[e] *= sc;
            if (sl & 1) mv_adj_sub(acc, u, v[sl]);
            else mv_add(acc, u, v[sl]);
        }
    }
}

// MODE 0: out = D in.  MODE 1: out = D in + m4 p, p.out reduced, then the
// solver's scalar step (FinMdagm).
// Every mbarrier wait gives up after `wait_limit` polls.  The CTA then
// stops as a whole (the failure is OR-ed over the CTA at the end of the
// stage), thread 0 waits -- with a generous limit -- for every copy still
// in flight, so nothing lands in shared memory after the CTA has left,
// records the failure in *err and the CTA returns.
template <typename SV, typename SL, int MODE>
__global__ void __launch_bounds__(TmaCfg<SL>::T)
k_dslash_tma(DslashArgs<SV, SL> a, const char *links, VecView<SV> pv, double m4, SolverState *st,
             double *partials, int gate, int mode, int *err, unsigned wait_limit)
{
    using A = typename Acc<SV>::type;
    constexpr int C = TmaCfg<SL>::C, T = TmaCfg<SL>::T, NS = TmaCfg<SL>::NS;
    if (st && gated_off(st, gate)) return;
    extern __shared__ __align__(128) unsigned char smem[];
    uint4 *buf = reinterpret_cast<uint4 *>(smem);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + (size_t)NS * C * T * 16);
    const int tid = threadIdx.x;
    const int vh = a.g.vh;
    const int ntiles = (vh + T - 1) / T;
    const int my_tiles = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const int total = 4 * my_tiles;
    if (tid == 0) {
        for (int b = 0; b < NS; ++b) mbar_init(&bars[b], 1);
        fence_mbar_init();
    }
    __syncthreads();
    const uint64_t policy = policy_evict_first();
    auto issue = [&](int g) {
        const int tile = (int)blockIdx.x + (g >> 2) * (int)gridDim.x;
        const int d = g & 3;
        const int j0 = tile * T;
        const int n = min(T, vh - j0);
        const int b = g % NS;
        mbar_arrive_expect_tx(&bars[b], (uint32_t)(C * n * 16));
#pragma unroll 1
        for (int q = 0; q < C; ++q)
            bulk_g2s(buf + ((size_t)b * C + q) * T, links + ((((size_t)d * C + q) * vh + j0) << 4),
                     (uint32_t)(n * 16), &bars[b], policy);
    };
    if (tid == 0) {
        fence_proxy_async_smem();
        for (int g = 0; g < NS - 1 && g < total; ++g) issue(g);
    }
    double dot[1] = {0.0};
    A acc[6];
    int g = 0;
    bool failed = false;
    for (; g < total; ++g) {
        if (tid == 0 && g + NS - 1 < total) {
            fence_proxy_async_smem();
            issue(g + NS - 1);
        }
        const int tile = (int)blockIdx.x + (g >> 2) * (int)gridDim.x;
        const int d = g & 3;
        const int j = tile * T + tid;
        const int b = g % NS;
        if (d == 0) {
#pragma unroll
            for (int i = 0; i < 6; ++i) acc[i] = A(0);
        }
        const bool ok = mbar_wait_bounded(&bars[b], (uint32_t)((g / NS) & 1), wait_limit);
        if (ok && j < vh) {
            const SiteCoords s = decode(a.g, a.cb, j);
            tma_direction<SV, SL, A>(a, s, d, buf + (size_t)b * C * T + tid, acc);
            if (d == 3) {
                if constexpr (MODE == 0) {
                    a.out.store(j, acc);
                } else {
                    A p[6];
                    pv.load_cg(j, p);
                    const A m = (A)m4;
#pragma unroll
                    for (int i = 0; i < 6; ++i) acc[i] = acc[i] + m * p[i];
                    a.out.store(j, acc);  // acc now holds the stored (rounded) value
#pragma unroll
                    for (int i = 0; i < 6; ++i) dot[0] += (double)(p[i] * acc[i]);
                }
            }
        }
        // the barrier also keeps buffer b alive until every thread is done
        // with it (the next stage's copy into it is issued after this point)
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
    }
    if (failed) {
        if (tid == 0) {
            atomicExch(err, 1);
            // stages g .. g+NS-1 may still be in flight, one per barrier
            const int last = min(g + NS - 1, total - 1);
            for (int s2 = g; s2 <= last; ++s2)
                (void)mbar_wait_bounded(&bars[s2 % NS], (uint32_t)((s2 / NS) & 1), kDrainPolls);
        }
        return;
    }
    if constexpr (MODE == 1)
        grid_reduce<1>(dot, partials, &st->counter, FinMdagm{st, mode});
}

// ---------------------------------------------------------------------------
// TMA neighbour-tile Dslash (variant 3).  A persistent CTA walks the (z, t)
// planes of the output parity (np = Nxh*Ny sites each); for each plane one
// thread issues cp.async.bulk copies of the nine input planes its sites
// gather from -- its own (z, t), z -/+ 1, z -/+ 3, t -/+ 1, t -/+ 3, three
// colour components each, 27 contiguous runs of np complex numbers -- into
// shared memory, completing on an mbarrier; the threads then compute their
// sites with every neighbour read from shared memory and the links streamed
// from global memory as in the register kernel.  The input vectors, the
// data with reuse, thus cross L2 -> SM once per plane (9 x 24 B per site in
// FP32) instead of through per-thread gathers (16 x 24 B).  The wait is
// bounded like the link pipeline's; no copy uses .multicast::cluster.
// ---------------------------------------------------------------------------
constexpr int kTileMaxThreads = 512;

template <typename SV>
__host__ __device__ constexpr size_t tile_smem_bytes(int np)
{
    return (size_t)27 * np * sizeof(cx_t<SV>) + 16;
}

// MODE 0: out = D in.  MODE 1: out = D in + m4 pv, pv.out reduced, then the
// solver's scalar step.
template <typename SV, typename SL, int MODE>
__global__ void __launch_bounds__(kTileMaxThreads)
k_dslash_tile(DslashArgs<SV, SL> a, VecView<SV> pv, double m4, SolverState *st, double *partials, int gate, int mode,
              int *err, unsigned wait_limit)
{
    using A = typename Acc<SV>::type;
    using E = cx_t<SV>;
    if (st && gated_off(st, gate)) return;
    extern __shared__ __align__(128) unsigned char smem[];
    const Geom &g = a.g;
    const int np = g.sz;  // Nxh * Ny
    E *tile = reinterpret_cast<E *>(smem);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + (size_t)27 * np * sizeof(E));
    const int tid = threadIdx.x;
    const int nplanes = g.nz * g.nt;
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    const E *in = a.in.p;
    const uint32_t run = (uint32_t)(np * sizeof(E));
    double dot[1] = {0.0};
    uint32_t phase = 0;
    bool failed = false;
    for (int plane = blockIdx.x; plane < nplanes; plane += gridDim.x) {
        const int z = plane % g.nz, t = plane / g.nz;
        if (tid == 0) {
            // the barrier at the end of the previous plane ordered every read
            // of the tile before this point
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(bar, 27u * run);
#pragma unroll 1
            for (int sl = 0; sl < 9; ++sl) {
                // slot sl: 1/2 z -/+ 1, 3/4 z -/+ 3, 5/6 t -/+ 1, 7/8 t -/+ 3
                const int hop = (sl - 1) % 4 < 2 ? 1 : 3;
                const int step = sl == 0 ? 0 : ((sl & 1) ? -hop : hop);
                const int zs = wrap(z + (sl >= 1 && sl <= 4 ? step : 0), g.nz);
                const int ts = wrap(t + (sl >= 5 ? step : 0), g.nt);
                const size_t p0 = (size_t)(ts * g.nz + zs) * np;
#pragma unroll 1
                for (int c = 0; c < 3; ++c)
                    bulk_g2s(tile + ((size_t)sl * 3 + c) * np, in + (size_t)c * g.vh + p0, run, bar,
                             policy_evict_last());
            }
        }
        const bool ok = mbar_wait_bounded(bar, phase, wait_limit);
        phase ^= 1u;
        if (ok) {
            const NbTile<SV> nb{tile, np, plane * np};
            for (int i = tid; i < np; i += blockDim.x) {
                const int j = plane * np + i;
                A acc[6];
                dslash_site<SV, SL, A>(a, j, acc, nb);
                if constexpr (MODE == 0) {
                    a.out.store(j, acc);
                } else {
                    A p[6];
                    pv.load_cg(j, p);
                    const A m = (A)m4;
#pragma unroll
                    for (int k = 0; k < 6; ++k) acc[k] = acc[k] + m * p[k];
                    a.out.store(j, acc);
#pragma unroll
                    for (int k = 0; k < 6; ++k) dot[0] += (double)(p[k] * acc[k]);
                }
            }
        }
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
    }
    if (failed) {
        if (tid == 0) {
            atomicExch(err, 1);
            // the plane's copies may still be in flight (the phase just waited on)
            (void)mbar_wait_bounded(bar, phase ^ 1u, kDrainPolls);
        }
        return;
    }
    if constexpr (MODE == 1)
        grid_reduce<1>(dot, partials, &st->counter, FinMdagm{st, mode});
}

template <typename SV, typename SL>
static DslashArgs<SV, SL> make_args(const Launch &L, VecBlock out, VecBlock in, const LinkSet &ls, int cb)
{
    DslashArgs<SV, SL> a;
    a.out = view<SV>(out, L.g->vh);
    a.in = view<SV>(in, L.g->vh);
    if constexpr (std::is_same<SL, __half>::value) {
        a.links = LinkView<__half>{static_cast<const int4 *>(ls.blk[cb]), L.g->vh,
                                   ls.link_max[0] / 32767.0f, ls.link_max[1] / 32767.0f};
    } else if constexpr (std::is_same<SL, float>::value) {
        a.links = LinkView<float>{static_cast<const float4 *>(ls.blk[cb]), L.g->vh};
    } else if constexpr (std::is_same<SL, Recon12>::value) {
        a.links = LinkView<Recon12>{{static_cast<const float4 *>(ls.blk[cb]), L.g->vh},
                                    static_cast<const unsigned *>(ls.sign[cb]), ls.recon_scale};
    } else if constexpr (std::is_same<SL, Recon13>::value) {
        a.links = LinkView<Recon13>{{static_cast<const float4 *>(ls.blk[cb]), L.g->vh},
                                    static_cast<const float4 *>(ls.lam[cb])};
    } else {
        a.links = LinkView<double>{static_cast<const double2 *>(ls.blk[cb]), L.g->vh};
    }
    a.g = *L.g;
    a.cb = cb;
    return a;
}

// Grid of the site loops: every block resident at once (no partial last
// wave), each thread striding over the sites.
template <typename K>
static int resident_grid(K kernel, int vh)
{
    static int per_sm = -1, sms = 0;
    if (per_sm < 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, 0) != cudaSuccess || per_sm < 1)
            per_sm = 1;
    }
    const int need = grid_for(vh);
    const int full = per_sm * sms;
    return need < full ? need : full;
}

// grid of the persistent TMA kernel: all CTAs resident
template <typename SV, typename SL, int MODE>
static int tma_grid(int vh)
{
    static int per_sm = -1, sms = 0;
    if (per_sm < 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(k_dslash_tma<SV, SL, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tma_smem_bytes<SL>());
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dslash_tma<SV, SL, MODE>, TmaCfg<SL>::T,
                                                          tma_smem_bytes<SL>()) != cudaSuccess || per_sm < 1)
            per_sm = 1;
    }
    const int ntiles = (vh + TmaCfg<SL>::T - 1) / TmaCfg<SL>::T;
    return ntiles < per_sm * sms ? ntiles : per_sm * sms;
}

// ---------------------------------------------------------------------------
// Kernel variants and the autotuner.
//   0  register streaming, grid of resident blocks striding over the sites
//   1  register streaming, one thread per site (full grid)
//   2  TMA bulk-copy pipeline, persistent CTAs
// The first Dslash of each (precision, volume) times every variant on scratch
// vectors with the caller's links and keeps the fastest; QPHIX_B200_DSLASH=
// plain|full|tma forces one.  The fused M^dag M kernel follows the choice.
// ---------------------------------------------------------------------------
constexpr int kVariants = 4;

// -1: tuned; 0..3 forced (QPHIX_B200_DSLASH at load, QPHIX_B200_set_dslash_variant)
static int g_forced = -2;

static int forced_variant()
{
    if (g_forced == -2) {
        const char *e = std::getenv("QPHIX_B200_DSLASH");
        g_forced = -1;
        if (e && !std::strcmp(e, "plain")) g_forced = 0;
        if (e && !std::strcmp(e, "full")) g_forced = 1;
        if (e && !std::strcmp(e, "tma")) g_forced = 2;
        if (e && !std::strcmp(e, "tile")) g_forced = 3;
    }
    return g_forced;
}

void set_forced_variant(int v)
{
    if (v < -1 || v >= kVariants) throw std::runtime_error("set_dslash_variant: variant must be -1, 0, 1, 2 or 3");
    g_forced = v;
}

void set_wait_limit(long polls)
{
    g_wait_limit = polls < 0 ? kDefaultWaitPolls : (unsigned)std::min<long>(polls, 0x7fffffffL);
}

struct TuneEntry {
    int vh = -1;
    int variant = 0;
    float us[kVariants] = {0, 0, 0, 0};
};
// per (vector precision, link storage: Prec, or 3 / 4 = 12-real / 13-real Naik)
static TuneEntry g_tune[3][5];

template <typename SL>
static int link_slot(Prec pl)
{
    return std::is_same<SL, Recon12>::value ? 3 : std::is_same<SL, Recon13>::value ? 4 : (int)pl;
}

// key of a tuning result in the persistent cache
static std::string tune_key(const char *kernel, int vh, Prec pv, int slot)
{
    return std::string(kernel) + ":" + tune_device_tag() + ":vh" + std::to_string(vh) + ":v" +
           std::to_string((int)pv) + ":l" + std::to_string(slot);
}

// a cached choice for this (kernel, volume, precisions), if the cache has one
static bool tune_from_cache(TuneEntry &t, const std::string &key, int vh)
{
    std::vector<double> v;
    if (!tune_cache_get(key, v) || v.size() != 1 + kVariants) return false;
    const int variant = (int)v[0];
    if (variant < 0 || variant >= kVariants) return false;
    t.vh = vh;
    t.variant = variant;
    for (int i = 0; i < kVariants; ++i) t.us[i] = (float)v[1 + i];
    return true;
}

static void tune_to_cache(const TuneEntry &t, const std::string &key)
{
    tune_cache_put(key, {(double)t.variant, t.us[0], t.us[1], t.us[2], t.us[3]});
}

// the tuner times the pipeline with the default wait limit
struct DefaultWaitLimit {
    unsigned keep;
    DefaultWaitLimit() : keep(g_wait_limit) { g_wait_limit = kDefaultWaitPolls; }
    ~DefaultWaitLimit() { g_wait_limit = keep; }
};

// the TMA pipeline stages 18-real FP32 pairs; compressed Naik links run the
// register variants only
template <typename SL>
constexpr bool has_tma() { return !std::is_same<SL, Recon12>::value && !std::is_same<SL, Recon13>::value; }

// the tile variant stages FP32 or FP64 vectors; nine planes must fit the
// 227 KB of shared memory a CTA may have, beside the kernel's static shared
// memory (the grid reduction's, at most 1 KB)
constexpr size_t kMaxDynSmem = 232448 - 1024;
template <typename SV>
static bool tile_ok(const Geom &g)
{
    if constexpr (std::is_same<SV, float>::value || std::is_same<SV, double>::value)
        return tile_smem_bytes<SV>(g.sz) <= kMaxDynSmem;
    else
        return false;
}

template <typename SV, typename SL>
static bool variant_ok(int v, const Geom &g)
{
    if (v == 2) return has_tma<SL>();
    if (v == 3) return tile_ok<SV>(g);
    return v == 0 || v == 1;
}

// launch shape of the tile variant: one CTA per plane at a time, all CTAs
// resident
struct TileShape {
    int block, grid;
    size_t smem;
};
template <typename SV, typename SL, int MODE>
static TileShape tile_shape(const Geom &g)
{
    TileShape t;
    t.block = std::min(kTileMaxThreads, (g.sz + 31) / 32 * 32);
    t.smem = tile_smem_bytes<SV>(g.sz);
    // the opt-in above 48 KB, for this lattice's planes (static + dynamic
    // shared memory must stay within the per-CTA limit)
    static size_t attr = 0;
    if (t.smem > attr) {
        const cudaError_t e = cudaFuncSetAttribute(k_dslash_tile<SV, SL, MODE>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();  // not sticky; the launch would fail, so report it here
            throw std::runtime_error(std::string("tile Dslash: cudaFuncSetAttribute: ") + cudaGetErrorString(e));
        }
        attr = t.smem;
    }
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dslash_tile<SV, SL, MODE>, t.block, t.smem) !=
            cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    t.grid = std::min(g.nz * g.nt, per_sm * sms);
    return t;
}

template <typename SV, typename SL>
static void launch_variant(int variant, const DslashArgs<SV, SL> &a, const LinkSet &ls, int cb, const Launch &L,
                           const SolverState *st, int gate)
{
    if (variant == 3) {
        if constexpr (std::is_same<SV, float>::value || std::is_same<SV, double>::value) {
            if (tile_ok<SV>(*L.g)) {
                const TileShape ts = tile_shape<SV, SL, 0>(*L.g);
                k_dslash_tile<SV, SL, 0><<<ts.grid, ts.block, ts.smem, L.stream>>>(
                    a, a.out, 0.0, const_cast<SolverState *>(st), nullptr, gate, 0, L.err, g_wait_limit);
                return;
            }
        }
        variant = 1;
    }
    if constexpr (!has_tma<SL>()) {
        if (variant == 2) variant = 1;
    } else if (variant == 2) {
        k_dslash_tma<SV, SL, 0><<<tma_grid<SV, SL, 0>(L.g->vh), TmaCfg<SL>::T, tma_smem_bytes<SL>(), L.stream>>>(
            a, static_cast<const char *>(ls.blk[cb]), a.out, 0.0, const_cast<SolverState *>(st), nullptr, gate, 0,
            L.err, g_wait_limit);
        return;
    }
    if (variant == 1) {
        k_dslash<SV, SL><<<grid_for(L.g->vh), kBlock, 0, L.stream>>>(a, st, gate);
    } else {
        k_dslash<SV, SL><<<resident_grid(k_dslash<SV, SL>, L.g->vh), kBlock, 0, L.stream>>>(a, st, gate);
    }
}

template <typename SV, typename SL>
static int tuned_variant(Prec pv, Prec pl, const Launch &L, const DslashArgs<SV, SL> &a, const LinkSet &ls, int cb)
{
    const int f = forced_variant();
    if (f >= 0) return f;
    TuneEntry &t = g_tune[(int)pv][link_slot<SL>(pl)];
    if (t.vh == L.g->vh) return t.variant;
    const std::string key = tune_key("dslash", L.g->vh, pv, link_slot<SL>(pl));
    if (tune_from_cache(t, key, L.g->vh) && variant_ok<SV, SL>(t.variant, *L.g)) return t.variant;
    DefaultWaitLimit wl;
    // time the variants on scratch vectors so no caller data is touched twice
    const size_t vb = vec_bytes(pv, L.g->vh);
    void *vin = nullptr, *vout = nullptr;
    cudaMallocAsync(&vin, vb, L.stream);
    cudaMallocAsync(&vout, vb, L.stream);
    cudaMemsetAsync(vin, 0, vb, L.stream);
    DslashArgs<SV, SL> s = a;
    s.in = view<SV>(VecBlock{vin}, L.g->vh);
    s.out = view<SV>(VecBlock{vout}, L.g->vh);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int best = 0;
    for (int v = 0; v < kVariants; ++v) {
        t.us[v] = 0.f;
        if (!variant_ok<SV, SL>(v, *L.g)) continue;
        launch_variant<SV, SL>(v, s, ls, cb, L, nullptr, -1);  // warm
        cudaEventRecord(e0, L.stream);
        for (int r = 0; r < 3; ++r) launch_variant<SV, SL>(v, s, ls, cb, L, nullptr, -1);
        cudaEventRecord(e1, L.stream);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        t.us[v] = ms * 1e3f / 3;
        if (t.us[v] < t.us[best]) best = v;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(vin, L.stream);
    cudaFreeAsync(vout, L.stream);
    t.vh = L.g->vh;
    t.variant = best;
    tune_to_cache(t, key);
    return best;
}

static void cuda_check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// element type and components per site of the pack kernel
template <typename SV> struct PackElem { using type = cx_t<SV>; static constexpr int C = 3; };
template <> struct PackElem<__half> { using type = int4; static constexpr int C = 1; };

// The Dslash with the halo (halo.h): pack the input parity's first and last
// three t-slices; with several GPUs send them over NCCL on the
// communication stream while the interior runs; then the boundary bands.
template <typename SV, typename SL>
static void halo_dslash(const Launch &L, DslashArgs<SV, SL> a, VecBlock in, Prec pvp, const SolverState *st,
                        int gate, VecView<SV> pv, double m4)
{
    const Halo &h = *L.halo;
    const Geom &g = *L.g;
    const int pi = (int)pvp;
    a.gback = view<SV>(VecBlock{h.gback[pi]}, 3 * g.st);
    a.gfwd = view<SV>(VecBlock{h.gfwd[pi]}, 3 * g.st);
    using E = typename PackElem<SV>::type;
    k_halo_pack<E, PackElem<SV>::C><<<grid_for(3 * g.st), kBlock, 0, L.stream>>>(
        static_cast<const E *>(in.data), static_cast<E *>(h.sback[pi]), static_cast<E *>(h.sfwd[pi]), g.vh, g.st,
        g.nt, st, gate);
    const bool remote = h.nranks > 1;
    if (remote) {
        cuda_check(cudaEventRecord(h.ev_packed, L.stream), "halo: cudaEventRecord");
        cuda_check(cudaStreamWaitEvent(h.comm_stream, h.ev_packed, 0), "halo: cudaStreamWaitEvent");
        nccl_exchange(h.comm, h.sback[pi], h.sfwd[pi], h.gback[pi], h.gfwd[pi], h.face_bytes[pi], h.prev, h.next,
                      h.comm_stream);
        cuda_check(cudaEventRecord(h.ev_recv, h.comm_stream), "halo: cudaEventRecord");
    }
    auto run = [&](SiteRange r) {
        if (r.n > 0) k_dslash_dd<SV, SL><<<grid_for(r.n), kBlock, 0, L.stream>>>(a, r, pv, m4, st, gate);
    };
    if (g.nt >= 6) {
        const int inner = (g.nt - 6) * g.st;
        run(SiteRange{inner, inner, 3 * g.st, 0});  // 3 <= t < Nt-3: no ghost needed
        if (remote) cuda_check(cudaStreamWaitEvent(L.stream, h.ev_recv, 0), "halo: cudaStreamWaitEvent");
        run(SiteRange{6 * g.st, 3 * g.st, 0, inner});  // t < 3 and t >= Nt-3
    } else {
        if (remote) cuda_check(cudaStreamWaitEvent(L.stream, h.ev_recv, 0), "halo: cudaStreamWaitEvent");
        run(SiteRange{g.vh, g.vh, 0, 0});
    }
}

template <typename SV, typename SL>
static void launch_dslash(const Launch &L, VecBlock out, VecBlock in, const LinkSet &ls, int cb,
                          const SolverState *st, int gate, Prec pv)
{
    auto a = make_args<SV, SL>(L, out, in, ls, cb);
    if (L.halo) {
        halo_dslash<SV, SL>(L, a, in, pv, st, gate, VecView<SV>{}, 0.0);
        return;
    }
    launch_variant<SV, SL>(tuned_variant<SV, SL>(pv, ls.prec, L, a, ls, cb), a, ls, cb, L, st, gate);
}

// storage combinations served: vectors and links in the same precision, and
// FP32 vectors with 16-bit links
#define QB_DISPATCH_VL(pv, ls_, F, ...)                                                          \
    do {                                                                                        \
        const Prec pl_ = (ls_).prec;                                                            \
        if ((ls_).recon) {                                                                      \
            if ((pv) != Prec::Single) throw std::runtime_error("Dslash: compressed links need FP32 vectors"); \
            if ((ls_).recon == 2) F<float, Recon13>(__VA_ARGS__);                               \
            else F<float, Recon12>(__VA_ARGS__);                                                \
        } else if ((pv) == Prec::Double && pl_ == Prec::Double) F<double, double>(__VA_ARGS__); \
        else if ((pv) == Prec::Single && pl_ == Prec::Single) F<float, float>(__VA_ARGS__);     \
        else if ((pv) == Prec::Half && pl_ == Prec::Half) F<__half, __half>(__VA_ARGS__);      \
        else if ((pv) == Prec::Single && pl_ == Prec::Half) F<float, __half>(__VA_ARGS__);      \
        else throw std::runtime_error("Dslash: unsupported vector/link precision pair");       \
    } while (0)

void dslash(Prec p, const Launch &L, VecBlock out, VecBlock in, const LinkSet &ls, int cb)
{
    QB_DISPATCH_VL(p, ls, launch_dslash, L, out, in, ls, cb, nullptr, -1, p);
}

void dslash_gated(Prec p, const Launch &L, VecBlock out, VecBlock in, const LinkSet &ls, int cb,
                  SolverState *st, int gate)
{
    QB_DISPATCH_VL(p, ls, launch_dslash, L, out, in, ls, cb, st, gate, p);
}



template <typename SV, typename SL>
static void launch_mdagm_variant(int variant, const DslashArgs<SV, SL> &a, const LinkSet &ls, VecView<SV> pv,
                                 double m4, int cb, SolverState *st, double *partials, int gate, int mode,
                                 const Launch &L)
{
    if (variant == 3) {
        if constexpr (std::is_same<SV, float>::value || std::is_same<SV, double>::value) {
            if (tile_ok<SV>(*L.g)) {
                const TileShape ts = tile_shape<SV, SL, 1>(*L.g);
                k_dslash_tile<SV, SL, 1><<<ts.grid, ts.block, ts.smem, L.stream>>>(a, pv, m4, st, partials, gate,
                                                                                   mode, L.err, g_wait_limit);
                return;
            }
        }
        variant = 1;
    }
    if constexpr (!has_tma<SL>()) {
        if (variant == 2) variant = 1;
    } else if (variant == 2) {
        k_dslash_tma<SV, SL, 1><<<tma_grid<SV, SL, 1>(L.g->vh), TmaCfg<SL>::T, tma_smem_bytes<SL>(), L.stream>>>(
            a, static_cast<const char *>(ls.blk[cb]), pv, m4, st, partials, gate, mode, L.err, g_wait_limit);
        return;
    }
    if (variant == 1) {
        k_dslash_mdagm<SV, SL><<<grid_for(L.g->vh), kBlock, 0, L.stream>>>(a, pv, m4, st, partials, gate, mode);
    } else {
        k_dslash_mdagm<SV, SL><<<resident_grid(k_dslash_mdagm<SV, SL>, L.g->vh), kBlock, 0, L.stream>>>(
            a, pv, m4, st, partials, gate, mode);
    }
}

// The fused M^dag M kernel (K2) is tuned on its own: its grid-wide reduction
// favours fewer, longer-lived blocks more than the plain Dslash does.
static TuneEntry g_tune_mdagm[3][5];

template <typename SV, typename SL>
static int tuned_variant_mdagm(Prec pv, Prec pl, const Launch &L, const DslashArgs<SV, SL> &a, const LinkSet &ls,
                               int cb)
{
    const int f = forced_variant();
    if (f >= 0) return f;
    TuneEntry &t = g_tune_mdagm[(int)pv][link_slot<SL>(pl)];
    if (t.vh == L.g->vh) return t.variant;
    const std::string key = tune_key("mdagm", L.g->vh, pv, link_slot<SL>(pl));
    if (tune_from_cache(t, key, L.g->vh) && variant_ok<SV, SL>(t.variant, *L.g)) return t.variant;
    DefaultWaitLimit wl;
    // scratch vectors, solver state and partials: no caller data is touched
    const size_t vb = vec_bytes(pv, L.g->vh);
    void *vin = nullptr, *vout = nullptr, *vp = nullptr;
    SolverState *st = nullptr;
    double *part = nullptr;
    cudaMallocAsync(&vin, vb, L.stream);
    cudaMallocAsync(&vout, vb, L.stream);
    cudaMallocAsync(&vp, vb, L.stream);
    cudaMemsetAsync(vin, 0, vb, L.stream);
    cudaMemsetAsync(vp, 0, vb, L.stream);
    cudaMallocAsync(&st, sizeof(SolverState), L.stream);
    cudaMemsetAsync(st, 0, sizeof(SolverState), L.stream);
    cudaMallocAsync(&part, sizeof(double) * 4 * kMaxPartials, L.stream);
    DslashArgs<SV, SL> s = a;
    s.in = view<SV>(VecBlock{vin}, L.g->vh);
    s.out = view<SV>(VecBlock{vout}, L.g->vh);
    const VecView<SV> p = view<SV>(VecBlock{vp}, L.g->vh);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int best = 0;
    for (int v = 0; v < kVariants; ++v) {
        t.us[v] = 0.f;
        if (!variant_ok<SV, SL>(v, *L.g)) continue;
        launch_mdagm_variant<SV, SL>(v, s, ls, p, 0.0, cb, st, part, -1, 0, L);  // warm
        cudaEventRecord(e0, L.stream);
        for (int r = 0; r < 3; ++r) launch_mdagm_variant<SV, SL>(v, s, ls, p, 0.0, cb, st, part, -1, 0, L);
        cudaEventRecord(e1, L.stream);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        t.us[v] = ms * 1e3f / 3;
        if (t.us[v] < t.us[best]) best = v;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (void *q : {vin, vout, vp, (void *)st, (void *)part})
        if (q) cudaFreeAsync(q, L.stream);
    t.vh = L.g->vh;
    t.variant = best;
    tune_to_cache(t, key);
    return best;
}

// kernel 0: the Dslash (K1), 1: the fused M^dag M kernel (K2); slot: link
// storage (Prec, or 3 / 4 for 12-real / 13-real Naik links); us receives
// kVariants timings
int dslash_variant(int kernel, Prec pv, int slot, float us[4])
{
    if (slot < 0 || slot > 4) return -1;
    const TuneEntry &t = (kernel == 0 ? g_tune : g_tune_mdagm)[(int)pv][slot];
    for (int v = 0; v < kVariants; ++v) us[v] = t.us[v];
    if (forced_variant() >= 0) return forced_variant();
    return t.vh < 0 ? -1 : t.variant;
}

template <typename SV, typename SL>
static void launch_mdagm(const Launch &L, VecBlock ttt, VecBlock tmp, const LinkSet &ls,
                         VecBlock pv, double m4, int cb, SolverState *st, double *partials,
                         int gate, int mode, Prec p)
{
    auto a = make_args<SV, SL>(L, ttt, tmp, ls, cb);
    if (L.halo) {
        // ttt = D tmp + m4 p through the halo, then p.ttt summed over the GPUs
        // and the solver's scalar step
        const int vh = L.g->vh;
        halo_dslash<SV, SL>(L, a, tmp, p, st, gate, view<SV>(pv, vh), m4);
        k_dd_dot<SV><<<grid_for(vh), kBlock, 0, L.stream>>>(view<SV>(pv, vh), view<SV>(ttt, vh), st, partials, gate);
        if (L.halo->nranks > 1) nccl_allreduce_sum(L.halo->comm, st->dd_red, 1, L.stream);
        k_dd_fin<1, FinMdagm><<<1, 32, 0, L.stream>>>(st, gate, FinMdagm{st, mode});
        return;
    }
    const int variant = tuned_variant_mdagm<SV, SL>(p, ls.prec, L, a, ls, cb);
    launch_mdagm_variant<SV, SL>(variant, a, ls, view<SV>(pv, L.g->vh), m4, cb, st, partials, gate, mode, L);
}

template <typename SV, typename SL>
static void prepare_impl(Prec pv, const LinkSet &ls, const Launch &L)
{
    VecBlock none{};
    auto a = make_args<SV, SL>(L, none, none, ls, 0);
    (void)tuned_variant<SV, SL>(pv, ls.prec, L, a, ls, 0);
    (void)tuned_variant_mdagm<SV, SL>(pv, ls.prec, L, a, ls, 0);
    (void)resident_grid(k_dslash<SV, SL>, L.g->vh);
    (void)resident_grid(k_dslash_mdagm<SV, SL>, L.g->vh);
    if constexpr (has_tma<SL>()) {
        (void)tma_grid<SV, SL, 0>(L.g->vh);
        (void)tma_grid<SV, SL, 1>(L.g->vh);
    }
    if constexpr (std::is_same<SV, float>::value || std::is_same<SV, double>::value) {
        if (tile_ok<SV>(*L.g)) {
            (void)tile_shape<SV, SL, 0>(*L.g);
            (void)tile_shape<SV, SL, 1>(*L.g);
        }
    }
}

void dslash_prepare(Prec pv, const LinkSet &ls, const Launch &L)
{
    QB_DISPATCH_VL(pv, ls, prepare_impl, pv, ls, L);
}

void dslash_mdagm_dot(Prec p, const Launch &L, VecBlock ttt, VecBlock tmp, const LinkSet &ls,
                      VecBlock pv, double m4, int cb, SolverState *st, double *partials, int gate,
                      int mode)
{
    QB_DISPATCH_VL(p, ls, launch_mdagm, L, ttt, tmp, ls, pv, m4, cb, st, partials, gate, mode, p);
}

// FP64 Dslash and fused M^dag M launches with a fixed kernel variant (one
// thread per site): no autotuning, hence no scratch allocation.  Used by the
// allocation-free entry point.
void dslash_fixed_d(const Launch &L, VecBlock out, VecBlock in, const LinkSet &ls, int cb)
{
    auto a = make_args<double, double>(L, out, in, ls, cb);
    k_dslash<double, double><<<grid_for(L.g->vh), kBlock, 0, L.stream>>>(a, nullptr, -1);
}

void dslash_mdagm_fixed_d(const Launch &L, VecBlock ttt, VecBlock tmp, const LinkSet &ls, VecBlock pv, double m4,
                          int cb, SolverState *st, double *partials)
{
    auto a = make_args<double, double>(L, ttt, tmp, ls, cb);
    k_dslash_mdagm<double, double><<<grid_for(L.g->vh), kBlock, 0, L.stream>>>(a, view<double>(pv, L.g->vh), m4,
                                                                                st, partials, -1, 0);
}

}  // namespace qb
