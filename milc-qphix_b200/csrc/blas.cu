// Solver BLAS kernels (K3, K4, K5): one thread per site, all six reals of
// the site in registers, FP64 reductions finished in the last block.
//
// Reference: the CG BLAS of ks_d_congrad_fn.cpp:62-188 (calc_source_norm,
// calc_rsq, calc_rsq2, calc_pkp, axpy), the multi-shift BLAS of
// ks_multicg_offset.cpp:69-184 (calc_rsq2, update_dest, update_pm) and
// relative_residue (ks_blas_utils_c.cpp:110-149).  The reference accumulates
// in its fptype; here every reduction accumulates in FP64 and the step sizes
// are rounded to the solve precision exactly where the reference assigns
// them to an fptype variable.
#include <climits>
#include <type_traits>

#include "device_common.cuh"
#include "halo.h"

namespace qb {

// ------------------------------------------------------------------ norms --
// Finishing steps of the reductions, as functors so a domain-decomposed
// solve can run them after the sum over GPUs (k_dd_fin).
struct FinNorm2 {
    SolverState *st;
    int which;
    double *out;
    __device__ void operator()(const double *t) const
    {
        if (which == 0) st->source_norm = t[0];
        else if (which == 1) st->rsq = t[0];
        if (out) *out = t[0];
    }
};

template <typename S>
__global__ void __launch_bounds__(kBlock)
k_norm2(VecView<S> v, SolverState *st, double *partials, int which, double *out, SolverState *split)
{
    using A = typename Acc<S>::type;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    double s[1] = {0.0};
    if (j < v.vh) {
        A a[6];
        v.load_cg(j, a);
#pragma unroll
        for (int i = 0; i < 6; ++i) s[0] += (double)(a[i] * a[i]);
    }
    grid_reduce<1>(s, partials, &st->counter2, FinNorm2{st, which, out}, split);
}

// per-site |r|^2/|x|^2 term of relative_residue (ks_blas_utils_c.cpp:110-134)
template <typename A>
__device__ __forceinline__ double relres_term(const A r[6], const A x[6])
{
    double num = 0, den = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        num += (double)(r[i] * r[i]);
        den += (double)(x[i] * x[i]);
    }
    if (num == 0) return 0.0;
    return den == 0 ? 1.0 : num / den;
}

// ---------------------------------------------------------- CG restart --
// calc_rsq (ks_d_congrad_fn.cpp:82-99): ttt += (-m4) x; r = b + ttt; p = r;
// rsq = |r|^2 (+ relative residue sum when requested)
struct FinRestart {
    SolverState *st;
    double *out;
    __device__ void operator()(const double *t) const
    {
        if (out) {
            out[0] = t[0];
        } else {
            st->rsq = t[0];
            st->relrsq = t[1];
        }
    }
};

template <typename S>
__global__ void __launch_bounds__(kBlock)
k_cg_restart(VecView<S> ttt, VecView<S> x, VecView<S> b, VecView<S> r, VecView<S> pv, bool setp,
             SolverState *st, double *partials, bool relres, double *out, SolverState *split)
{
    using A = typename Acc<S>::type;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    double s[2] = {0.0, 0.0};
    if (j < ttt.vh) {
        A t[6], xv[6], bv[6], rv[6];
        ttt.load_cg(j, t);
        x.load_cg(j, xv);
        b.load_cg(j, bv);
        const A m = (A)(-st->msq_x4);
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            t[i] = t[i] + m * xv[i];
            rv[i] = bv[i] + t[i];
        }
        ttt.store(j, t);
        r.store(j, rv);  // rv now holds the stored (rounded) residual
        if (setp) {
            A pc[6];
#pragma unroll
            for (int i = 0; i < 6; ++i) pc[i] = rv[i];
            pv.store(j, pc);
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) s[0] += (double)(rv[i] * rv[i]);
        if (relres) s[1] = relres_term(rv, xv);
    }
    grid_reduce<2>(s, partials, &st->counter2, FinRestart{st, out}, split);
}

// --------------------------------------------------------- CG iteration --
// calc_rsq2 (ks_d_congrad_fn.cpp:131-147): x += a p; r += a ttt; rsq = |r|^2
// followed by the scalar bookkeeping of :543-566 and the completion test at
// the top of the loop (:360-363), evaluated on the device.
// V: sites of the whole lattice (relative_residue divides by the global
// volume, ks_blas_utils_c.cpp:148)
struct FinCgUpdate {
    SolverState *st;
    int gate;
    bool relres;
    double V;
    __device__ void operator()(const double *t) const
    {
        const int single = st->prec_single;
        const double oldrsq = st->rsq;
        const double rsq = t[0];
        st->oldrsq = oldrsq;
        st->rsq = rsq;
        double relrsq = st->relrsq;
        if (relres) relrsq = round_to(sqrt(2.0 * t[1] / V), single);
        st->relrsq = relrsq;
        st->size_r = round_to(rsq, single) / st->source_norm;
        st->size_relr = round_to(relrsq, single);
        st->b = round_to(round_to(rsq, single) / oldrsq, single);
        const bool conv = (st->rsqmin <= 0 || st->rsqmin > st->size_r) &&
                          (st->relrsqmin <= 0 || st->relrsqmin > st->size_relr);
        if (!isfinite(rsq) && !st->error) st->error = 1;  // non-finite residual: breakdown
        if ((st->iteration % st->niter == 0) || conv || st->error || run_guard(st)) stop_run(st, gate);
    }
};

template <typename S>
__global__ void __launch_bounds__(kBlock)
k_cg_update(VecView<S> x, VecView<S> pv, VecView<S> r, VecView<S> ttt, SolverState *st,
            double *partials, int gate, bool relres, double V, SolverState *split)
{
    using A = typename Acc<S>::type;
    if (gated_off(st, gate)) return;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    double s[2] = {0.0, 0.0};
    if (j < x.vh) {
        A xv[6], p[6], rv[6], t[6];
        x.load_cg(j, xv);
        pv.load_cg(j, p);
        r.load_cg(j, rv);
        ttt.load_cg(j, t);
        const A a = (A)st->a;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            xv[i] = xv[i] + a * p[i];
            rv[i] = rv[i] + a * t[i];
        }
        x.store(j, xv);
        r.store(j, rv);
#pragma unroll
        for (int i = 0; i < 6; ++i) s[0] += (double)(rv[i] * rv[i]);
        if (relres) s[1] = relres_term(rv, xv);
    }
    grid_reduce<2>(s, partials, &st->counter, FinCgUpdate{st, gate, relres, V}, split);
}

// axpy (ks_d_congrad_fn.cpp:178-188): p = r + b p
template <typename S>
__global__ void __launch_bounds__(kBlock) k_cg_axpy(VecView<S> r, VecView<S> pv, SolverState *st, int gate)
{
    using A = typename Acc<S>::type;
    if (gated_off(st, gate)) return;
    if (st->skip_axpy) return;  // p update redone by the host after a reliable update
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= r.vh) return;
    A rv[6], p[6];
    r.load_cg(j, rv);
    pv.load_cg(j, p);
    const A b = (A)st->b;
#pragma unroll
    for (int i = 0; i < 6; ++i) p[i] = rv[i] + b * p[i];
    pv.store(j, p);
}

// end of an inner iteration of the mixed CG (one thread): b, and whether
// to stop for a reliable update
__device__ __forceinline__ void mx_finish(SolverState *st, double rsq, int gate, double delta2)
{
    const double oldrsq = st->rsq;
    st->oldrsq = oldrsq;
    st->rsq = rsq;
    st->b = rsq / oldrsq;
    bool stalled = false;
    if (rsq < st->ru_best) {
        st->ru_best = rsq;
        st->ru_best_iter = st->iteration;
    } else if (st->ru_stall_window > 0 && st->iteration - st->ru_best_iter >= st->ru_stall_window) {
        stalled = true;
        st->ru_stalled = 1;
    }
    if (!isfinite(rsq) && !st->error) st->error = 1;  // non-finite residual: breakdown
    const bool ru = (rsq < delta2 * st->rsq_ru) || (rsq <= st->rsqstop) || stalled ||
                    (st->iteration >= st->max_cg) || st->error || run_guard(st);
    if (ru) {
        st->skip_axpy = 1;  // this iteration's p update waits for the true residual
        stop_run(st, gate);
    }
}

struct FinMx {
    SolverState *st;
    int gate;
    double delta2;
    __device__ void operator()(const double *t) const { mx_finish(st, t[0], gate, delta2); }
};

// ------------------------------------------- flat vectorised p / x, r updates --
// In FP32 and FP64 a parity block is one contiguous array of 6 Vh reals
// (component-major), so the element-wise updates of the inner CG need no
// site structure: each thread moves two 16-byte words per vector, half the
// array apart (both halves coalesced), which doubles the bytes in flight of
// the per-site kernels above.  Same arithmetic, element by element.
template <typename R> struct Wide;
template <> struct Wide<float> { using type = float4; static constexpr int n = 4; };
template <> struct Wide<double> { using type = double2; static constexpr int n = 2; };

template <typename R>
__device__ __forceinline__ void wide_get(const typename Wide<R>::type &w, R v[Wide<R>::n]);
template <> __device__ __forceinline__ void wide_get<float>(const float4 &w, float v[4])
{
    v[0] = w.x; v[1] = w.y; v[2] = w.z; v[3] = w.w;
}
template <> __device__ __forceinline__ void wide_get<double>(const double2 &w, double v[2])
{
    v[0] = w.x; v[1] = w.y;
}
__device__ __forceinline__ float4 wide_make(const float v[4]) { return make_float4(v[0], v[1], v[2], v[3]); }
__device__ __forceinline__ double2 wide_make(const double v[2]) { return make_double2(v[0], v[1]); }

// p = r + b p
template <typename R>
__global__ void __launch_bounds__(kBlock) k_axpy_flat(const typename Wide<R>::type *r, typename Wide<R>::type *p,
                                                      long long n, SolverState *st, int gate)
{
    if (gated_off(st, gate)) return;
    if (st->skip_axpy) return;  // p update redone by the host after a reliable update
    constexpr int W = Wide<R>::n;
    const long long half = (n + 1) / 2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const R b = (R)st->b;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const long long i = t + k * half;
        if (t >= half || i >= n) continue;
        R rv[W], pv[W];
        wide_get<R>(__ldcg(r + i), rv);
        wide_get<R>(__ldcg(p + i), pv);
#pragma unroll
        for (int e = 0; e < W; ++e) pv[e] = rv[e] + b * pv[e];
        p[i] = wide_make(pv);
    }
}

// x += a p; r += a ttt; |r|^2 -> the reliable-update decision of k_mx_update
template <typename R>
__global__ void __launch_bounds__(kBlock)
k_mx_update_flat(typename Wide<R>::type *x, const typename Wide<R>::type *p, typename Wide<R>::type *r,
                 const typename Wide<R>::type *ttt, long long n, SolverState *st, double *partials, int gate,
                 double delta2, SolverState *split)
{
    if (gated_off(st, gate)) return;
    constexpr int W = Wide<R>::n;
    const long long half = (n + 1) / 2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const R a = (R)st->a;
    double s[1] = {0.0};
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const long long i = t + k * half;
        if (t >= half || i >= n) continue;
        R xv[W], pv[W], rv[W], tv[W];
        wide_get<R>(__ldcg(x + i), xv);
        wide_get<R>(__ldcg(p + i), pv);
        wide_get<R>(__ldcg(r + i), rv);
        wide_get<R>(__ldcg(ttt + i), tv);
#pragma unroll
        for (int e = 0; e < W; ++e) {
            xv[e] = xv[e] + a * pv[e];
            rv[e] = rv[e] + a * tv[e];
            s[0] += (double)(rv[e] * rv[e]);
        }
        x[i] = wide_make(xv);
        r[i] = wide_make(rv);
    }
    grid_reduce<1>(s, partials, &st->counter, FinMx{st, gate, delta2}, split);
}

// ------------------------------------------------------------ multi-shift --
// calc_rsq2 (ks_multicg_offset.cpp:124-140) + the convergence test (:520)
// + the alpha recurrences (:587-598), evaluated on the device.
struct FinMsResidual {
    SolverState *st;
    int gate;
    // one warp: lane k updates shifts k, k + 32, ... (per-shift arithmetic
    // as in the sequential form)
    static constexpr bool kWarp = true;
    __device__ void operator()(const double *t, int lane) const
    {
        const int single = st->prec_single;
        const double rsq = t[0];
        int done = 0;
        if (lane == 0) {
            const double oldrsq = st->rsq;
            st->oldrsq = oldrsq;
            st->rsq = rsq;
            if (!isfinite(rsq) && !st->error) st->error = 1;  // non-finite residual: breakdown
            if (st->error) {  // (or a zero p.Ap in the Dslash kernel before)
                stop_run(st, gate);
                done = 1;
            } else if (rsq <= st->rsqstop) {
                st->converged = 1;
                stop_run(st, gate);
                done = 1;
            } else {
                st->alpha[st->j_low] = round_to(rsq / oldrsq, single);
            }
        }
        if (__shfl_sync(0xffffffffu, done, 0)) return;
        __syncwarp();
        const int jl = st->j_low;
        const int nn = st->num_now;
        const double a_jl = st->alpha[jl], b_jl = st->beta_i[jl];
        const int it = st->iteration;
        const double stop = st->shift_stop;
        for (int k = lane; k < nn; k += 32) {
            if (k == jl) continue;
            const double zb = round_to(st->zeta_i[k] * b_jl, single);
            if (zb != 0.0)
                st->alpha[k] = round_to(round_to(round_to(a_jl * st->zeta_ip1[k], single) * st->beta_i[k], single) / zb,
                                        single);
            else { st->alpha[k] = 0.0; st->finished[k] = 1; }
            if (stop > 0.0 && st->shift_done_at[k] == INT_MAX) {
                const double z = st->zeta_ip1[k];
                if (z * z * rsq <= stop) st->shift_done_at[k] = it;
            }
        }
        __syncwarp();
        if (lane == 0) {
            // the iteration completes (its vector updates are not gated off);
            // the host then replaces r by the FP64 residual of the base shift
            if (st->ms_delta2 > 0.0 && rsq < st->ms_delta2 * st->rsq_ru) {
                st->ms_ru = 1;
                stop_run(st, gate);
            }
            // deferred shift updates: this iteration takes the segment's last slot
            if (st->ms_seg_cap > 0 && st->iteration - st->ms_seg_start >= st->ms_seg_cap) {
                st->ms_seg_full = 1;
                stop_run(st, gate);
            }
            if (st->iteration >= st->max_cg || run_guard(st)) stop_run(st, gate);
        }
    }
};

template <typename S>
__global__ void __launch_bounds__(kBlock)
k_ms_residual(VecView<S> r, VecView<S> ttt, SolverState *st, double *partials, int gate, SolverState *split)
{
    using A = typename Acc<S>::type;
    if (gated_off(st, gate)) return;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    double s[1] = {0.0};
    if (j < r.vh) {
        A rv[6], t[6];
        r.load_cg(j, rv);
        ttt.load_cg(j, t);
        const A bl = (A)st->beta_i[st->j_low];
#pragma unroll
        for (int i = 0; i < 6; ++i) rv[i] = rv[i] + bl * t[i];
        r.store(j, rv);
#pragma unroll
        for (int i = 0; i < 6; ++i) s[0] += (double)(rv[i] * rv[i]);
    }
    grid_reduce<1>(s, partials, &st->counter, FinMsResidual{st, gate}, split);
}

// update_pm / update_dest (ks_multicg_offset.cpp:142-184) for every active
// shift in one pass over the sites: r is read once, x_j and p_j once each.
template <typename S, typename X>
__global__ void __launch_bounds__(kBlock)
k_ms_update(VecBlock *xs, VecBlock *ps, VecView<S> r, int n, SolverState *st, int gate)
{
    using A = typename Acc<S>::type;
    using AX = typename Acc<X>::type;
    if (gated_off(st, gate)) return;
    __shared__ double sb[kMaxShifts], sz[kMaxShifts], sa[kMaxShifts];
    __shared__ int sd[kMaxShifts];
    const int nn = st->num_now;
    const bool conv = st->converged;
    const int it = st->iteration;
    for (int k = threadIdx.x; k < nn; k += blockDim.x) {
        sb[k] = st->beta_i[k];
        sz[k] = st->zeta_ip1[k];
        sa[k] = st->alpha[k];
        sd[k] = st->shift_done_at[k];
    }
    __syncthreads();
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= r.vh) return;
    A rv[6];
    if (!conv) r.load_cg(j, rv);
    for (int k = 0; k < nn; ++k) {
        // a shift that reached its sloppy tolerance gets its last x update in
        // that iteration and is left alone afterwards
        if (sd[k] < it) continue;
        VecView<S> pk = view<S>(ps[k], r.vh);
        VecView<X> xk = view<X>(xs[k], r.vh);
        A p[6];
        AX xv[6];
        pk.load_cg(j, p);
        xk.load_cg(j, xv);
        const AX bk = (AX)sb[k];
#pragma unroll
        for (int i = 0; i < 6; ++i) xv[i] = xv[i] + bk * (AX)p[i];
        xk.store(j, xv);
        if (!conv && sd[k] != it) {
            const A ak = (A)sa[k];
            const double zk = sz[k];
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                const A tt = (A)((double)rv[i] * zk);
                p[i] = tt + ak * p[i];
            }
            pk.store(j, p);
        }
    }
}

// ------------------------------------ multi-shift, deferred shift updates --
// The shifted directions and solutions are linear combinations of the base
// residuals: p_k(t+1) = z_k r(t+1) + a_k p_k(t), x_k += b_k p_k(t).  Instead
// of updating 2n vectors every iteration, an iteration stores its residual
// (the vector the updates would read) and the scalars they would use;
// k_ms_coef expands the recurrences into coefficients and k_ms_flush applies
// them once per segment in FP64, so a segment rounds p_k once instead of
// every iteration.  The base direction is the Dslash input and is updated here,
// with the arithmetic of k_ms_update (its iterations are unchanged).
__global__ void __launch_bounds__(kBlock)
k_ms_defer(VecView<float> p_low, VecView<float> r, float2 *hist, MsHistEntry *hs, int n, SolverState *st, int gate)
{
    if (gated_off(st, gate)) return;
    const int it = st->iteration;
    const bool conv = st->converged;
    const int slot = it - st->ms_seg_start - 1;
    // the stop test of the residual kernel keeps slot < ms_seg_cap; a slot
    // outside the buffer is reported and not written
    if (slot < 0 || slot >= st->ms_seg_cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            st->error = 3;
            stop_run(st, gate);
        }
        return;
    }
    const int jl = st->j_low;
    const int nn = st->num_now;
    if (blockIdx.x == 0) {
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            MsHistEntry e;
            e.b = st->beta_i[k];
            e.a = st->alpha[k];
            e.z = st->zeta_ip1[k];
            const int sd = st->shift_done_at[k];
            e.upd = k >= nn || sd < it ? 0 : (1 | (!conv && sd != it ? 2 : 0));
            hs[(size_t)slot * n + k] = e;
        }
    }
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= r.vh) return;
    float rv[6];
    r.load_cg(j, rv);
    VecView<float> h{hist + (size_t)slot * 3 * r.vh, r.vh};
    h.store(j, rv);
    if (!conv) {
        float p[6];
        p_low.load_cg(j, p);
        const float ak = (float)st->alpha[jl];
        const double zk = st->zeta_ip1[jl];
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            const float tt = (float)((double)rv[i] * zk);
            p[i] = tt + ak * p[i];
        }
        p_low.store(j, p);
    }
}

// The coefficients of a segment's expansion, on the device (one block per
// shift, no host round trip).  With p(t) = P_t p(0) + sum_{u<t} D_t[u] r(u),
//   t-th update:  x += b_t p(t) (upd bit 0);  p(t+1) = z_t r(t) + a_t p(t) (bit 1)
// the column u of D and CX = sum_t b_t D_t[u] depends only on the entries
// t >= u, so thread u computes it alone; thread 0 adds the scalars
// GX = sum_t b_t P_t, P = P_m and the shift's job word (shift | x << 16 |
// p << 17; the base direction is kept by the iterations, not rebuilt).
__global__ void __launch_bounds__(kBlock)
k_ms_coef(const MsHistEntry *hs, int m, int n, int j_low, double *coef, int *jobs)
{
    const int s = blockIdx.x;
    double *c = coef + (size_t)s * 2 * (m + 1);
    for (int u = threadIdx.x; u < m; u += blockDim.x) {
        double D = 0.0, CX = 0.0;
        for (int t = u; t < m; ++t) {
            const MsHistEntry e = hs[(size_t)t * n + s];
            if (t == u) {
                if (e.upd & 2) D = e.z;
            } else {
                if (e.upd & 1) CX = fma(e.b, D, CX);
                if (e.upd & 2) D *= e.a;
            }
        }
        c[2 + 2 * u] = CX;
        c[3 + 2 * u] = D;
    }
    if (threadIdx.x == 0) {
        double P = 1.0, GX = 0.0;
        int any = 0;
        for (int t = 0; t < m; ++t) {
            const MsHistEntry e = hs[(size_t)t * n + s];
            if (e.upd & 1) GX = fma(e.b, P, GX);
            if (e.upd & 2) P *= e.a;
            any |= e.upd;
        }
        c[0] = GX;
        c[1] = P;
        jobs[s] = s | ((any & 1) << 16) | ((any & 2) && s != j_low ? 1 << 17 : 0);
    }
}

// One thread per complex number of the parity block and kFlushJobs jobs;
// the job groups of a range of numbers are adjacent blocks, so the stored
// residuals come from DRAM once per flush and from L2 for the other
// groups.  FP64 accumulation, kFlushDepth slots loaded ahead of their
// arithmetic (about 48 KB in flight per SM at three blocks per SM).
// Coefficients per job: {GX, P, (CX[t], D[t])...}, one uniform 16-byte load
// per slot and job.
constexpr int kFlushJobs = 4;
constexpr int kFlushDepth = 8;
__global__ void __launch_bounds__(kBlock, 3)
k_ms_flush(const float2 *hist, int m, const double *coef, const int *jobs, int njobs, VecBlock *xs,
           const VecBlock *p0s, VecBlock *ps, int n3)
{
    const int groups = (njobs + kFlushJobs - 1) / kFlushJobs;
    const int k0 = (int)(blockIdx.x % groups) * kFlushJobs;
    const int e = (int)(blockIdx.x / groups) * kBlock + threadIdx.x;
    if (e >= n3) return;
    const int nj = min(kFlushJobs, njobs - k0);
    const int stride = 2 * (m + 1);
    const double2 *cf = reinterpret_cast<const double2 *>(coef + (size_t)k0 * stride);
    const int cstride = m + 1;  // in double2
    // jobs without an update in the segment (finished shifts) are skipped
    bool live[kFlushJobs];
    bool any = false;
#pragma unroll
    for (int q = 0; q < kFlushJobs; ++q) {
        live[q] = q < nj && (jobs[k0 + q] >> 16 & 3) != 0;
        any |= live[q];
    }
    if (!any) return;
    double ax[kFlushJobs][2], ap[kFlushJobs][2];
#pragma unroll
    for (int q = 0; q < kFlushJobs; ++q) {
        ax[q][0] = ax[q][1] = ap[q][0] = ap[q][1] = 0.0;
        if (live[q]) {
            const int s = jobs[k0 + q] & 0xffff;
            const float2 p0 = static_cast<const float2 *>(p0s[s].data)[e];
            const double2 g = __ldg(cf + q * cstride);
            ax[q][0] = g.x * p0.x;
            ax[q][1] = g.x * p0.y;
            ap[q][0] = g.y * p0.x;
            ap[q][1] = g.y * p0.y;
        }
    }
    auto step = [&](int t, float2 hv) {
#pragma unroll
        for (int q = 0; q < kFlushJobs; ++q) {
            if (live[q]) {
                const double2 cc = __ldg(cf + q * cstride + 1 + t);
                ax[q][0] = fma(cc.x, (double)hv.x, ax[q][0]);
                ax[q][1] = fma(cc.x, (double)hv.y, ax[q][1]);
                ap[q][0] = fma(cc.y, (double)hv.x, ap[q][0]);
                ap[q][1] = fma(cc.y, (double)hv.y, ap[q][1]);
            }
        }
    };
    int t = 0;
    for (; t + kFlushDepth <= m; t += kFlushDepth) {
        float2 hv[kFlushDepth];
#pragma unroll
        for (int u = 0; u < kFlushDepth; ++u) hv[u] = __ldg(hist + (size_t)(t + u) * n3 + e);
#pragma unroll
        for (int u = 0; u < kFlushDepth; ++u) step(t + u, hv[u]);
    }
    for (; t < m; ++t) step(t, __ldg(hist + (size_t)t * n3 + e));
#pragma unroll
    for (int q = 0; q < kFlushJobs; ++q) {
        if (!live[q]) continue;
        const int jb = jobs[k0 + q];
        const int s = jb & 0xffff;
        if (jb >> 16 & 1) {
            double2 *x = static_cast<double2 *>(xs[s].data) + e;
            const double2 xv = *x;
            *x = make_double2(xv.x + ax[q][0], xv.y + ax[q][1]);
        }
        if (jb >> 17 & 1) static_cast<float2 *>(ps[s].data)[e] = make_float2((float)ap[q][0], (float)ap[q][1]);
    }
}

// ------------------------------------------------- mixed-precision inner CG --
// x_s += a p; r_s += a ttt; rsq = |r_s|^2; b = rsq/oldrsq; request a
// reliable update when |r_s|^2 < delta^2 |r_RU|^2 or the sloppy residual
// passes the target.  The request cancels this iteration's p update, which the
// host redoes with the true residual.

// SX: storage of x_s (FP32 when the other vectors are 16-bit: a 16-bit
// partial solution would round every update to the site's 15-bit range)
template <typename SX, typename S>
__global__ void __launch_bounds__(kBlock)
k_mx_update(VecView<SX> x, VecView<S> pv, VecView<S> r, VecView<S> ttt, SolverState *st,
            double *partials, int gate, double delta2, SolverState *split)
{
    using A = typename Acc<S>::type;
    if (gated_off(st, gate)) return;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    double s[1] = {0.0};
    if (j < x.vh) {
        A xv[6], p[6], rv[6], t[6];
        x.load_cg(j, xv);
        pv.load_cg(j, p);
        r.load_cg(j, rv);
        ttt.load_cg(j, t);
        const A a = (A)st->a;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            xv[i] = xv[i] + a * p[i];
            rv[i] = rv[i] + a * t[i];
        }
        x.store(j, xv);
        r.store(j, rv);
#pragma unroll
        for (int i = 0; i < 6; ++i) s[0] += (double)(rv[i] * rv[i]);
    }
    grid_reduce<1>(s, partials, &st->counter, FinMx{st, gate, delta2}, split);
}

// -------------------------------------------------------------- elementwise --
template <typename D, typename S>
__global__ void __launch_bounds__(kBlock) k_copy(VecView<D> d, VecView<S> s)
{
    using AD = typename Acc<D>::type;
    using AS = typename Acc<S>::type;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= d.vh) return;
    AS a[6];
    AD b[6];
    s.load_cg(j, a);
#pragma unroll
    for (int i = 0; i < 6; ++i) b[i] = (AD)a[i];
    d.store(j, b);
}

template <typename Y, typename X>
__global__ void __launch_bounds__(kBlock) k_add(VecView<Y> y, VecView<X> x)
{
    using AY = typename Acc<Y>::type;
    using AX = typename Acc<X>::type;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= y.vh) return;
    AX a[6];
    AY b[6];
    x.load_cg(j, a);
    y.load_cg(j, b);
#pragma unroll
    for (int i = 0; i < 6; ++i) b[i] = b[i] + (AY)a[i];
    y.store(j, b);
}

// --------------------------------------------------------------- dispatch --
// A domain-decomposed solve (L.halo set) splits every reduction: the
// reducing kernel leaves this GPU's totals in st->dd_red, they are summed
// over the GPUs in place (one ncclAllReduce; nothing with one GPU), and a
// one-thread kernel takes the finishing step.
inline SolverState *split_of(const Launch &L, SolverState *st) { return L.halo ? st : nullptr; }

template <int NV, typename Fin>
void dd_finish(const Launch &L, SolverState *st, int gate, Fin fin)
{
    if (!L.halo) return;
    if (L.halo->nranks > 1) nccl_allreduce_sum(L.halo->comm, st->dd_red, NV, L.stream);
    k_dd_fin<NV, Fin><<<1, 32, 0, L.stream>>>(st, gate, fin);
}

// sites of the whole lattice (all GPUs)
inline double global_sites(const Launch &L) { return L.halo ? (double)L.halo->global_sites : 2.0 * L.g->vh; }

#define QB_DISPATCH(p, F, ...)                               \
    switch (p) {                                             \
    case Prec::Double: F<double>(__VA_ARGS__); break;        \
    case Prec::Single: F<float>(__VA_ARGS__); break;         \
    case Prec::Half: F<__half>(__VA_ARGS__); break;          \
    }

template <typename S>
static void norm2_impl(const Launch &L, VecBlock v, SolverState *st, double *partials, int which, double *out)
{
    k_norm2<S><<<grid_for(L.g->vh), kBlock, 0, L.stream>>>(view<S>(v, L.g->vh), st, partials, which, out,
                                                          split_of(L, st));
    dd_finish<1>(L, st, -1, FinNorm2{st, which, out});
}

void norm2_to_state(Prec p, const Launch &L, VecBlock v, SolverState *st, double *partials, int which)
{
    QB_DISPATCH(p, norm2_impl, L, v, st, partials, which, nullptr);
}

template <typename S>
static void restart_impl(const Launch &L, VecBlock ttt, VecBlock x, VecBlock b, VecBlock r,
                         VecBlock pv, bool setp, SolverState *st, double *partials, bool relres,
                         double *out)
{
    const int vh = L.g->vh;
    k_cg_restart<S><<<grid_for(vh), kBlock, 0, L.stream>>>(view<S>(ttt, vh), view<S>(x, vh), view<S>(b, vh),
                                                           view<S>(r, vh), view<S>(pv, vh), setp, st,
                                                           partials, relres, out, split_of(L, st));
    dd_finish<2>(L, st, -1, FinRestart{st, out});
}

void cg_restart_residual(Prec p, const Launch &L, VecBlock ttt, VecBlock x, VecBlock b, VecBlock r,
                         VecBlock pv, SolverState *st, double *partials, bool relres)
{
    QB_DISPATCH(p, restart_impl, L, ttt, x, b, r, pv, true, st, partials, relres, nullptr);
}

template <typename S>
static void update_impl(const Launch &L, VecBlock x, VecBlock pv, VecBlock r, VecBlock ttt,
                        SolverState *st, double *partials, int gate, bool relres)
{
    const int vh = L.g->vh;
    const double V = global_sites(L);
    k_cg_update<S><<<grid_for(vh), kBlock, 0, L.stream>>>(view<S>(x, vh), view<S>(pv, vh), view<S>(r, vh),
                                                          view<S>(ttt, vh), st, partials, gate, relres, V,
                                                          split_of(L, st));
    dd_finish<2>(L, st, gate, FinCgUpdate{st, gate, relres, V});
}

void cg_update(Prec p, const Launch &L, VecBlock x, VecBlock pv, VecBlock r, VecBlock ttt,
               SolverState *st, double *partials, int gate, bool relres)
{
    QB_DISPATCH(p, update_impl, L, x, pv, r, ttt, st, partials, gate, relres);
}

template <typename S>
static void axpy_impl(const Launch &L, VecBlock r, VecBlock pv, SolverState *st, int gate)
{
    const int vh = L.g->vh;
    if constexpr (std::is_same<S, __half>::value) {
        k_cg_axpy<S><<<grid_for(vh), kBlock, 0, L.stream>>>(view<S>(r, vh), view<S>(pv, vh), st, gate);
    } else {
        using V = typename Wide<S>::type;
        const long long n = 6LL * vh / Wide<S>::n;
        const int grid = (int)(((n + 1) / 2 + kBlock - 1) / kBlock);
        k_axpy_flat<S><<<grid, kBlock, 0, L.stream>>>(static_cast<const V *>(r.data), static_cast<V *>(pv.data), n,
                                                      st, gate);
    }
}

void cg_axpy(Prec p, const Launch &L, VecBlock r, VecBlock pv, SolverState *st, int gate)
{
    QB_DISPATCH(p, axpy_impl, L, r, pv, st, gate);
}

template <typename S>
static void msres_impl(const Launch &L, VecBlock r, VecBlock ttt, SolverState *st, double *partials, int gate)
{
    const int vh = L.g->vh;
    k_ms_residual<S><<<grid_for(vh), kBlock, 0, L.stream>>>(view<S>(r, vh), view<S>(ttt, vh), st, partials, gate,
                                                            split_of(L, st));
    dd_finish<1>(L, st, gate, FinMsResidual{st, gate});
}

void ms_residual(Prec p, const Launch &L, VecBlock r, VecBlock ttt, SolverState *st, double *partials, int gate)
{
    QB_DISPATCH(p, msres_impl, L, r, ttt, st, partials, gate);
}

void ms_update(Prec p, const Launch &L, Prec xprec, VecBlock *x, VecBlock *pv, VecBlock r, int n,
               SolverState *st, int gate)
{
    const int vh = L.g->vh;
    const int grid = grid_for(vh);
    if (xprec == Prec::Double && p == Prec::Double)
        k_ms_update<double, double><<<grid, kBlock, 0, L.stream>>>(x, pv, view<double>(r, vh), n, st, gate);
    else if (xprec == Prec::Double && p == Prec::Single)
        k_ms_update<float, double><<<grid, kBlock, 0, L.stream>>>(x, pv, view<float>(r, vh), n, st, gate);
    else if (xprec == Prec::Double && p == Prec::Half)
        k_ms_update<__half, double><<<grid, kBlock, 0, L.stream>>>(x, pv, view<__half>(r, vh), n, st, gate);
    else if (xprec == Prec::Single && p == Prec::Single)
        k_ms_update<float, float><<<grid, kBlock, 0, L.stream>>>(x, pv, view<float>(r, vh), n, st, gate);
    else if (xprec == Prec::Single && p == Prec::Half)
        k_ms_update<__half, float><<<grid, kBlock, 0, L.stream>>>(x, pv, view<__half>(r, vh), n, st, gate);
}

void ms_defer(const Launch &L, VecBlock p_low, VecBlock r, VecBlock hist, MsHistEntry *hist_s, int n,
              SolverState *st, int gate)
{
    const int vh = L.g->vh;
    k_ms_defer<<<grid_for(vh), kBlock, 0, L.stream>>>(view<float>(p_low, vh), view<float>(r, vh),
                                                       static_cast<float2 *>(hist.data), hist_s, n, st, gate);
}

void ms_coef(const Launch &L, const MsHistEntry *hist_s, int m, int n, int j_low, double *coef, int *jobs)
{
    k_ms_coef<<<n, kBlock, 0, L.stream>>>(hist_s, m, n, j_low, coef, jobs);
}

void ms_flush(const Launch &L, VecBlock hist, int m, const double *coef, const int *jobs, int njobs,
              VecBlock *x, const VecBlock *p0, VecBlock *p)
{
    const int n3 = 3 * L.g->vh;
    const unsigned groups = (njobs + kFlushJobs - 1) / kFlushJobs;
    const unsigned grid = groups * (unsigned)grid_for(n3);
    k_ms_flush<<<grid, kBlock, 0, L.stream>>>(static_cast<const float2 *>(hist.data), m, coef, jobs, njobs, x, p0,
                                              p, n3);
}

template <typename S>
static void mx_impl(const Launch &L, VecBlock x, VecBlock pv, VecBlock r, VecBlock ttt, SolverState *st,
                    double *partials, int gate, double delta2)
{
    const int vh = L.g->vh;
    if constexpr (std::is_same<S, __half>::value) {
        k_mx_update<float, S><<<grid_for(vh), kBlock, 0, L.stream>>>(view<float>(x, vh), view<S>(pv, vh),
                                                                     view<S>(r, vh), view<S>(ttt, vh), st,
                                                                     partials, gate, delta2, split_of(L, st));
    } else {
        using V = typename Wide<S>::type;
        const long long n = 6LL * vh / Wide<S>::n;
        const int grid = (int)(((n + 1) / 2 + kBlock - 1) / kBlock);
        k_mx_update_flat<S><<<grid, kBlock, 0, L.stream>>>(static_cast<V *>(x.data), static_cast<const V *>(pv.data),
                                                           static_cast<V *>(r.data), static_cast<const V *>(ttt.data),
                                                           n, st, partials, gate, delta2, split_of(L, st));
    }
    dd_finish<1>(L, st, gate, FinMx{st, gate, delta2});
}

void mx_update(Prec p, const Launch &L, VecBlock x, VecBlock pv, VecBlock r, VecBlock ttt,
               SolverState *st, double *partials, int gate, double delta2)
{
    QB_DISPATCH(p, mx_impl, L, x, pv, r, ttt, st, partials, gate, delta2);
}

template <typename D, typename S>
static void copy2(const Launch &L, VecBlock d, VecBlock s)
{
    const int vh = L.g->vh;
    k_copy<D, S><<<grid_for(vh), kBlock, 0, L.stream>>>(view<D>(d, vh), view<S>(s, vh));
}

template <typename D>
static void copy1(const Launch &L, VecBlock d, Prec sp, VecBlock s)
{
    switch (sp) {
    case Prec::Double: copy2<D, double>(L, d, s); break;
    case Prec::Single: copy2<D, float>(L, d, s); break;
    case Prec::Half: copy2<D, __half>(L, d, s); break;
    }
}

void vec_copy(Prec dst_p, VecBlock dst, Prec src_p, VecBlock src, const Launch &L)
{
    QB_DISPATCH(dst_p, copy1, L, dst, src_p, src);
}

void vec_zero(Prec p, VecBlock v, const Launch &L)
{
    cudaMemsetAsync(v.data, 0, vec_bytes(p, L.g->vh), L.stream);
}

template <typename Y, typename X>
static void add2(const Launch &L, VecBlock y, VecBlock x)
{
    const int vh = L.g->vh;
    k_add<Y, X><<<grid_for(vh), kBlock, 0, L.stream>>>(view<Y>(y, vh), view<X>(x, vh));
}

template <typename Y>
static void add1(const Launch &L, VecBlock y, Prec xp, VecBlock x)
{
    switch (xp) {
    case Prec::Double: add2<Y, double>(L, y, x); break;
    case Prec::Single: add2<Y, float>(L, y, x); break;
    case Prec::Half: add2<Y, __half>(L, y, x); break;
    }
}

void vec_add(Prec yp, VecBlock y, Prec xp, VecBlock x, const Launch &L)
{
    QB_DISPATCH(yp, add1, L, y, xp, x);
}

void cg_true_residual(Prec p, const Launch &L, VecBlock ttt, VecBlock x, VecBlock b, VecBlock r,
                      SolverState *st, double *partials, double *out)
{
    QB_DISPATCH(p, restart_impl, L, ttt, x, b, r, r, false, st, partials, false, out);
}

void norm2_dev(Prec p, const Launch &L, VecBlock v, SolverState *st, double *partials, double *out)
{
    QB_DISPATCH(p, norm2_impl, L, v, st, partials, 2, out);
}

}  // namespace qb
