// Solver drivers: CG and multi-shift CG with the reference's control flow,
// and their mixed-precision counterparts.
//
// The iteration bodies run as device kernels with every scalar (rsq, pkp,
// a, b, the shift recurrences) kept in a device-resident SolverState; the
// host enqueues chunks of iterations and reads the state once per chunk.
// Each kernel of iteration k of a chunk returns immediately when an earlier
// iteration of the chunk already met the stop condition (k > stop_at), so a
// chunk that overshoots costs a few empty launches, never extra arithmetic,
// and the sequence of arithmetic is exactly the reference's.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>

#include "context.h"
#include "device_common.cuh"

namespace qb {

namespace {

struct Ws {
    std::vector<VecBlock> v;
    std::vector<Prec> p;
    VecBlock get(Prec prec)
    {
        v.push_back(alloc_vec(prec));
        p.push_back(prec);
        return v.back();
    }
    ~Ws()
    {
        for (auto &b : v) free_vec(b);
    }
};

inline double round_prec(double v, bool single) { return single ? (double)(float)v : v; }

// |v|^2 with a wait
double norm2_sync(Prec p, VecBlock v)
{
    Context &c = ctx();
    const Launch L = c.launch();
    norm2_dev(p, L, v, c.d_state, c.d_partials, c.d_scalars);
    QB_CUDA(cudaMemcpyAsync(c.h_scalars, c.d_scalars, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    sync_check();
    return c.h_scalars[0];
}

// Event-timed launch brackets (kernel timing mode).  Marks are kept for the
// whole solve and read once at the end, so timing adds nothing to the
// host's critical path between chunks; launches whose gate was cancelled
// (k > stop_at of their chunk) are not credited.
struct TimedLaunches {
    struct Mark { int kind; int gate; int chunk; cudaEvent_t a, b; };
    std::vector<Mark> marks;
    std::vector<int> stop_of_chunk;
    bool on;
    explicit TimedLaunches(bool enabled) : on(enabled) { ctx().ktimer.reset(); }
    ~TimedLaunches()
    {
        try { finish(); } catch (...) {}
    }
    template <typename F> void run(int kind, int gate, F f)
    {
        if (!on) { f(); return; }
        Context &c = ctx();
        cudaEvent_t a = c.ktimer.next(), b = c.ktimer.next();
        QB_CUDA(cudaEventRecord(a, c.stream));
        f();
        QB_CUDA(cudaEventRecord(b, c.stream));
        marks.push_back({kind, gate, (int)stop_of_chunk.size(), a, b});
    }
    // end of a chunk whose device stop index is stop_at (INT_MAX: none)
    void collect(int stop_at)
    {
        if (on) stop_of_chunk.push_back(stop_at);
    }
    void finish()
    {
        if (!on) return;
        Context &c = ctx();
        for (auto &m : marks) {
            const int stop = m.chunk < (int)stop_of_chunk.size() ? stop_of_chunk[m.chunk] : INT_MAX;
            if (m.gate >= 0 && m.gate > stop) continue;
            float ms = 0;
            if (cudaEventElapsedTime(&ms, m.a, m.b) != cudaSuccess) continue;
            if (m.kind == 0) { c.stats.dslash_launches++; c.stats.dslash_ms += ms; }
            else { c.stats.mdagm_launches++; c.stats.mdagm_ms += ms; }
        }
        marks.clear();
        stop_of_chunk.clear();
        c.ktimer.reset();
    }
};

// The reference CG and multi-shift divide by p.Ap and |r|^2 unchecked
// (ks_d_congrad_fn.cpp:511, ks_multicg_offset.cpp:475-520): a NaN or Inf in
// the source or the links, or a zero p.Ap, runs on to the iteration limit
// and returns garbage as success.  Here the device records the breakdown in
// SolverState::error (1: non-finite residual, 2: zero or non-finite p.Ap)
// and ends the run; the call returns QPHIX_FAIL with this message.
[[noreturn]] void breakdown(const char *who, int code, int iteration)
{
    if (code == 3)
        throw Error(std::string(who) + ": internal error at iteration " + std::to_string(iteration) +
                    " (deferred multi-shift update outside its segment)");
    throw Error(std::string(who) + ": CG breakdown at iteration " + std::to_string(iteration) +
                (code == 2 ? " (p.Ap is zero or not finite)" : " (the residual is not finite)"));
}

void require_finite(const char *who, double v, const char *what)
{
    if (!std::isfinite(v)) throw Error(std::string(who) + ": " + what + " is not finite");
}

int next_chunk(int current, double size_prev, double size_now, int done, double target, int cap)
{
    Context &c = ctx();
    int chunk = current;
    if (target > 0 && size_now > 0 && size_prev > size_now && done > 0) {
        const double rate = std::log(size_prev / size_now) / done;
        const double left = std::log(size_now / target) / rate;
        chunk = (int)std::ceil(left) + 1;
    } else {
        chunk = current * 2;
    }
    if (chunk < 2) chunk = 2;
    if (chunk > c.max_chunk) chunk = c.max_chunk;
    if (cap > 0 && chunk > cap) chunk = cap;
    return chunk;
}

// Runs the device iterations of one solver phase until the device stops.
// `enqueue(gate)` enqueues one iteration; `next(chunk, it0)` sizes the next
// chunk from the host mirror S.
//  * Graph mode: the iteration is captured once (per phase configuration)
//    into the body of a CUDA-graph while loop; the update kernel's last
//    block clears the loop condition when the stop test fires, so a whole
//    phase runs with no host round trip.  A hard iteration cap and the
//    kernel failure word also end the loop.
//  * Chunk mode (kernel timing on, or QPHIX_B200_GRAPHS=0): chunks of gated
//    iterations, one state read per chunk.
class IterLoop {
public:
    IterLoop() = default;
    IterLoop(const IterLoop &) = delete;
    IterLoop &operator=(const IterLoop &) = delete;
    ~IterLoop() { release(); }
    void invalidate() { release(); }
    // host time spent capturing and instantiating graphs so far
    double build_seconds() const { return build_sec_; }

    template <typename Enq, typename Next>
    void run(Enq enqueue, Next next, TimedLaunches &tl, int cap, int first_chunk = 8)
    {
        Context &c = ctx();
        SolverState &S = *c.h_state;
        S.stop_at = INT_MAX;
        S.skip_axpy = 0;
        S.err = c.d_err;
        S.counter = S.counter2 = 0;
        // NCCL calls are not captured: a solve over several GPUs runs in chunks
        if (graphs_enabled() && !tl.on && !(c.halo.on && c.halo.nranks > 1)) {
            if (!exec_) {
                const double t0 = wall_seconds();
                build(enqueue);
                build_sec_ += wall_seconds() - t0;
            }
            S.use_cond = 1;
            S.cond = handle_;
            S.iter_cap = S.iteration + (cap > 0 ? cap : 1);
            upload_state();
            QB_CUDA(cudaGraphLaunch(exec_, c.stream));
            download_state();
            S.use_cond = 0;
            if (S.stop_at == INT_MAX) throw Error("solver: device loop ended without a stop");
            return;
        }
        S.use_cond = 0;
        S.iter_cap = INT_MAX;
        upload_state();
        int chunk = first_chunk;
        for (;;) {
            for (int k = 0; k < chunk; ++k) enqueue(k);
            const int it0 = S.iteration;
            QB_CUDA(cudaGetLastError());
            download_state();
            tl.collect(S.stop_at);
            if (S.stop_at != INT_MAX) break;
            if (S.iteration == it0) throw Error("solver: device iterations made no progress");
            chunk = next(chunk, it0);
        }
    }

private:
    static bool graphs_enabled()
    {
        static int v = -1;
        if (v < 0) {
            const char *e = std::getenv("QPHIX_B200_GRAPHS");
            v = (e && e[0] == '0') ? 0 : 1;
        }
        return v == 1;
    }

    template <typename Enq> void build(Enq enqueue)
    {
        Context &c = ctx();
        QB_CUDA(cudaGraphCreate(&graph_, 0));
        QB_CUDA(cudaGraphConditionalHandleCreate(&handle_, graph_, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams p = {};
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = handle_;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        cudaGraphNode_t node;
        QB_CUDA(cudaGraphAddNode(&node, graph_, nullptr, 0, &p));
        cudaGraph_t body = p.conditional.phGraph_out[0];
        QB_CUDA(cudaStreamBeginCaptureToGraph(c.stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue(-1);
        } catch (...) {
            cudaGraph_t dummy;
            cudaStreamEndCapture(c.stream, &dummy);
            throw;
        }
        QB_CUDA(cudaStreamEndCapture(c.stream, &body));
        QB_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
    }

    void release()
    {
        if (exec_) cudaGraphExecDestroy(exec_);
        if (graph_) cudaGraphDestroy(graph_);
        exec_ = nullptr;
        graph_ = nullptr;
        handle_ = 0;
    }

    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
    cudaGraphConditionalHandle handle_ = 0;
    double build_sec_ = 0;
};

}  // namespace

// ===========================================================================
// CG, reference control flow: QPHIX_fptype_asqtad_invert,
// ks_d_congrad_fn.cpp:221-619, statement for statement; only the loops over
// sites moved into kernels.
// ===========================================================================
int cg_reference(Prec P, const LinkSet &ls, SolveArgs &A)
{
    Context &c = ctx();
    const Launch L = c.launch();
    SolverState &S = *c.h_state;
    const bool single = (P == Prec::Single);
    auto R = [&](double v) { return round_prec(v, single); };
    QPHIX_info_t *info = A.info;
    QPHIX_invert_arg_t *inv = A.inv;
    QPHIX_resid_arg_t *res = A.res;

    VecBlock t_src, t_dest;
    if (inv->parity != QPHIX_ODD) { t_src = A.in[0]; t_dest = A.out[0]; }
    else { t_src = A.in[1]; t_dest = A.out[1]; }

    const int niter = inv->max;
    const int max_restarts = inv->nrestart;
    const double rsqmin = R(res->resid);
    const double relrsqmin = R(res->relresid);
    const int max_cg = max_restarts * niter;
    const double msq_x4 = R(4.0 * A.mass * A.mass);
    int parity = inv->parity & 1;
    int otherparity = 1 - parity;
    int parity0 = inv->parity;
    const double V = 2.0 * c.g.vh;
    // relative_residue divides by the volume of the whole lattice (ks_blas_utils_c.cpp:148)
    const double Vglobal = c.halo.on ? (double)c.halo.global_sites : V;
    const bool relres = relrsqmin > 0;
    if (niter <= 0) throw Error("invert: inv_arg->max must be positive");

    Ws ws;
    VecBlock ttt = ws.get(P), tmp = ws.get(P), cg_p = ws.get(P), resid = ws.get(P);
    info->final_sec = wall_seconds();
    info->final_flop = 0.;
    TimedLaunches tl(c.kernel_timing);

    auto conv = [&](double r1, double r2) {
        return (rsqmin <= 0 || rsqmin > r1) && (relrsqmin <= 0 || relrsqmin > r2);
    };

    int total_iters = 0, iteration = 0, nrestart = 0;
    double rsq = 0, relrsq = 0, source_norm = 0;
    bool finished = false;
    S.error = 0;
    while (!finished) {
        // start: (:309-350)
        source_norm = norm2_sync(P, t_src);
        require_finite("asqtad_invert", source_norm, "|source|^2");
        nrestart = 0;
        total_iters += iteration;
        iteration = 0;
        res->size_r = 0;
        res->size_relr = 0;
        if (source_norm == 0.0) {
            vec_zero(P, t_dest, L);
            sync_check();
            info->final_sec = wall_seconds() - info->final_sec;
            res->final_rel = 0;
            res->final_rsq = 0;
            res->final_iter = total_iters;
            res->final_restart = nrestart;
            c.stats.iterations = total_iters;
            return iteration;
        }
        bool switch_parity = false;
        dslash_prepare(P, ls, L);
        IterLoop loop;  // rebuilt per parity pass: the vectors differ
        for (;;) {
            if ((iteration % niter == 0) || conv(res->size_r, res->size_relr)) {
                // (re)initialisation with the true residual (:365-448)
                S.msq_x4 = msq_x4;
                S.counter = S.counter2 = 0;
                upload_state();
                tl.run(0, -1, [&] { dslash(P, L, tmp, t_dest, ls, otherparity); });
                tl.run(0, -1, [&] { dslash(P, L, ttt, tmp, ls, parity); });
                cg_restart_residual(P, L, ttt, t_dest, t_src, resid, cg_p, c.d_state, c.d_partials, relres);
                download_state();
                tl.collect(INT_MAX);
                rsq = S.rsq;
                require_finite("asqtad_invert", rsq, "the restart residual |b - M x|^2");
                if (relres) relrsq = R(std::sqrt(2 * S.relrsq / Vglobal));
                res->final_rsq = R(rsq) / source_norm;
                res->final_rel = R(relrsq);
                iteration++;
                if (iteration >= max_cg || nrestart >= max_restarts ||
                    conv(res->final_rsq, res->final_rel)) {
                    if (parity0 == QPHIX_EVENODD) {
                        // (:437-444): the reference's parity bookkeeping, kept as is
                        otherparity = parity0 & 1;
                        parity = 1 - otherparity;
                        parity0 = QPHIX_EVEN;
                        t_src = A.in[1];
                        t_dest = A.out[1];
                        switch_parity = true;
                    }
                    break;
                }
                if (iteration != 0) nrestart++;
            }
            // iterations on the device (:450-576)
            S.rsq = rsq;
            S.relrsq = relrsq;
            S.source_norm = source_norm;
            S.rsqmin = rsqmin;
            S.relrsqmin = relrsqmin;
            S.msq_x4 = msq_x4;
            S.iteration = iteration;
            S.niter = niter;
            S.prec_single = single;
            S.size_r = res->size_r;
            S.size_relr = res->size_relr;
            double size_prev = res->size_r > 0 ? res->size_r : 1.0;
            loop.run(
                [&](int k) {
                    tl.run(0, k, [&] { dslash_gated(P, L, tmp, cg_p, ls, otherparity, c.d_state, k); });
                    tl.run(1, k, [&] {
                        dslash_mdagm_dot(P, L, ttt, tmp, ls, cg_p, -msq_x4, parity, c.d_state, c.d_partials, k, 0);
                    });
                    cg_update(P, L, t_dest, cg_p, resid, ttt, c.d_state, c.d_partials, k, relres);
                    cg_axpy(P, L, resid, cg_p, c.d_state, k);
                },
                [&](int chunk, int it0) {
                    const int cap = niter - (S.iteration % niter);
                    const int n = next_chunk(chunk, size_prev, S.size_r, S.iteration - it0, rsqmin, cap);
                    size_prev = S.size_r;
                    return n;
                },
                tl, niter - (iteration % niter) + 1);
            if (S.error) breakdown("asqtad_invert", S.error, S.iteration);
            iteration = S.iteration;
            rsq = S.rsq;
            relrsq = S.relrsq;
            res->size_r = S.size_r;
            res->size_relr = S.size_relr;
            res->final_rsq = res->size_r;
        }
        if (!switch_parity) finished = true;
    }
    info->final_sec = wall_seconds() - info->final_sec;
    total_iters += iteration;
    res->final_iter = total_iters;
    res->final_restart = nrestart;
    info->final_flop = 1187. * total_iters * V;
    info->status = QPHIX_SUCCESS;
    c.stats.iterations = total_iters;
    c.stats.true_rsq = res->final_rsq;
    return iteration;
}

// ===========================================================================
// Mixed precision CG: FP64 solution and true residual, sloppy inner CG in
// precision ps with reliable updates (the true residual is recomputed in
// FP64 whenever the sloppy residual has dropped by `reliable_delta`).
// Converges on the FP64 true residual |b - M x|^2 / |b|^2 < tol.
// ===========================================================================
namespace {

// iterations without a new smallest inner residual after which the mixed CG
// takes a reliable update and restarts its search direction
constexpr int kInnerStallWindow = 256;

// Mixed multi-shift: a shift whose recurrence residual zeta_k^2 |r|^2 is this
// factor below the sloppy floor gets no further vector updates in the sloppy
// phase.  Its solution is then as accurate as the FP32 recurrence allows
// (stopping at the floor itself lengthened the refinements: 2379 against
// 1942 iterations at 32^3x64), and the update traffic of the heavy shifts,
// which get there in a fraction of the iterations, is saved.
constexpr double kShiftStopFactor = 1e-6;
// reliable-update threshold of the per-shift refinements, relative to the
// CG's: at 32^3x64 0.25, 0.1 and 0.05 give the same iterations with 49, 40
// and 38 reliable updates (303, 296, 293 ms of refinement)
constexpr double kRefineDeltaFactor = 0.1;
// inner stagnation window of a refinement on 16-bit links (24 restarts
// healthy refinements too often; 256 lets an ill-conditioned one crawl)
constexpr int kRefineStallWindow = 48;
// least |r|^2 reduction of one reliable-update cycle of a refinement on
// 16-bit links before it continues on FP32 links
constexpr double kRefineEscalate = 20.0;
// systems of one batched refinement (the batched solver's limit)
constexpr int kBatchRefineMax = 64;
// QPHIX_B200_MS_REFINE=batched refines the shifts of a mixed multi-shift in
// one batched solve instead of one after the other (mixed CG each)
bool refine_batched()
{
    const char *e = std::getenv("QPHIX_B200_MS_REFINE");
    return e && std::strcmp(e, "batched") == 0;
}

struct MixedResult {
    double true_rsq_rel = 0;
    int iterations = 0;
    int reliable_updates = 0;
    int escalated = 0;
    // wall-clock split (QPHIX_B200_VERBOSE >= 2 only): set-up and first
    // true residual, inner CG loops, reliable updates, and the graph
    // captures inside the inner loops
    double t_setup = 0, t_loop = 0, t_ru = 0, t_graph = 0;
};

// `ls_up`: FP32 links to continue with when a 16-bit inner solve stops
// converging (see below); may be null.
// escalate_ratio / escalate_after: a 16-bit inner solve continues in FP32
// after `escalate_after` reliable updates in a row whose true |r|^2 fell by
// less than 1 / escalate_ratio (or that an inner stagnation forced)
// stall_window: inner iterations without a new smallest |r|^2 that force a
// reliable update (and count as a stall)
MixedResult mixed_pass(Prec ps, const LinkSet &ls64, const LinkSet &lss, const LinkSet *ls_up, VecBlock x,
                       VecBlock b, int parity, double mass, double tol, int max_cg, TimedLaunches &tl,
                       double escalate_ratio = 0.25, int escalate_after = 2, int stall_window = kInnerStallWindow)
{
    Context &c = ctx();
    const LinkSet *ls_cur = &lss;
    const Launch L = c.launch();
    SolverState &S = *c.h_state;
    const int other = 1 - parity;
    const double m4 = 4.0 * mass * mass;
    const double delta2 = c.reliable_delta * c.reliable_delta;
    MixedResult out;
    const bool split = c.verbose >= 2;
    double t_mark = split ? wall_seconds() : 0.0;
    auto lap = [&](double &acc) {
        if (!split) return;
        sync_check();
        const double now = wall_seconds();
        acc += now - t_mark;
        t_mark = now;
    };

    const double bnorm = norm2_sync(Prec::Double, b);
    require_finite("asqtad_invert", bnorm, "|source|^2");
    S.error = 0;
    if (bnorm == 0.0) {
        vec_zero(Prec::Double, x, L);
        sync_check();
        return out;
    }
    Ws ws;
    VecBlock tmp64 = ws.get(Prec::Double), ttt64 = ws.get(Prec::Double), r64 = ws.get(Prec::Double);
    // the partial solution x_s is FP32 under a 16-bit inner solve
    VecBlock xs = ws.get(inner_x_prec(ps)), rs = ws.get(ps), pv = ws.get(ps), tmps = ws.get(ps), ttts = ws.get(ps);

    auto true_residual = [&]() {
        S.msq_x4 = m4;
        S.counter = S.counter2 = 0;
        upload_state();
        dslash(Prec::Double, L, tmp64, x, ls64, other);
        dslash(Prec::Double, L, ttt64, tmp64, ls64, parity);
        cg_true_residual(Prec::Double, L, ttt64, x, b, r64, c.d_state, c.d_partials, c.d_scalars);
        QB_CUDA(cudaMemcpyAsync(c.h_scalars, c.d_scalars, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        sync_check();
        return c.h_scalars[0];
    };

    double rsq = true_residual();
    require_finite("asqtad_invert", rsq, "the true residual |b - M x|^2");
    out.true_rsq_rel = rsq / bnorm;
    if (out.true_rsq_rel < tol) return out;

    vec_copy(ps, rs, Prec::Double, r64, L);
    vec_copy(ps, pv, ps, rs, L);
    vec_zero(inner_x_prec(ps), xs, L);
    S.rsq = rsq;
    S.rsq_ru = rsq;
    S.rsqstop = tol * bnorm;
    S.msq_x4 = m4;
    S.iteration = 0;
    S.max_cg = max_cg;
    S.prec_single = 0;
    S.ru_best = rsq;
    S.ru_best_iter = 0;
    S.ru_stall_window = stall_window;
    S.ru_stalled = 0;
    int stalled = 0;
    dslash_prepare(ps, *ls_cur, L);
    IterLoop loop;
    lap(out.t_setup);
    for (;;) {
        double size_prev = S.rsq;
        loop.run(
            [&](int k) {
                tl.run(0, k, [&] { dslash_gated(ps, L, tmps, pv, *ls_cur, other, c.d_state, k); });
                tl.run(1, k, [&] {
                    dslash_mdagm_dot(ps, L, ttts, tmps, *ls_cur, pv, -m4, parity, c.d_state, c.d_partials, k, 0);
                });
                mx_update(ps, L, xs, pv, rs, ttts, c.d_state, c.d_partials, k, delta2);
                cg_axpy(ps, L, rs, pv, c.d_state, k);
            },
            [&](int chunk, int it0) {
                const double target = std::max(S.rsqstop, delta2 * S.rsq_ru);
                const int n = next_chunk(chunk, size_prev, S.rsq, S.iteration - it0, target, 0);
                size_prev = S.rsq;
                return n;
            },
            tl, max_cg - S.iteration + 1);
        if (S.error) breakdown("asqtad_invert (mixed precision)", S.error, S.iteration);
        lap(out.t_loop);
        out.iterations = S.iteration;
        const double oldrsq = S.oldrsq;
        const double sloppy_rsq = S.rsq;
        // reliable update: x += x_s, r = b - M x in FP64
        vec_add(Prec::Double, x, inner_x_prec(ps), xs, L);
        vec_zero(inner_x_prec(ps), xs, L);
        const double prev_true = rsq;
        rsq = true_residual();
        require_finite("asqtad_invert (mixed precision)", rsq, "the true residual |b - M x|^2");
        out.reliable_updates++;
        out.true_rsq_rel = rsq / bnorm;
        if (c.verbose)
            std::fprintf(stderr, "qphix_b200 mixed CG: iter %d RU %d prec %d sloppy %.3e true %.3e\n",
                         S.iteration, out.reliable_updates, (int)ps, sloppy_rsq / bnorm, rsq / bnorm);
        if (out.true_rsq_rel < tol || S.iteration >= max_cg) break;
        // A 16-bit inner solve perturbs the operator by ~1e-4 relative; once
        // the residual lives in the lowest modes of an ill-conditioned system
        // the corrections stop reducing the true residual, or the inner CG
        // itself stops reducing its residual.  Two reliable updates in a row
        // that fail to halve the true residual, or that an inner stagnation
        // forced, switch the inner solve to FP32.
        const bool inner_stall = S.ru_stalled != 0;
        stalled = (rsq > escalate_ratio * prev_true || inner_stall) ? stalled + 1 : 0;
        if (stalled >= escalate_after && (ps == Prec::Half || ls_cur->prec == Prec::Half) && ls_up && ls_up->valid) {
            VecBlock p32 = ws.get(Prec::Single);
            vec_copy(Prec::Single, p32, ps, pv, L);
            pv = p32;
            // the partial solution restarts at zero (x holds the sum so far)
            xs = ws.get(Prec::Single);
            vec_zero(Prec::Single, xs, L);
            rs = ws.get(Prec::Single);
            tmps = ws.get(Prec::Single);
            ttts = ws.get(Prec::Single);
            ps = Prec::Single;
            ls_cur = ls_up;
            stalled = 0;
            out.escalated = 1;
            loop.invalidate();
            dslash_prepare(ps, *ls_cur, L);
        }
        vec_copy(ps, rs, Prec::Double, r64, L);
        // after an inner stagnation the search direction is restarted (p = r)
        S.b = inner_stall ? 0.0 : rsq / oldrsq;
        S.rsq = rsq;
        S.rsq_ru = rsq;
        S.ru_best = rsq;
        S.ru_best_iter = S.iteration;
        S.ru_stalled = 0;
        S.skip_axpy = 0;
        S.counter = S.counter2 = 0;
        upload_state();
        cg_axpy(ps, L, rs, pv, c.d_state, -1);  // p = r + beta p with the true residual
        lap(out.t_ru);
    }
    lap(out.t_ru);
    out.t_graph = loop.build_seconds();
    return out;
}

}  // namespace

int cg_mixed(Prec ps, const LinkSet &ls64, const LinkSet &lss, const LinkSet *ls_up, SolveArgs &A)
{
    Context &c = ctx();
    QPHIX_info_t *info = A.info;
    QPHIX_invert_arg_t *inv = A.inv;
    QPHIX_resid_arg_t *res = A.res;
    info->final_sec = wall_seconds();
    TimedLaunches tl(c.kernel_timing);
    const int max_cg = inv->max * inv->nrestart;
    const double tol = res->resid;
    int parity = inv->parity & 1;
    int parity0 = inv->parity;
    VecBlock b = (inv->parity != QPHIX_ODD) ? A.in[0] : A.in[1];
    VecBlock x = (inv->parity != QPHIX_ODD) ? A.out[0] : A.out[1];
    int total = 0, last = 0, rus = 0;
    double worst = 0;
    for (;;) {
        MixedResult m = mixed_pass(ps, ls64, lss, ls_up, x, b, parity, A.mass, tol, max_cg, tl);
        c.stats.escalated |= m.escalated;
        total += m.iterations;
        last = m.iterations;
        rus += m.reliable_updates;
        worst = std::max(worst, m.true_rsq_rel);
        res->final_rsq = m.true_rsq_rel;
        res->size_r = m.true_rsq_rel;
        if (parity0 == QPHIX_EVENODD) {
            // same parity sequence as the reference solver (ks_d_congrad_fn.cpp:437-444)
            parity = 0;
            parity0 = QPHIX_EVEN;
            b = A.in[1];
            x = A.out[1];
            continue;
        }
        break;
    }
    res->final_rel = 0;
    res->size_relr = 0;
    res->final_iter = total;
    res->final_restart = rus;
    info->final_sec = wall_seconds() - info->final_sec;
    info->final_flop = 1187. * total * 2.0 * c.g.vh;
    info->status = QPHIX_SUCCESS;
    c.stats.iterations = total;
    c.stats.reliable_updates = rus;
    c.stats.true_rsq = worst;
    return last;
}

// ===========================================================================
// Multi-shift CG, reference control flow: QPHIX_fptype_asqtad_invert_multi,
// ks_multicg_offset.cpp:205-689.
// ===========================================================================
namespace {

struct MsPass {
    int iteration = 0;
    int reliable_updates = 0;
    bool converged = false;
    double rsq = 0, source_norm = 0;
};

// Deferred shift updates of the mixed multi-shift (FP32 Krylov vectors).
// A segment runs m iterations that store their residuals r(t) (slot t: the
// residual after iteration t, which that iteration's direction updates read)
// and every shift's scalars; no shifted vector is touched.  At the end of
// the segment (a reliable update of the base, a full buffer, convergence)
// the recurrences
//   x += b_t p(t)          (upd bit 0)
//   p(t+1) = z_t r(t) + a_t p(t)   (upd bit 1)
// are expanded on the device (k_ms_coef): p(t) = P_t p(0) + sum_{u<t}
// D_t[u] r(u), so
//   x += GX p(0) + sum_u CX[u] r(u),   p(m) = P_m p(0) + sum_u D_m[u] r(u),
// with GX = sum_t b_t P_t and CX[u] = sum_{t>u} b_t D_t[u], and k_ms_flush
// applies them in FP64.  The base direction (the Dslash input) is updated
// every iteration as before; its solution is deferred like the others, from
// a copy of the direction taken at the start of the segment.
class MsDeferred {
public:
    // nullptr when fewer than kMinSlots residuals fit in the memory budget
    static std::unique_ptr<MsDeferred> make(int n, int j_low, const std::vector<VecBlock> &pm)
    {
        Context &c = ctx();
        const size_t slot = vec_bytes(Prec::Single, c.g.vh);
        size_t free_b = 0, total_b = 0;
        QB_CUDA(cudaMemGetInfo(&free_b, &total_b));
        const size_t budget = std::min(kBudgetBytes, free_b / 4);
        size_t fit = std::min<size_t>(budget / slot, kMsSegMax);
        // QPHIX_B200_MS_SEGMENT: fewer iterations per segment (at least
        // kMinSlots), to exercise the segment hand-over on small lattices
        if (const char *e = std::getenv("QPHIX_B200_MS_SEGMENT"))
            fit = std::min<size_t>(fit, (size_t)std::max(std::atoi(e), kMinSlots));
        if (fit < (size_t)kMinSlots) return nullptr;
        return std::unique_ptr<MsDeferred>(new MsDeferred(n, j_low, pm, (int)fit));
    }
    ~MsDeferred() { release(); }
    VecBlock hist() const { return hist_; }
    MsHistEntry *hist_scalars() const { return d_hist_; }

    // a segment begins after the current iteration, from the current base direction
    void begin(SolverState &S, const Launch &L)
    {
        S.ms_seg_cap = cap_;
        S.ms_seg_start = S.iteration;
        S.ms_seg_full = 0;
        vec_copy(Prec::Single, p_low0_, Prec::Single, pm_[j_low_], L);
    }

    // apply the segment's updates to the solutions d_x (FP64) and the shifted
    // directions d_p (FP32), then begin the next segment; no host round trip
    void flush(SolverState &S, VecBlock *d_x, VecBlock *d_p, const Launch &L)
    {
        const int m = S.iteration - S.ms_seg_start;
        if (m < 0 || m > cap_) throw Error("invert_multi: deferred segment out of range");
        if (m > 0) {
            ms_coef(L, d_hist_, m, n_, j_low_, d_coef_, d_jobs_);
            ms_flush(L, hist_, m, d_coef_, d_jobs_, n_, d_x, d_p0_, d_p);
        }
        begin(S, L);
    }

private:
    static constexpr size_t kBudgetBytes = size_t(4) << 30;
    static constexpr int kMinSlots = 16;

    MsDeferred(int n, int j_low, const std::vector<VecBlock> &pm, int cap)
        : cap_(cap), n_(n), j_low_(j_low), pm_(pm)
    {
        Context &c = ctx();
        try {  // (a failed allocation releases the ones before it)
            hist_.data = dev_alloc(vec_bytes(Prec::Single, c.g.vh) * cap_);
            d_hist_ = static_cast<MsHistEntry *>(dev_alloc(sizeof(MsHistEntry) * cap_ * n_));
            d_coef_ = static_cast<double *>(dev_alloc(sizeof(double) * 2 * (cap_ + 1) * n_));
            d_jobs_ = static_cast<int *>(dev_alloc(sizeof(int) * n_));
            d_p0_ = static_cast<VecBlock *>(dev_alloc(sizeof(VecBlock) * n_));
            p_low0_ = alloc_vec(Prec::Single);
            std::vector<VecBlock> p0(pm);
            p0[j_low_] = p_low0_;
            QB_CUDA(cudaMemcpyAsync(d_p0_, p0.data(), sizeof(VecBlock) * n_, cudaMemcpyHostToDevice, c.stream));
            QB_CUDA(cudaStreamSynchronize(c.stream));
        } catch (...) {
            release();
            throw;
        }
    }

    void release()
    {
        dev_free(hist_.data);
        dev_free(d_hist_);
        dev_free(d_coef_);
        dev_free(d_jobs_);
        dev_free(d_p0_);
        if (p_low0_.data) free_vec(p_low0_);
        hist_.data = p_low0_.data = nullptr;
        d_hist_ = nullptr;
        d_coef_ = nullptr;
        d_jobs_ = nullptr;
        d_p0_ = nullptr;
    }

    int cap_, n_, j_low_;
    std::vector<VecBlock> pm_;
    VecBlock hist_, p_low0_;
    MsHistEntry *d_hist_ = nullptr;
    double *d_coef_ = nullptr;
    int *d_jobs_ = nullptr;
    VecBlock *d_p0_ = nullptr;
};

// one parity pass of the multi-shift recurrence; x[] in precision xp, the
// Krylov vectors in precision p
MsPass ms_pass(Prec p, Prec xp, const LinkSet &ls, VecBlock src, std::vector<VecBlock> &x,
               std::vector<VecBlock> &pm, VecBlock ttt, VecBlock tmp, VecBlock resid, VecBlock *d_x,
               VecBlock *d_p, int parity, const std::vector<double> &shifts, int j_low,
               double offset_low, double rsqmin, int max_cg, bool single, TimedLaunches &tl,
               double shift_rsqmin, double ru_delta2 = 0.0,
               const std::function<double()> &reliable_update = std::function<double()>(),
               double ru_rsqmin = 0.0, MsDeferred *df = nullptr)
{
    Context &c = ctx();
    const Launch L = c.launch();
    SolverState &S = *c.h_state;
    const int n = (int)x.size();
    const int other = 1 - parity;
    MsPass out;
    out.source_norm = norm2_sync(p, src);
    require_finite("asqtad_invert_multi", out.source_norm, "|source|^2");
    S.error = 0;
    for (int j = 0; j < n; ++j) vec_zero(xp, x[j], L);
    for (int j = 0; j < n; ++j) vec_copy(p, pm[j], p, src, L);
    vec_copy(p, resid, p, src, L);
    out.rsq = out.source_norm;
    if (out.source_norm == 0.) {
        sync_check();
        return out;
    }
    S.rsqstop = rsqmin * out.source_norm;
    for (int j = 0; j < n; ++j) {
        S.shifts[j] = shifts[j];
        S.zeta_im1[j] = S.zeta_i[j] = 1.0;
        S.beta_im1[j] = -1.0;
        S.alpha[j] = 0.0;
    }
    S.num_now = n;
    S.n_shifts = n;
    S.j_low = j_low;
    S.rsq = out.rsq;
    S.iteration = 0;
    S.max_cg = max_cg;
    S.first_iter = 1;
    S.converged = 0;
    S.prec_single = single;
    S.shift_stop = shift_rsqmin * out.source_norm;
    for (int j = 0; j < n; ++j) S.shift_done_at[j] = INT_MAX;
    S.ms_delta2 = reliable_update ? ru_delta2 : 0.0;
    S.rsq_ru = out.source_norm;
    S.ms_seg_cap = 0;
    if (df) df->begin(S, L);
    const double m4 = round_prec(-1.0 * offset_low, single);
    double size_prev = out.rsq;
    dslash_prepare(p, ls, L);
    IterLoop loop;
    int ru_stalls = 0;
    double t_run = 0, t_flush = 0, t_ru = 0;  // verbose: host-side phase times
    for (;;) {
        S.ms_ru = 0;
        const double t0 = c.verbose ? wall_seconds() : 0.0;
        loop.run(
            [&](int k) {
                tl.run(0, k, [&] { dslash_gated(p, L, tmp, pm[j_low], ls, other, c.d_state, k); });
                tl.run(1, k, [&] {
                    dslash_mdagm_dot(p, L, ttt, tmp, ls, pm[j_low], m4, parity, c.d_state, c.d_partials, k, 1);
                });
                ms_residual(p, L, resid, ttt, c.d_state, c.d_partials, k);
                if (df) ms_defer(L, pm[j_low], resid, df->hist(), df->hist_scalars(), n, c.d_state, k);
                else ms_update(p, L, xp, d_x, d_p, resid, n, c.d_state, k);
            },
            [&](int chunk, int it0) {
                const int m = next_chunk(chunk, size_prev, S.rsq, S.iteration - it0, S.rsqstop, max_cg - S.iteration);
                size_prev = S.rsq;
                return m;
            },
            tl, max_cg + 1);
        if (S.error) breakdown("asqtad_invert_multi", S.error, S.iteration);
        const bool seg_full = S.ms_seg_full != 0;
        const double t1 = c.verbose ? wall_seconds() : 0.0;
        if (df) df->flush(S, d_x, d_p, L);  // (and begins the next segment)
        if (c.verbose) {
            sync_check();
            const double t2 = wall_seconds();
            t_run += t1 - t0;
            t_flush += t2 - t1;
        }
        if (S.converged || S.iteration >= max_cg) break;
        if (seg_full && !S.ms_ru) continue;  // a full segment, flushed: carry on
        if (!S.ms_ru) break;
        // reliable update of the base shift: r = b - (A + sigma_low) x_low in FP64
        const double prev = S.rsq_ru;
        const double t3 = c.verbose ? wall_seconds() : 0.0;
        const double rsq = reliable_update();
        if (c.verbose) t_ru += wall_seconds() - t3;
        require_finite("asqtad_invert_multi", rsq, "the base shift's true residual");
        S.rsq = rsq;
        S.rsq_ru = rsq;
        ++out.reliable_updates;
        if (rsq <= ru_rsqmin * out.source_norm) {
            S.converged = 1;
            break;
        }
        // two updates in a row that do not halve the true residual: the
        // recurrence has lost the base shift; the refinement takes over
        ru_stalls = (rsq > 0.5 * prev) ? ru_stalls + 1 : 0;
        if (ru_stalls >= 2) break;
    }
    out.iteration = S.iteration;
    out.converged = S.converged != 0;
    out.rsq = S.rsq;
    if (c.verbose)
        std::fprintf(stderr, "qphix_b200 multi-shift pass: device loops %.1f ms, segment flushes %.1f ms, "
                             "reliable updates %.1f ms\n", 1e3 * t_run, 1e3 * t_flush, 1e3 * t_ru);
    if (c.verbose) {
        std::fprintf(stderr, "qphix_b200 multi-shift: iter %d converged %d rsq/src %.3e active %d pkp %.3e\n",
                     S.iteration, out.converged, S.rsq / out.source_norm, S.num_now, S.pkp);
        for (int j = 0; j < n; ++j)
            std::fprintf(stderr, "  shift %d: %.4e beta %.4e zeta %.4e alpha %.4e finished %d\n", j, S.shifts[j],
                         S.beta_i[j], S.zeta_ip1[j], S.alpha[j], S.finished[j]);
    }
    return out;
}

void upload_blocks(VecBlock *d, const std::vector<VecBlock> &h)
{
    Context &c = ctx();
    QB_CUDA(cudaMemcpyAsync(d, h.data(), sizeof(VecBlock) * h.size(), cudaMemcpyHostToDevice, c.stream));
    sync_check();
}

}  // namespace

int multishift_reference(Prec P, const LinkSet &ls, MultiArgs &A)
{
    Context &c = ctx();
    const int n = A.n;
    if (n <= 0) return 0;  // (:218-225)
    if (n > kMaxShifts) throw Error("invert_multi: more offsets than MAXNDMASS (150)");
    const bool single = (P == Prec::Single);
    auto R = [&](double v) { return round_prec(v, single); };
    QPHIX_info_t *info = A.info;
    QPHIX_invert_arg_t *inv = A.inv;
    int parity0 = inv->parity;
    VecBlock t_src = (parity0 != QPHIX_ODD) ? A.in[0] : A.in[1];
    std::vector<VecBlock> t_dest = (parity0 != QPHIX_ODD) ? A.out[0] : A.out[1];
    const int niter = inv->max;
    const int max_restarts = inv->nrestart;
    const double rsqmin = R(A.res[0]->resid);
    const int max_cg = max_restarts * niter;
    int parity = parity0 & 1;
    const double V = 2.0 * c.g.vh;

    Ws ws;
    VecBlock ttt = ws.get(P), tmp = ws.get(P), resid = ws.get(P);
    std::vector<VecBlock> pm(n);
    for (int j = 0; j < n; ++j) pm[j] = ws.get(P);
    std::vector<double> shifts(n);
    double offset_low = 1.0e+20;
    int j_low = -1;
    for (int j = 0; j < n; ++j) {  // (:332-342)
        shifts[j] = R(R(A.mass[j] * A.mass[j]) * 4.0);
        if (shifts[j] < offset_low) { offset_low = shifts[j]; j_low = j; }
    }
    for (int j = 0; j < n; ++j)
        if (j != j_low) shifts[j] = R(shifts[j] - shifts[j_low]);
    for (int j = 0; j < n; ++j) c.h_state->finished[j] = 0;

    VecBlock *d_x = static_cast<VecBlock *>(dev_alloc(sizeof(VecBlock) * n));
    VecBlock *d_p = static_cast<VecBlock *>(dev_alloc(sizeof(VecBlock) * n));
    upload_blocks(d_p, pm);
    TimedLaunches tl(c.kernel_timing);
    info->final_sec = wall_seconds();
    info->final_flop = 0.;
    int total_iters = 0, iteration = 0;
    const int nrestart = 0;
    for (;;) {
        upload_blocks(d_x, t_dest);
        MsPass r = ms_pass(P, P, ls, t_src, t_dest, pm, ttt, tmp, resid, d_x, d_p, parity, shifts, j_low,
                           offset_low, rsqmin, max_cg, single, tl, 0.0);
        iteration = r.iteration;
        total_iters += r.iteration;
        if (r.source_norm == 0.) {  // (:377-419)
            for (int j = 0; j < n; ++j) {
                A.res[j]->final_rsq = 0.;
                A.res[j]->size_r = 0.;
                A.res[j]->size_relr = 0.;
                A.res[j]->final_iter = iteration;
                A.res[j]->final_restart = nrestart;
            }
            break;
        }
        for (int j = 0; j < n; ++j) {  // (:544-550, 626-632)
            A.res[j]->final_rsq = R(r.rsq) / r.source_norm;
            A.res[j]->size_r = A.res[j]->final_rsq;
            A.res[j]->size_relr = A.res[j]->final_rel;
            A.res[j]->final_iter = iteration;
            A.res[j]->final_restart = nrestart;
        }
        if (parity0 == QPHIX_EVENODD) {  // (:534-543, 644-653)
            const int otherparity = parity0 & 1;
            parity = 1 - otherparity;
            parity0 = QPHIX_EVEN;
            t_src = A.in[1];
            t_dest = A.out[1];
            continue;
        }
        break;
    }
    dev_free(d_x);
    dev_free(d_p);
    info->final_sec = wall_seconds() - info->final_sec;
    info->final_flop = (1205. + 15. * n) * total_iters * V;
    info->status = QPHIX_SUCCESS;
    c.stats.iterations = total_iters;
    c.stats.true_rsq = A.res[0]->final_rsq;
    return iteration;
}

// ===========================================================================
// Mixed-precision multi-shift: the shifted recurrence runs in the sloppy
// precision with FP64 solution accumulation until the base residual reaches
// the sloppy floor, then every shift is refined by mixed-precision CG
// started from its multi-shift solution, to its own tolerance on the FP64
// true residual.
// ===========================================================================
int multishift_mixed(Prec ps, const LinkSet &ls64, const LinkSet &lss, const LinkSet *ls_up, MultiArgs &A,
                     const LinkSet *ls32, const RefineOp *rop)
{
    Context &c = ctx();
    const int n = A.n;
    if (n <= 0) return 0;
    if (n > kMaxShifts) throw Error("invert_multi: more offsets than MAXNDMASS (150)");
    QPHIX_info_t *info = A.info;
    QPHIX_invert_arg_t *inv = A.inv;
    int parity0 = inv->parity;
    VecBlock src = (parity0 != QPHIX_ODD) ? A.in[0] : A.in[1];
    std::vector<VecBlock> x = (parity0 != QPHIX_ODD) ? A.out[0] : A.out[1];
    const int max_cg = inv->max * inv->nrestart;
    int parity = parity0 & 1;
    // The sloppy recurrence alone stalls near its residual gap (|r|^2/|b|^2 ~
    // 1e-12 in FP32); reliable updates of the base shift (FP64 r = b - A x)
    // carry the base, and with it the shifts nearest to it, to the target.
    // Shifts far below the floor stop their vector updates (kShiftStopFactor).
    const double floor = (ps == Prec::Single) ? 1e-12 : 1e-6;
    const double target = A.res[0]->resid;
    // (16-bit links perturb the operator too much for the base to reach the
    // target; those modes stop at the floor and refine, as before)
    const bool base_ru_on = ps == Prec::Single && lss.prec == Prec::Single;
    const double rsq_sloppy = base_ru_on ? 1e-2 * target : std::max(target, floor);

    Ws ws;
    VecBlock ttt = ws.get(ps), tmp = ws.get(ps), resid = ws.get(ps), src_s = ws.get(ps);
    VecBlock tmp64 = ws.get(Prec::Double), ttt64 = ws.get(Prec::Double), r64 = ws.get(Prec::Double);
    std::vector<VecBlock> pm(n);
    for (int j = 0; j < n; ++j) pm[j] = ws.get(ps);
    std::vector<double> shifts(n);
    double offset_low = 1.0e+20;
    int j_low = -1;
    for (int j = 0; j < n; ++j) {
        shifts[j] = A.mass[j] * A.mass[j] * 4.0;
        if (shifts[j] < offset_low) { offset_low = shifts[j]; j_low = j; }
    }
    for (int j = 0; j < n; ++j)
        if (j != j_low) shifts[j] -= shifts[j_low];
    for (int j = 0; j < n; ++j) c.h_state->finished[j] = 0;
    // FP32 Krylov vectors: the shifted solutions and directions are updated
    // once per segment from the stored base residuals (MsDeferred), so an
    // iteration moves the bytes of one CG iteration whatever the number of
    // shifts, and each shifted direction is rounded to FP32 once per segment
    // instead of once per iteration.
    // (QPHIX_B200_MS_DEFER=0 keeps the per-iteration updates, for comparison)
    std::unique_ptr<MsDeferred> df;
    const char *defer_env = std::getenv("QPHIX_B200_MS_DEFER");
    if (ps == Prec::Single && !(defer_env && defer_env[0] == '0')) df = MsDeferred::make(n, j_low, pm);
    // Otherwise, with base reliable updates, the shifted solutions accumulate
    // between updates in FP32 partial sums y_j (24 instead of 48 bytes read
    // and written per site and shift each iteration); every reliable update
    // and the end of the recurrence add them into the FP64 x_j.
    const bool partial = base_ru_on && !df;
    std::vector<VecBlock> y(partial ? n : 0);
    for (auto &v : y) v = ws.get(Prec::Single);
    VecBlock *d_x = static_cast<VecBlock *>(dev_alloc(sizeof(VecBlock) * n));
    VecBlock *d_p = static_cast<VecBlock *>(dev_alloc(sizeof(VecBlock) * n));
    upload_blocks(d_p, pm);
    TimedLaunches tl(c.kernel_timing);
    info->final_sec = wall_seconds();
    int total = 0, last = 0, rus = 0;
    double worst = 0;
    for (;;) {
        const Launch L = c.launch();
        vec_copy(ps, src_s, Prec::Double, src, L);
        auto flush = [&](const Launch &Lf) {
            for (int j = 0; j < n; ++j) {
                vec_add(Prec::Double, x[j], Prec::Single, y[j], Lf);
                vec_zero(Prec::Single, y[j], Lf);
            }
        };
        if (partial) {
            for (int j = 0; j < n; ++j) vec_zero(Prec::Double, x[j], L);
            upload_blocks(d_x, y);
        } else {
            upload_blocks(d_x, x);
        }
        auto base_ru = [&]() -> double {
            const Launch Lr = c.launch();
            if (partial) flush(Lr);
            c.h_state->msq_x4 = offset_low;
            c.h_state->counter = c.h_state->counter2 = 0;
            upload_state();
            dslash(Prec::Double, Lr, tmp64, x[j_low], ls64, 1 - parity);
            dslash(Prec::Double, Lr, ttt64, tmp64, ls64, parity);
            cg_true_residual(Prec::Double, Lr, ttt64, x[j_low], src, r64, c.d_state, c.d_partials, c.d_scalars);
            vec_copy(ps, resid, Prec::Double, r64, Lr);
            QB_CUDA(cudaMemcpyAsync(c.h_scalars, c.d_scalars, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
            sync_check();
            return c.h_scalars[0];
        };
        MsPass r = ms_pass(ps, partial ? Prec::Single : Prec::Double, lss, src_s, partial ? y : x, pm, ttt, tmp,
                           resid, d_x, d_p, parity, shifts, j_low, offset_low, rsq_sloppy, max_cg, false, tl,
                           floor * kShiftStopFactor, c.reliable_delta * c.reliable_delta,
                           base_ru_on ? std::function<double()>(base_ru) : std::function<double()>(), target,
                           df.get());
        if (partial) flush(c.launch());
        double t_refine = 0;
        if (c.verbose) {
            sync_check();
            t_refine = wall_seconds();
            std::fprintf(stderr, "qphix_b200 mixed multi-shift: sloppy phase %d iterations, %d reliable updates, "
                                 "%.1f ms\n", r.iteration, r.reliable_updates, 1e3 * (t_refine - info->final_sec));
        }
        rus += r.reliable_updates;
        total += r.iteration;
        last = r.iteration;
        // refinement of every shift to its own tolerance from the sloppy
        // solution.  With FP32 links the refinements take their reliable
        // updates at a quarter of the CG threshold: at 32^3x64 the iteration
        // counts are the same for 0.05, 0.1 and 0.2 while the updates drop
        // from 65 to 40 (0.826 -> 0.801 s for the whole multi-shift).  With
        // 16-bit links the updates also detect a stalled refinement (which
        // then continues in FP32), so they keep the CG threshold.
        struct DeltaScope {  // restores the threshold on every exit path
            double &d, keep;
            DeltaScope(double &v, double f) : d(v), keep(v) { d = f * v; }
            ~DeltaScope() { d = keep; }
        } refine_delta(c.reliable_delta, base_ru_on ? kRefineDeltaFactor : 1.0);
        // All shifts at once (batch_refine): one batched solve reads the
        // links once per segment of up to 32 shifts and iteration instead of
        // once per shift and iteration.  FP32 inner vectors, one GPU.
        const bool batched = ls32 && n >= 2 && n <= kBatchRefineMax && !c.halo.on && refine_batched();
        if (batched) {
            std::vector<double> mj(A.mass, A.mass + n), tj(n);
            for (int j = 0; j < n; ++j) tj[j] = A.res[j]->resid > 0 ? A.res[j]->resid : A.res[0]->resid;
            std::vector<RefineResult> rr;
            batch_refine(ls64, *ls32, src, x, mj, tj, parity, max_cg, rr);
            int longest = 0;
            for (int j = 0; j < n; ++j) {
                longest = std::max(longest, rr[j].iterations);
                rus += rr[j].reliable_updates;
                worst = std::max(worst, rr[j].true_rsq_rel);
                A.res[j]->final_rsq = rr[j].true_rsq_rel;
                A.res[j]->size_r = rr[j].true_rsq_rel;
                A.res[j]->size_relr = A.res[j]->final_rel;
                A.res[j]->final_iter = r.iteration + rr[j].iterations;
                A.res[j]->final_restart = rr[j].reliable_updates;
            }
            total += longest;
        }
        double t_shift = c.verbose ? wall_seconds() : 0.0;
        for (int j = 0; j < n && !batched; ++j) {
            const double tol = A.res[j]->resid > 0 ? A.res[j]->resid : A.res[0]->resid;
            // A refinement on 16-bit links that stagnates for
            // kRefineStallWindow inner iterations, or gains less than a
            // factor kRefineEscalate in |r|^2 over one reliable-update
            // cycle, is too ill-conditioned for them (the link rounding
            // times the condition number is near 1) and continues on FP32
            // links: at 24^3x48, m = 0.0012 the lightest refined shift
            // takes 1084 iterations on 16-bit links without this and 207
            // with it (201 on FP32 links).
            const bool r16 = rop && (rop->vec == Prec::Half || rop->links->prec == Prec::Half);
            MixedResult m = rop ? mixed_pass(rop->vec, ls64, *rop->links, rop->up, x[j], src, parity, A.mass[j], tol,
                                             max_cg, tl, 1.0 / kRefineEscalate, 1,
                                             r16 ? kRefineStallWindow : kInnerStallWindow)
                                : mixed_pass(ps, ls64, lss, ls_up, x[j], src, parity, A.mass[j], tol, max_cg, tl);
            c.stats.escalated |= m.escalated;
            total += m.iterations;
            rus += m.reliable_updates;
            worst = std::max(worst, m.true_rsq_rel);
            if (c.verbose) {
                sync_check();
                const double now = wall_seconds();
                std::fprintf(stderr, "qphix_b200 mixed multi-shift: shift %d refinement %d iterations, %d updates, "
                                     "%.2f ms\n", j, m.iterations, m.reliable_updates, 1e3 * (now - t_shift));
                if (c.verbose >= 2)
                    std::fprintf(stderr, "qphix_b200 mixed multi-shift: shift %d set-up %.2f ms, inner %.2f ms, "
                                         "updates %.2f ms, escalated %d (graph builds %.2f ms of the inner)\n", j,
                                 1e3 * m.t_setup, 1e3 * m.t_loop, 1e3 * m.t_ru, m.escalated, 1e3 * m.t_graph);
                t_shift = now;
            }
            A.res[j]->final_rsq = m.true_rsq_rel;
            A.res[j]->size_r = m.true_rsq_rel;
            A.res[j]->size_relr = A.res[j]->final_rel;
            A.res[j]->final_iter = r.iteration + m.iterations;
            A.res[j]->final_restart = m.reliable_updates;
        }
        if (c.verbose) {
            sync_check();
            std::fprintf(stderr, "qphix_b200 mixed multi-shift: %s refinement %.1f ms\n",
                         batched ? "batched" : "sequential", 1e3 * (wall_seconds() - t_refine));
        }
        if (parity0 == QPHIX_EVENODD) {
            parity = 0;
            parity0 = QPHIX_EVEN;
            src = A.in[1];
            x = A.out[1];
            continue;
        }
        break;
    }
    dev_free(d_x);
    dev_free(d_p);
    info->final_sec = wall_seconds() - info->final_sec;
    info->final_flop = (1205. + 15. * n) * total * 2.0 * c.g.vh;
    info->status = QPHIX_SUCCESS;
    c.stats.iterations = total;
    c.stats.reliable_updates = rus;
    c.stats.true_rsq = worst;
    return last;
}

}  // namespace qb
