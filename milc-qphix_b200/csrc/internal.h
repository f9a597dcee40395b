// Internal definitions of libqphix_b200: device field layouts, the global
// context, handle structures and the kernel launcher interface.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <type_traits>
#include <vector>

#include "geometry.cuh"

namespace qb {

// ----------------------------------------------------------------------------
// Field layouts in HBM (one parity block of Vh sites each)
//
// Colour vector  : 3 complex components, component-major, site-minor:
//                  c2[c*Vh + j]  (double2 / float2).  A warp reading 32
//                  consecutive sites issues one fully used 512 B / 256 B
//                  transaction per component.
// 16-bit vector  : one 16-byte record per site, int4 rec[j] = {u0|u1,
//                  u2|u3, u4|u5, norm}: the 6 reals as 16-bit fixed point q
//                  of v/norm, stored offset-binary u = q + 32768, and the
//                  float norm = max |component| of the site (per-site
//                  scaling), so a neighbour gather is one load.
// Link block     : the 16 matrices an output site needs, grouped by
//                  direction d: slot s = 0 fat forward F_d(x), 1 fat backward
//                  B_d(x), 2 Naik forward L_d(x), 3 Naik backward LB_d(x);
//                  complex c = 9*s + 3*row + col, 36 per direction, stored in
//                  16-byte chunks of k complex (k = 1 FP64, 2 FP32, 4 16-bit),
//                  chunk-major then site: chunk q of direction d is element
//                  (d*36/k + q)*Vh + j (see link_cx_index).  Every link is
//                  read once per Dslash as a coalesced 16-byte stream;
//                  nothing about links is gathered.  The block for output
//                  parity cb is built from raw sites cb*Vh + j
//                  (qphix_f3.cpp:995-1018).
// Half links     : 16-bit fixed point per real, value = q * link_max/32767,
//                  stored offset-binary u = q + 32768, with one range for the
//                  fat slots and one for the Naik slots (Naik links are ~1/24
//                  the size of fat links).
// ----------------------------------------------------------------------------
constexpr int kMats = 16;
constexpr int kLinkReals = kMats * 18;  // reals per site in a link block

// index, in complex units of the block's precision, of complex c (0..35) of
// direction d at site j; k = complex numbers per 16-byte chunk
__host__ __device__ inline size_t link_cx_index(int k, int d, int c, int j, int vh)
{
    const int C = 36 / k;
    return (((size_t)d * C + c / k) * vh + j) * k + (c % k);
}

template <typename R> struct Cx;
template <> struct Cx<double> { using type = double2; };
template <> struct Cx<float> { using type = float2; };
template <typename R> using cx_t = typename Cx<R>::type;

enum class Prec : int { Half = 0, Single = 1, Double = 2 };

// One parity block of a colour vector in device memory.
struct VecBlock {
    void *data = nullptr;   // cx_t<R>[3*Vh]   (16-bit: int4[Vh])
};

// bytes of one parity block of a colour vector
inline size_t vec_bytes(Prec p, size_t vh) { return vh * (p == Prec::Double ? 48 : (p == Prec::Single ? 24 : 16)); }

// Link blocks of both output parities.
struct LinkSet {
    void *blk[2] = {nullptr, nullptr};  // cx_t<R>[16*9*Vh] per parity (half: short2)
    float link_max[2] = {0.f, 0.f};     // half only: fixed-point range of fat / Naik links
    Prec prec = Prec::Double;           // storage precision of the blocks
    bool valid = false;
    // FP32 with compressed Naik links (recon 1: 12-real, 2: 13-real): per
    // direction the fat pair (9 float4) and rows 0-1 of the Naik pair (6
    // float4); row 2 is rebuilt as lambda * conj(row0 x row1) with
    //   recon 1: lambda = sign * recon_scale, one real magnitude for the
    //            field, the sign bits per site in sign[cb] (bit 2d: forward,
    //            2d+1: backward Naik link of d) -- SU(3) times a real factor;
    //   recon 2: lambda complex per link, lam[cb][d*Vh + j] = float4(lambda
    //            forward, lambda backward) -- U(3) times a real factor, the
    //            form of HISQ Naik links built from unitarised links.
    int recon = 0;
    float recon_scale = 0.f;
    void *sign[2] = {nullptr, nullptr};  // unsigned[Vh] per parity (recon 1)
    void *lam[2] = {nullptr, nullptr};   // float4[4*Vh] per parity (recon 2)
};

// storage tags of FP32 links with 12-real / 13-real Naik links (LinkSet::recon)
struct Recon12 {};
struct Recon13 {};
constexpr int kReconChunks = 15;  // float4 chunks per direction and site

// ----------------------------------------------------------------------------
// Device-resident scalars of a running solve.  All reductions accumulate in
// FP64 and finish in the last block of the reducing kernel, in a fixed order
// (bit-reproducible), so the host never waits inside an iteration.
// ----------------------------------------------------------------------------
constexpr int kMaxShifts = 150;  // MAXNDMASS, ks_d_congrad_fn.h:4

struct SolverState {
    // CG (ks_d_congrad_fn.cpp) and the multi-shift base system
    double rsq, oldrsq, pkp, relrsq;
    double a, b;             // step sizes, rounded to the solve precision
    double source_norm;
    double size_r, size_relr;
    double rsqmin, relrsqmin;  // stopping thresholds (squared, relative)
    double msq_x4;
    double rsqstop;
    double rsq_ru;           // mixed CG: |r|^2 at the last reliable update
    int iteration;           // the reference's `iteration`
    int niter;               // restart interval (inv_arg->max)
    int stop_at;             // chunk-local iteration at which the device stopped
    int converged;           // multi-shift: rsq <= rsqstop seen
    int prec_single;         // 1: round a, b to float like the F build
    int num_now;             // multi-shift: active shifts
    int j_low;
    int n_shifts;
    int first_iter;
    int axpy_skip_at;        // (unused) kept for layout stability
    int skip_axpy;           // mixed CG: the stopping iteration's p update waits for the host
    int use_cond;            // iterations run inside a CUDA-graph while loop
    int iter_cap;            // hard cap on st->iteration for one device run
    unsigned long long cond; // cudaGraphConditionalHandle of that loop
    int *err;                // kernel failure word (bounded waits); stops the loop
    int max_cg;              // multi-shift: iteration cap (max * nrestart)
    // mixed CG: stagnation of the inner solve.  The smallest inner |r|^2
    // since the last reliable update and the iteration it was seen; no new
    // minimum for ru_stall_window iterations forces a reliable update and
    // sets ru_stalled.
    double ru_best;
    int ru_best_iter;
    int ru_stall_window;
    int ru_stalled;
    int error;
    unsigned int counter;    // last-block counter of the grid reductions
    unsigned int counter2;
    // multi-shift recurrences (ks_multicg_offset.cpp:475-498, 587-598)
    double shifts[kMaxShifts];
    double zeta_i[kMaxShifts], zeta_im1[kMaxShifts], zeta_ip1[kMaxShifts];
    double beta_i[kMaxShifts], beta_im1[kMaxShifts], alpha[kMaxShifts];
    int finished[kMaxShifts];
    // mixed multi-shift (sloppy phase): shift k stops being updated after the
    // iteration shift_done_at[k] at which its residual zeta_k^2 |r|^2 fell to
    // shift_stop (0: never; the reference recurrence updates every shift)
    double shift_stop;
    int shift_done_at[kMaxShifts];
    // mixed multi-shift: the base shift's reliable update is due when its
    // |r|^2 falls below ms_delta2 * rsq_ru (0: never); ms_ru records that
    // the device loop stopped for it
    double ms_delta2;
    int ms_ru;
    // mixed multi-shift, deferred shift updates (ms_seg_cap > 0): iteration
    // it of the segment that began after iteration ms_seg_start stores its
    // residual and scalars in slot it - ms_seg_start - 1; the device loop
    // stops (ms_seg_full) when the last of the ms_seg_cap slots is taken
    int ms_seg_start;
    int ms_seg_cap;
    int ms_seg_full;
    // domain decomposition: this GPU's totals of the last split reduction,
    // summed in place over the GPUs before k_dd_fin reads them
    double dd_red[4];
};

// ----------------------------------------------------------------------------
// Kernel launchers (implemented in the .cu files)
// ----------------------------------------------------------------------------
struct Halo;
struct Launch {
    cudaStream_t stream;
    const Geom *g;
    int *err;                     // device word set by a kernel whose bounded wait gave up
    const Halo *halo = nullptr;   // t faces through ghost buffers (domain decomposition)
};

// out[cb] = D in[1-cb];  links = block of output parity cb
void dslash(Prec p, const Launch &L, VecBlock out, VecBlock in, const LinkSet &links, int cb);
// ttt[cb] = D tmp[1-cb] + m4 * p[cb];  state->pkp = sum p.ttt; state->a = -rsq/pkp;
// `gate`: chunk-local iteration index k, skipped when k > state->stop_at (k < 0: never)
// mode 0: CG (a from rsq/pkp), mode 1: multi-shift (shift recurrences)
void dslash_mdagm_dot(Prec p, const Launch &L, VecBlock ttt, VecBlock tmp, const LinkSet &links,
                      VecBlock pv, double m4, int cb, SolverState *st, double *partials, int gate,
                      int mode);
// plain dslash gated by the chunk iteration (first half of M^dag M)
void dslash_gated(Prec p, const Launch &L, VecBlock out, VecBlock in, const LinkSet &links,
                  int cb, SolverState *st, int gate);

// FP64 launches with a fixed variant and caller-provided scratch (no tuning,
// no allocation): out[cb] = D in[1-cb]; ttt[cb] = D tmp[1-cb] + m4 pv, p.ttt
// reduced into st->pkp through `partials`
void dslash_fixed_d(const Launch &L, VecBlock out, VecBlock in, const LinkSet &ls, int cb);
void dslash_mdagm_fixed_d(const Launch &L, VecBlock ttt, VecBlock tmp, const LinkSet &ls, VecBlock pv, double m4,
                          int cb, SolverState *st, double *partials);

// run the autotuner and one-time launch set-up for this vector/link pair now
// (required before a stream capture, which must not synchronise)
void dslash_prepare(Prec pv, const LinkSet &ls, const Launch &L);

// variant chosen by the autotuner for kernel 0 (Dslash) or 1 (fused M^dag M)
// with vectors in pv and link storage `slot` (Prec, or 3 / 4 = 12-real /
// 13-real Naik links); us = its timings; -1 before the first tuning
int dslash_variant(int kernel, Prec pv, int slot, float us[4]);
constexpr int kDslashVariants = 4;
// -1: autotuned variants; 0..2: that variant everywhere
void set_forced_variant(int v);
// poll limit of the TMA pipeline's waits (< 0: the default)
void set_wait_limit(long polls);

// BLAS (blas.cu) ---------------------------------------------------------------
// state->source_norm = |v|^2
void norm2_to_state(Prec p, const Launch &L, VecBlock v, SolverState *st, double *partials,
                    int which);
// calc_rsq (ks_d_congrad_fn.cpp:82-99): ttt += (-m4) x; r = b + ttt; p = r; rsq = |r|^2
void cg_restart_residual(Prec p, const Launch &L, VecBlock ttt, VecBlock x, VecBlock b,
                         VecBlock r, VecBlock pv, SolverState *st, double *partials, bool relres);
// calc_rsq2 (:131-147) + stop test: x += a p; r += a ttt; rsq = |r|^2 -> b, size_r
void cg_update(Prec p, const Launch &L, VecBlock x, VecBlock pv, VecBlock r, VecBlock ttt,
               SolverState *st, double *partials, int gate, bool relres);
// axpy (:178-188): p = r + b p
void cg_axpy(Prec p, const Launch &L, VecBlock r, VecBlock pv, SolverState *st, int gate);
// multi-shift: r += beta_low ttt; rsq; convergence test (ks_multicg_offset.cpp:504-520)
void ms_residual(Prec p, const Launch &L, VecBlock r, VecBlock ttt, SolverState *st,
                 double *partials, int gate);
// multi-shift: update_pm / update_dest for all active shifts in one pass
void ms_update(Prec p, const Launch &L, Prec xprec, VecBlock *x, VecBlock *pv, VecBlock r,
               int n, SolverState *st, int gate);
// One iteration's scalars of one shift, as the vector updates would use them:
// x += b p (upd bit 0), then p = z r + a p (upd bit 1).
struct MsHistEntry {
    double b, a, z;
    int upd;
};
constexpr int kMsSegMax = 256;  // iterations of one deferred segment at most

// Batched refinement (batch.cu): the systems (4 m_k^2 - D D) x_k = b of the
// library's lattice in one batched solve from the initial guesses x_k, each
// to its squared relative tolerance tol_k on the FP64 true residual; l32 is
// the 18-real FP32 copy of l64.  At most 64 systems.
struct RefineResult {
    double true_rsq_rel = 0;
    int iterations = 0, reliable_updates = 0;
};
void batch_refine(const LinkSet &l64, const LinkSet &l32, VecBlock b, const std::vector<VecBlock> &x,
                  const std::vector<double> &mass, const std::vector<double> &tol, int parity, int iter_cap,
                  std::vector<RefineResult> &out);
// multi-shift with deferred shift updates (FP32 Krylov vectors): only the
// base direction is updated, p_low = z r + a p_low; r is stored in the
// iteration's slot of `hist` (FP32 parity blocks, slot s at s * 3 Vh
// complex numbers) and every shift's scalars in hist_s[slot * n + k]
void ms_defer(const Launch &L, VecBlock p_low, VecBlock r, VecBlock hist, MsHistEntry *hist_s, int n,
              SolverState *st, int gate);
// The expansion coefficients of a deferred segment of m iterations from its
// scalar history, for the n shifts (job k = shift k; coef and jobs as
// ms_flush reads them)
void ms_coef(const Launch &L, const MsHistEntry *hist_s, int m, int n, int j_low, double *coef, int *jobs);
// End of a deferred segment of m iterations.  For every job k (jobs[k] =
// shift | do_x << 16 | do_p << 17), with c = coef + k * 2 (m + 1) and p0_s
// the shift's direction at the start of the segment:
//   x_s += c[0] p0_s + sum_t c[2 + 2t] hist_t      (x FP64)
//   p_s  = c[1] p0_s + sum_t c[3 + 2t] hist_t      (p FP32)
// (x, p0, p: device arrays indexed by shift)
void ms_flush(const Launch &L, VecBlock hist, int m, const double *coef, const int *jobs, int njobs,
              VecBlock *x, const VecBlock *p0, VecBlock *p);

// elementwise helpers
void vec_copy(Prec dst_p, VecBlock dst, Prec src_p, VecBlock src, const Launch &L);
void vec_zero(Prec p, VecBlock v, const Launch &L);
// y += x  (x in xp, y in yp; used for reliable updates x_fp64 += x_sloppy)
void vec_add(Prec yp, VecBlock y, Prec xp, VecBlock x, const Launch &L);
// r = b + (ttt - m4 x) with ttt = D D x: true residual; |r|^2 -> *out (device)
void cg_true_residual(Prec p, const Launch &L, VecBlock ttt, VecBlock x, VecBlock b, VecBlock r,
                      SolverState *st, double *partials, double *out);
// |v|^2 -> *out (device)
void norm2_dev(Prec p, const Launch &L, VecBlock v, SolverState *st, double *partials, double *out);

// Mixed-precision CG inner-loop kernels (sloppy precision p, FP64 reductions)
// state: rsq (sloppy), pkp, a, b as for CG; reliable-update trigger in host.
// x is FP32 when p is Half (see inner_x_prec)
void mx_update(Prec p, const Launch &L, VecBlock x, VecBlock pv, VecBlock r, VecBlock ttt,
               SolverState *st, double *partials, int gate, double delta2);
inline Prec inner_x_prec(Prec p) { return p == Prec::Half ? Prec::Single : p; }

// layout remap (remap.cu) -------------------------------------------------------
// raw MILC block (6 reals/site, AoS) <-> device block
void vec_from_raw(Prec p, VecBlock dst, const void *raw_dev, bool raw_double, const Launch &L);
void vec_to_raw(Prec p, void *raw_dev, bool raw_double, VecBlock src, const Launch &L);
// raw MILC link field (72 reals/site over all V sites) -> slot `slot` (0..3) of both blocks
void links_from_raw(Prec p, LinkSet &ls, const void *raw_dev, bool raw_double, int slot,
                    const Launch &L);
// slot -> raw (forward slots only are extracted by the API)
void links_to_raw(Prec p, void *raw_dev, bool raw_double, const LinkSet &ls, int slot,
                  const Launch &L);
// convert a link set between precisions (FP64 -> FP32 / half)
void links_convert(Prec dst_p, LinkSet &dst, Prec src_p, const LinkSet &src, const Launch &L);
// FP32 copy of an FP64 link set with compressed Naik links (recon.cu).
// Checks every Naik link's third row against lambda * conj(row0 x row1):
// 12-real when lambda = sign * s with one magnitude s for all links, else
// 13-real when each link has its own complex lambda; fills dst (allocated
// here) and returns its recon mode (1 or 2), or leaves dst empty and returns
// 0 when neither holds.  want = 0 takes 12-real where it holds, else
// 13-real; want = 1 or 2 asks for that form only (a 12-real field also has
// the 13-real form).  dev[0..4] receive the check's statistics (mean
// |ratio|, relative spread of |ratio|, relative imaginary part, relative
// residual of the rows rebuilt with a real ratio, and with a complex one).
int links_compress(LinkSet &dst, const LinkSet &src64, const Launch &L, double dev[5], int want = 0);
// fills ls_half.link_max[] from the ranges of `src` (fat and Naik slots)
void links_absmax(Prec p, const LinkSet &src, LinkSet &ls_half, const Launch &L, double *scratch);

}  // namespace qb
