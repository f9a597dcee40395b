// Batched solves: many CG systems on several lattices in one device run.
//
// The reference solves one system per call (QPHIX_*_asqtad_invert,
// ks_d_congrad_fn.cpp:221-619) on the one lattice QPHIX_init fixed.  A
// batch holds the gauge fields of several lattices of different sizes and
// solves (4 m_k^2 - D_eo D_oe) x_k = b_k for up to kBMaxSys systems at once:
//
//  * Systems on the same lattice form segments of nrhs = G * 2^k <= 32
//    right-hand sides (G = 1..4).  A segment's colour vectors are stored
//    site-major with the right-hand side fastest, c2[(c*Vh + j)*nrhs + r], so
//    one thread applies every link it loads to G right-hand sides: the link
//    stream -- 1152 of the 1200 bytes per site of a single-RHS FP32 Dslash --
//    is shared by the whole segment.
//  * Every kernel runs over all segments of all lattices: a resident grid
//    walks a table of 256-item tiles; per-system reductions are kept in
//    registers per segment, combined per block in shared memory and
//    finished by the last block in a fixed order (bit-reproducible).
//  * The inner CG runs in FP32; each system gets FP64 reliable updates
//    (x += x_s, r = b - M x in FP64) when its residual has dropped by the
//    reliable-update delta, and converges on its FP64 true residual.
//  * The whole solve is one CUDA-graph launch: a device-side while loop
//    over the iteration kernels and, inside it, a conditional node that
//    runs the FP64 reliable-update kernels only in iterations where some
//    system asked for one.  Without graphs (QPHIX_B200_GRAPHS=0) the host
//    enqueues iterations in chunks and the same kernels skip themselves.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "context.h"
#include "device_common.cuh"

namespace qb {

constexpr int kBMaxSys = 64;  // systems per batched solve (64-bit masks)
constexpr int kBMaxSeg = 64;
constexpr int kBMaxLat = 16;

// One segment under one kernel's thread mapping: items are (site, group of
// G right-hand sides) for the Dslash kernels and single complex numbers for
// the vector kernels.
struct BSeg {
    Geom g;
    int nrhs;         // right-hand sides (G * 2^k)
    int G;            // right-hand sides per thread
    int lg_ngrp;      // log2(groups of G right-hand sides)
    int sys0;         // first batch system of the segment
    int tile0;        // first tile of the segment
    int items;
    long long voff;   // offset of the segment in a batched field (complex numbers)
    const void *links[2];  // link blocks of output parity 0 / 1 (kernel's precision)
};

struct BTable {
    int nseg, ntiles;
    BSeg seg[kBMaxSeg];
};

struct BSys {
    double m4;        // 4 m^2
    double resid;     // squared relative tolerance
    double bnorm;     // |b|^2
    double rsqstop;   // resid * bnorm
    double rsq;       // |r|^2 of the inner iteration
    double rsq_old;   // |r|^2 one iteration earlier
    double rsq_ru;    // |r|^2 at the last reliable update
    double pkp, a, b;
    double true_rsq;  // |b - M x|^2 at the last reliable update (FP64)
    int active;       // not yet converged
    int flag;         // reliable update requested
    int iterations, reliable_updates;
};

struct BState {
    int nsys;
    int iteration, iter_cap;
    int stop;                 // the device loop has ended
    int any_flag;             // a reliable-update phase is pending
    int use_cond;
    int nonfinite;
    unsigned long long cond_loop, cond_ru;
    unsigned long long active_mask, flag_mask;
    double delta2;
    unsigned int counter;
    BSys sys[kBMaxSys];
};

struct BFields {
    double2 *x, *b, *t64;            // FP64 solution, source, Dslash scratch
    float2 *xs, *r, *p, *ap, *t32;   // FP32 inner CG
};

// ------------------------------------------------------------ tile walk --
// Shared state of one block: tile starts of the segments, the current
// segment and the per-system block sums.
template <int NV>
struct BShared {
    int tile0[kBMaxSeg + 1];
    double acc[NV > 0 ? NV : 1][kBMaxSys];
    double w[NV > 0 ? NV : 1][kBlock / 32][32];
    unsigned long long active, flag;
    double coef[2][kBMaxSys];
    BSeg seg;
    bool last;
};

template <int NV>
__device__ __forceinline__ void b_prologue(const BTable *tab, const BState *st, BShared<NV> &sh)
{
    const int nseg = tab->nseg;
    for (int i = threadIdx.x; i < nseg; i += blockDim.x) sh.tile0[i] = tab->seg[i].tile0;
    if (threadIdx.x == 0) {
        sh.tile0[nseg] = tab->ntiles;
        sh.active = st->active_mask;
        sh.flag = st->flag_mask;
    }
    for (int i = threadIdx.x; i < NV * kBMaxSys; i += blockDim.x) sh.acc[i / kBMaxSys][i % kBMaxSys] = 0.0;
}

__device__ __forceinline__ int b_seg_of(const int *tile0, int t, int cur)
{
    int s = cur < 0 ? 0 : cur;
    while (t >= tile0[s + 1]) ++s;
    return s;
}

// Moves the block to segment s (uniform call, after the caller flushed the
// previous segment's sums).
template <int NV>
__device__ __forceinline__ void b_enter(const BTable *tab, int s, BShared<NV> &sh)
{
    __syncthreads();
    if (threadIdx.x == 0) sh.seg = tab->seg[s];
    __syncthreads();
}

// Adds the per-thread sums acc[v][e] (system sys0 + q*G + e of the thread's
// group q) of the current segment into the block's per-system sums; uniform.
template <int NV>
__device__ __forceinline__ void b_flush(double (&acc)[NV][4], BShared<NV> &sh)
{
    const BSeg &sg = sh.seg;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int ngrp = 1 << sg.lg_ngrp;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            double x = acc[v][e];
            for (int o = 16; o >= ngrp; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (e < sg.G && lane < ngrp) sh.w[v][w][lane * sg.G + e] = x;
            acc[v][e] = 0.0;
        }
    }
    __syncthreads();
    if (threadIdx.x < sg.nrhs) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            double s = 0.0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += sh.w[v][k][threadIdx.x];
            sh.acc[v][sg.sys0 + threadIdx.x] += s;
        }
    }
    __syncthreads();
}

// Grid-wide end of a reducing kernel: block sums -> partials; the last block
// adds them in block order per system and calls fin(k, totals) for every
// system k (thread k), then fin_all() (thread 0).
template <int NV, typename Fin, typename FinAll>
__device__ __forceinline__ void b_finish(BShared<NV> &sh, BState *st, double *partials, Fin fin, FinAll fin_all)
{
    const int nsys = st->nsys;
    for (int i = threadIdx.x; i < NV * nsys; i += blockDim.x) {
        const int v = i / nsys, k = i % nsys;
        partials[((size_t)v * kBMaxSys + k) * gridDim.x + blockIdx.x] = sh.acc[v][k];
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) sh.last = (atomicAdd(&st->counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!sh.last) return;
    __threadfence();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int i = w; i < NV * nsys; i += nw) {
        const int v = i / nsys, k = i % nsys;
        const double *p = partials + ((size_t)v * kBMaxSys + k) * gridDim.x;
        double s = 0.0;
        for (int b = lane; b < (int)gridDim.x; b += 32) s += __ldcg(p + b);
        s = warp_sum(s);
        if (lane == 0) sh.acc[v][k] = s;
    }
    __syncthreads();
    if (threadIdx.x < nsys) {
        double t[NV > 0 ? NV : 1];
#pragma unroll
        for (int v = 0; v < NV; ++v) t[v] = sh.acc[v][threadIdx.x];
        fin(threadIdx.x, t);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        fin_all();
        st->counter = 0;
        __threadfence();
    }
}

// masks over the batch systems after a per-system step
__device__ __forceinline__ void b_masks(BState *st)
{
    unsigned long long a = 0, f = 0;
    for (int k = 0; k < st->nsys; ++k) {
        if (st->sys[k].active) a |= 1ull << k;
        if (st->sys[k].flag) f |= 1ull << k;
    }
    st->active_mask = a;
    st->flag_mask = f;
}

// ------------------------------------------------- multi-RHS vector loads --
// 32-byte loads and stores (sm_100): four right-hand sides of one colour
// component in one instruction, so the four threads of a site move a whole
// 128-byte line each time.  The addresses are 32-byte aligned: segments of
// four or more systems start on multiples of 24 * Vh * nrhs bytes and Vh is
// a multiple of 128.  Read-only data of the launch only (non-coherent path).
__device__ __forceinline__ void ld_nc_v8(const float2 *p, float w[8])
{
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(w[0]), "=f"(w[1]), "=f"(w[2]), "=f"(w[3]), "=f"(w[4]), "=f"(w[5]), "=f"(w[6]), "=f"(w[7])
        : "l"(p));
}

__device__ __forceinline__ void st_v8(float2 *p, const float w[8])
{
    asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(w[0]), "f"(w[1]), "f"(w[2]),
                 "f"(w[3]), "f"(w[4]), "f"(w[5]), "f"(w[6]), "f"(w[7])
                 : "memory");
}

template <int G>
__device__ __forceinline__ void bload(const float2 *f, int vh, int nrhs, int j, int q, float v[G][6])
{
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float2 *p = f + ((size_t)(c * vh + j) * nrhs + q * G);
        if constexpr (G == 4) {
            float w[8];
            ld_nc_v8(p, w);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                v[e][2 * c] = w[2 * e];
                v[e][2 * c + 1] = w[2 * e + 1];
            }
        } else if constexpr (G % 2 == 1) {
#pragma unroll
            for (int e = 0; e < G; ++e) {
                const float2 z = __ldg(p + e);
                v[e][2 * c] = z.x; v[e][2 * c + 1] = z.y;
            }
        } else {
#pragma unroll
            for (int e = 0; e < G; e += 2) {
                const float4 z = __ldg(reinterpret_cast<const float4 *>(p + e));
                v[e][2 * c] = z.x; v[e][2 * c + 1] = z.y;
                v[e + 1][2 * c] = z.z; v[e + 1][2 * c + 1] = z.w;
            }
        }
    }
}

template <int G>
__device__ __forceinline__ void bstore(float2 *f, int vh, int nrhs, int j, int q, const float v[G][6])
{
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float2 *p = f + ((size_t)(c * vh + j) * nrhs + q * G);
        if constexpr (G == 4) {
            float w[8];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                w[2 * e] = v[e][2 * c];
                w[2 * e + 1] = v[e][2 * c + 1];
            }
            st_v8(p, w);
        } else if constexpr (G % 2 == 1) {
#pragma unroll
            for (int e = 0; e < G; ++e) p[e] = make_float2(v[e][2 * c], v[e][2 * c + 1]);
        } else {
#pragma unroll
            for (int e = 0; e < G; e += 2)
                *reinterpret_cast<float4 *>(p + e) =
                    make_float4(v[e][2 * c], v[e][2 * c + 1], v[e + 1][2 * c], v[e + 1][2 * c + 1]);
        }
    }
}

template <int G>
__device__ __forceinline__ void bload(const double2 *f, int vh, int nrhs, int j, int q, double v[G][6])
{
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double2 *p = f + ((size_t)(c * vh + j) * nrhs + q * G);
#pragma unroll
        for (int e = 0; e < G; ++e) {
            const double2 z = __ldg(p + e);
            v[e][2 * c] = z.x; v[e][2 * c + 1] = z.y;
        }
    }
}

template <int G>
__device__ __forceinline__ void bstore(double2 *f, int vh, int nrhs, int j, int q, const double v[G][6], unsigned mask)
{
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double2 *p = f + ((size_t)(c * vh + j) * nrhs + q * G);
#pragma unroll
        for (int e = 0; e < G; ++e)
            if (mask >> e & 1u) p[e] = make_double2(v[e][2 * c], v[e][2 * c + 1]);
    }
}

// -------------------------------------------------- multi-RHS Dslash site --
// The FP32 multi-RHS site is bound by the FP32 pipe rather than by HBM, so
// its complex multiply-adds are written as explicit FMA chains: two FFMAs
// per real product pair, where acc += a*b - c*d compiles to FMUL, FFMA and
// FADD.  (The rounding order differs from mv_add by one FP32 ulp per term.)
__device__ __forceinline__ void fmv_add(float acc[6], const float u[18], const float v[6])
{
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float ur = u[6 * r + 2 * c], ui = u[6 * r + 2 * c + 1];
            acc[2 * r] = __fmaf_rn(ur, v[2 * c], acc[2 * r]);
            acc[2 * r] = __fmaf_rn(-ui, v[2 * c + 1], acc[2 * r]);
            acc[2 * r + 1] = __fmaf_rn(ur, v[2 * c + 1], acc[2 * r + 1]);
            acc[2 * r + 1] = __fmaf_rn(ui, v[2 * c], acc[2 * r + 1]);
        }
    }
}

// acc -= U^dag v
__device__ __forceinline__ void fmv_adj_sub(float acc[6], const float u[18], const float v[6])
{
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float ur = u[6 * c + 2 * r], ui = u[6 * c + 2 * r + 1];
            acc[2 * r] = __fmaf_rn(-ur, v[2 * c], acc[2 * r]);
            acc[2 * r] = __fmaf_rn(-ui, v[2 * c + 1], acc[2 * r]);
            acc[2 * r + 1] = __fmaf_rn(-ur, v[2 * c + 1], acc[2 * r + 1]);
            acc[2 * r + 1] = __fmaf_rn(ui, v[2 * c], acc[2 * r + 1]);
        }
    }
}

// acc[e] = (D in)(site j) for the G right-hand sides of group q
template <int G>
__device__ __forceinline__ void bsite(const BSeg &sg, int cb, int j, int q, const float2 *in, float acc[G][6])
{
    const SiteCoords s = decode(sg.g, cb, j);
    const LinkView<float> lv{static_cast<const float4 *>(sg.links[cb]), sg.g.vh};
#pragma unroll
    for (int e = 0; e < G; ++e)
#pragma unroll
        for (int i = 0; i < 6; ++i) acc[e][i] = 0.f;
    // A forward/backward pair is 9 float4 chunks (18 complex); the forward
    // matrix is in chunks 0-4 and the backward one in chunks 4-8 (chunk 4
    // holds the last forward and the first backward complex).  Loading five
    // chunks per matrix keeps 20 link floats live instead of 36, which leaves
    // registers for the G right-hand sides.  Sixteen stages (one matrix and
    // its neighbour each), software-pipelined: the loads of stage i + 1 are
    // issued before the arithmetic of stage i.
    float4 wc[2][5];
    float v[2][G][6];
    auto issue = [&](int st, int b) {
        const int d = st >> 2, h = (st >> 1) & 1, half = st & 1;
        const float4 *pair = lv.p + ((size_t)d * 18 + 9 * h) * lv.vh + j;
#pragma unroll
        for (int c = 0; c < 5; ++c) wc[b][c] = __ldcs(pair + (size_t)(4 * half + c) * lv.vh);
        bload<G>(in, sg.g.vh, sg.nrhs, neighbor(sg.g, s, 8 * h + 2 * d + (half ? 0 : 1)), q, v[b]);
    };
    issue(0, 0);
#pragma unroll
    for (int st = 0; st < 16; ++st) {
        const int b = st & 1;
        if (st + 1 < 16) issue(st + 1, b ^ 1);
        float w[20];
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            w[4 * c] = wc[b][c].x; w[4 * c + 1] = wc[b][c].y; w[4 * c + 2] = wc[b][c].z; w[4 * c + 3] = wc[b][c].w;
        }
#pragma unroll
        for (int e = 0; e < G; ++e) {
            if (st & 1) fmv_adj_sub(acc[e], w + 2, v[b][e]);
            else fmv_add(acc[e], w, v[b][e]);
        }
    }
}

template <int G>
__device__ __forceinline__ void bsite(const BSeg &sg, int cb, int j, int q, const double2 *in, double acc[G][6])
{
    const SiteCoords s = decode(sg.g, cb, j);
    const LinkView<double> lv{static_cast<const double2 *>(sg.links[cb]), sg.g.vh};
#pragma unroll
    for (int e = 0; e < G; ++e)
#pragma unroll
        for (int i = 0; i < 6; ++i) acc[e][i] = 0.0;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
#pragma unroll
        for (int sl = 0; sl < 4; ++sl) {
            const int k = (sl < 2 ? 0 : 8) + 2 * d + (sl & 1 ? 0 : 1);
            double u[18], v[G][6];
            lv.load_mat(d, sl, j, u);
            bload<G>(in, sg.g.vh, sg.nrhs, neighbor(sg.g, s, k), q, v);
#pragma unroll
            for (int e = 0; e < G; ++e) {
                if (sl & 1) mv_adj_sub(acc[e], u, v[e]);
                else mv_add(acc[e], u, v[e]);
            }
        }
    }
}

// ------------------------------------------------ FP32 inner Dslash (K1/K2) --
// MDAGM = false: out = D in.   MDAGM = true: out = m4 p - D in (= M p with
// in = D p), p.(M p) reduced per system -> a = rsq / pkp.
// Groups whose systems have all converged are skipped.
template <int G, bool MDAGM>
__device__ __forceinline__ void bdslash_s_item(int item, int cb, float2 *out, const float2 *in, const float2 *pv,
                                               const BShared<1> &sh, double (&acc)[1][4])
{
    const BSeg &sg = sh.seg;
    const int q = item & ((1 << sg.lg_ngrp) - 1);
    const int j = item >> sg.lg_ngrp;
    const unsigned act = (unsigned)((sh.active >> (sg.sys0 + q * G)) & ((1ull << G) - 1ull));
    if (!act) return;
    float a[G][6];
    bsite<G>(sg, cb, j, q, in + sg.voff, a);
    if constexpr (MDAGM) {
        float p[G][6];
        bload<G>(pv + sg.voff, sg.g.vh, sg.nrhs, j, q, p);
#pragma unroll
        for (int e = 0; e < G; ++e) {
            const float m4 = (float)sh.coef[0][sg.sys0 + q * G + e];
            float dot = 0.f;
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                a[e][i] = m4 * p[e][i] - a[e][i];
                dot += p[e][i] * a[e][i];
            }
            acc[0][e] += (double)dot;
        }
    }
    bstore<G>(out + sg.voff, sg.g.vh, sg.nrhs, j, q, a);
}

// GMAX: largest G of the table's segments.  With G = 1 the kernel fits in
// 64 registers (4 blocks of 256 per SM), with G = 2 in 80 (3 blocks); G = 3,
// 4 need 128 (2 blocks).
template <bool MDAGM, int GMAX>
__global__ void __launch_bounds__(kBlock, GMAX == 1 ? 4 : (GMAX == 2 ? 3 : 2)) k_bdslash_s(const BTable *tab, BState *st, float2 *out,
                                                         const float2 *in, const float2 *pv, int cb,
                                                         double *partials)
{
    __shared__ BShared<1> sh;
    // the first kernel of an iteration ends the graph's while loop once the
    // solve has stopped
    if (!MDAGM && blockIdx.x == 0 && threadIdx.x == 0 && st->use_cond && *(volatile int *)&st->stop)
        cudaGraphSetConditional(st->cond_loop, 0);
    if (*(volatile int *)&st->stop) return;
    b_prologue(tab, st, sh);
    if (MDAGM)
        for (int k = threadIdx.x; k < st->nsys; k += blockDim.x) sh.coef[0][k] = st->sys[k].m4;
    __syncthreads();
    double acc[1][4] = {{0, 0, 0, 0}};
    int cur = -1;
    for (int t = blockIdx.x; t < tab->ntiles; t += gridDim.x) {
        const int s = b_seg_of(sh.tile0, t, cur);
        if (s != cur) {
            if (MDAGM && cur >= 0) b_flush<1>(acc, sh);
            cur = s;
            b_enter(tab, s, sh);
        }
        const int item = (t - sh.seg.tile0) * kBlock + threadIdx.x;
        if (item < sh.seg.items) {
            if constexpr (GMAX > 2) {
                if (sh.seg.G == 4) bdslash_s_item<4, MDAGM>(item, cb, out, in, pv, sh, acc);
                else if (sh.seg.G == 3) bdslash_s_item<3, MDAGM>(item, cb, out, in, pv, sh, acc);
            }
            if constexpr (GMAX > 1) {
                if (sh.seg.G == 2) bdslash_s_item<2, MDAGM>(item, cb, out, in, pv, sh, acc);
            }
            if (sh.seg.G == 1) bdslash_s_item<1, MDAGM>(item, cb, out, in, pv, sh, acc);
        }
    }
    if constexpr (MDAGM) {
        if (cur >= 0) b_flush<1>(acc, sh);
        b_finish<1>(
            sh, st, partials,
            [&](int k, const double *t) {
                BSys &y = st->sys[k];
                if (!y.active) return;
                y.pkp = t[0];
                y.a = t[0] > 0.0 ? y.rsq / t[0] : 0.0;
                // p.(M p) <= 0 or not finite: breakdown of system k (M is
                // positive definite for m > 0); the whole batch stops
                if (!(t[0] > 0.0) || !isfinite(t[0])) {
                    st->nonfinite = isfinite(t[0]) ? 2 : 1;
                    st->stop = 1;
                }
            },
            [&] {});
    }
}

// ------------------------------------- FP64 reliable-update Dslash (R1/R2) --
// Only groups holding a flagged system run; only flagged systems are stored.
// RESID = false: out = D in.   RESID = true: with in = D x, the FP64 residual
// r = b - (m4 x - D in) is stored in FP32 into f.r and |r|^2 reduced per
// system (the reliable update's true residual).
template <int G, bool RESID>
__device__ __forceinline__ void bdslash_d_item(int item, int cb, double2 *out, const double2 *in, const BFields &f,
                                               const BShared<1> &sh, double (&acc)[1][4])
{
    const BSeg &sg = sh.seg;
    const int q = item & ((1 << sg.lg_ngrp) - 1);
    const int j = item >> sg.lg_ngrp;
    const unsigned mask = (unsigned)((sh.flag >> (sg.sys0 + q * G)) & ((1ull << G) - 1ull));
    if (!mask) return;
    double a[G][6];
    bsite<G>(sg, cb, j, q, in + sg.voff, a);
    if constexpr (!RESID) {
        bstore<G>(out + sg.voff, sg.g.vh, sg.nrhs, j, q, a, mask);
    } else {
        double x[G][6], b[G][6];
        bload<G>(f.x + sg.voff, sg.g.vh, sg.nrhs, j, q, x);
        bload<G>(f.b + sg.voff, sg.g.vh, sg.nrhs, j, q, b);
        float2 *r = f.r + sg.voff;
#pragma unroll
        for (int e = 0; e < G; ++e) {
            if (!(mask >> e & 1u)) continue;
            const double m4 = sh.coef[0][sg.sys0 + q * G + e];
            double n = 0.0;
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                a[e][i] = b[e][i] - (m4 * x[e][i] - a[e][i]);
                n += a[e][i] * a[e][i];
            }
            acc[0][e] += n;
#pragma unroll
            for (int c = 0; c < 3; ++c)
                r[(size_t)(c * sg.g.vh + j) * sg.nrhs + q * G + e] =
                    make_float2((float)a[e][2 * c], (float)a[e][2 * c + 1]);
        }
    }
}

template <bool RESID>
__global__ void __launch_bounds__(kBlock, 2) k_bdslash_d(const BTable *tab, BState *st, double2 *out,
                                                         const double2 *in, BFields f, int cb, double *partials)
{
    __shared__ BShared<1> sh;
    if (!*(volatile int *)&st->any_flag) return;
    b_prologue(tab, st, sh);
    if (RESID)
        for (int k = threadIdx.x; k < st->nsys; k += blockDim.x) sh.coef[0][k] = st->sys[k].m4;
    __syncthreads();
    double acc[1][4] = {{0, 0, 0, 0}};
    int cur = -1;
    for (int t = blockIdx.x; t < tab->ntiles; t += gridDim.x) {
        const int s = b_seg_of(sh.tile0, t, cur);
        if (s != cur) {
            if (RESID && cur >= 0) b_flush<1>(acc, sh);
            cur = s;
            b_enter(tab, s, sh);
        }
        const int item = (t - sh.seg.tile0) * kBlock + threadIdx.x;
        if (item < sh.seg.items) {
            switch (sh.seg.G) {
            case 3: bdslash_d_item<3, RESID>(item, cb, out, in, f, sh, acc); break;
            case 2: bdslash_d_item<2, RESID>(item, cb, out, in, f, sh, acc); break;
            default: bdslash_d_item<1, RESID>(item, cb, out, in, f, sh, acc); break;
            }
        }
    }
    if constexpr (RESID) {
        if (cur >= 0) b_flush<1>(acc, sh);
        b_finish<1>(
            sh, st, partials,
            [&](int k, const double *t) {
                BSys &y = st->sys[k];
                if (!y.flag) return;
                y.reliable_updates += 1;
                y.true_rsq = t[0];
                const bool finite = (t[0] == t[0]) && t[0] < 1e300;
                if (!finite) st->nonfinite = 1;
                if (t[0] <= y.rsqstop || !finite) {
                    y.active = 0;
                    y.flag = 0;
                } else {
                    y.b = y.rsq_old > 0.0 ? t[0] / y.rsq_old : 0.0;
                    y.rsq = t[0];
                    y.rsq_ru = t[0];
                }
            },
            [&] {
                // flag_mask stays: the p update of the reliable update needs it
                unsigned long long a = 0;
                for (int k = 0; k < st->nsys; ++k)
                    if (st->sys[k].active) a |= 1ull << k;
                st->active_mask = a;
                if (a == 0 || st->nonfinite) st->stop = 1;
            });
    }
}

// ------------------------------------------------------ vector kernels --
// Items are (complex number of a segment's (component, site) space, group
// of G right-hand sides); system = sys0 + q*G + e.
enum BOp : int {
    kBNormB = 0,    // |b|^2 -> bnorm, rsqstop, flags of the first reliable update
    kBUpdate = 1,   // x_s += a p, r -= a Ap, |r|^2 -> b, reliable-update flags
    kBAxpy = 2,     // p = r + b p   (active systems without a pending update)
    kBAccum = 3,    // x += x_s, x_s = 0   (flagged systems)
    kBAxpyRu = 4,   // p = r + b p   (flagged active systems; closes the update)
};

template <int OP>
__global__ void __launch_bounds__(kBlock) k_bvec(const BTable *tab, BState *st, BFields f, double *partials)
{
    constexpr int NV = (OP == kBNormB || OP == kBUpdate) ? 1 : 0;
    __shared__ BShared<NV> sh;
    if constexpr (OP == kBUpdate || OP == kBAxpy) {
        if (*(volatile int *)&st->stop) return;
    }
    if constexpr (OP == kBAccum || OP == kBAxpyRu) {
        if (!*(volatile int *)&st->any_flag) return;
    }
    b_prologue(tab, st, sh);
    for (int k = threadIdx.x; k < st->nsys; k += blockDim.x) {
        sh.coef[0][k] = st->sys[k].a;
        sh.coef[1][k] = st->sys[k].b;
    }
    __syncthreads();
    unsigned long long mask;
    if (OP == kBNormB) mask = ~0ull;
    else if (OP == kBUpdate) mask = sh.active;
    else if (OP == kBAxpy) mask = sh.active & ~sh.flag;
    else if (OP == kBAccum) mask = sh.flag;
    else mask = sh.flag & sh.active;
    double acc[NV > 0 ? NV : 1][4] = {{0, 0, 0, 0}};
    int cur = -1;
    for (int t = blockIdx.x; t < tab->ntiles; t += gridDim.x) {
        const int s = b_seg_of(sh.tile0, t, cur);
        if (s != cur) {
            if constexpr (NV > 0)
                if (cur >= 0) b_flush<NV>(acc, sh);
            cur = s;
            b_enter(tab, s, sh);
        }
        const BSeg &sg = sh.seg;
        const int item = (t - sg.tile0) * kBlock + threadIdx.x;
        if (item >= sg.items) continue;
        // item = (complex number of the (component, site) space, group q);
        // the thread handles the G right-hand sides of its group
        const int q = item & ((1 << sg.lg_ngrp) - 1);
        const size_t base = sg.voff + (size_t)(item >> sg.lg_ngrp) * sg.nrhs + q * sg.G;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            if (e >= sg.G) break;
            const int k = sg.sys0 + q * sg.G + e;
            if (!(mask >> k & 1ull)) continue;
            const size_t i = base + e;
            if constexpr (OP == kBNormB) {
                const double2 z = f.b[i];
                acc[0][e] += z.x * z.x + z.y * z.y;
            } else if constexpr (OP == kBUpdate) {
                const float a = (float)sh.coef[0][k];
                const float2 p = f.p[i], ap = f.ap[i];
                float2 x = f.xs[i], r = f.r[i];
                x.x += a * p.x; x.y += a * p.y;
                r.x -= a * ap.x; r.y -= a * ap.y;
                f.xs[i] = x;
                f.r[i] = r;
                acc[0][e] += (double)(r.x * r.x + r.y * r.y);
            } else if constexpr (OP == kBAxpy || OP == kBAxpyRu) {
                const float b = (float)sh.coef[1][k];
                const float2 r = f.r[i];
                float2 p = f.p[i];
                p.x = r.x + b * p.x;
                p.y = r.y + b * p.y;
                f.p[i] = p;
            } else {
                const float2 xs = f.xs[i];
                double2 x = f.x[i];
                x.x += (double)xs.x;
                x.y += (double)xs.y;
                f.x[i] = x;
                f.xs[i] = make_float2(0.f, 0.f);
            }
        }
    }
    if constexpr (NV > 0) {
        if (cur >= 0) b_flush<NV>(acc, sh);
        if constexpr (OP == kBNormB) {
            b_finish<1>(
                sh, st, partials,
                [&](int k, const double *t) {
                    BSys &y = st->sys[k];
                    y.bnorm = t[0];
                    y.rsqstop = y.resid * t[0];
                    y.active = t[0] > 0.0;
                    y.flag = y.active;
                    if (!isfinite(t[0])) st->nonfinite = 1;  // a source with NaN or Inf
                },
                [&] {
                    b_masks(st);
                    st->any_flag = st->flag_mask != 0;
                    st->stop = st->active_mask == 0 || st->nonfinite;
                });
        } else {
            b_finish<1>(
                sh, st, partials,
                [&](int k, const double *t) {
                    BSys &y = st->sys[k];
                    if (!y.active) { y.flag = 0; return; }
                    y.rsq_old = y.rsq;
                    y.rsq = t[0];
                    y.b = y.rsq_old > 0.0 ? t[0] / y.rsq_old : 0.0;
                    y.iterations += 1;
                    y.flag = (t[0] < st->delta2 * y.rsq_ru || t[0] <= y.rsqstop || !(t[0] == t[0])) ? 1 : 0;
                    if (!isfinite(t[0])) st->nonfinite = 1;
                },
                [&] {
                    b_masks(st);
                    st->any_flag = st->flag_mask != 0;
                    st->iteration += 1;
                    if (st->use_cond) cudaGraphSetConditional(st->cond_ru, st->any_flag ? 1u : 0u);
                    if (st->iteration >= st->iter_cap || st->nonfinite) st->stop = 1;
                });
        }
    } else if constexpr (OP == kBAxpyRu) {
        // the last block to finish closes the reliable-update phase
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            if (atomicAdd(&st->counter, 1u) == gridDim.x - 1) {
                for (int k = 0; k < st->nsys; ++k) st->sys[k].flag = 0;
                st->flag_mask = 0;
                st->any_flag = 0;
                st->counter = 0;
                __threadfence();
            }
        }
    }
}

// raw MILC parity block (6 reals per site) <-> slot r of a segment
__global__ void k_b_from_raw(double2 *f, long long voff, int vh, int nrhs, int r, const double *raw)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= vh) return;
#pragma unroll
    for (int c = 0; c < 3; ++c)
        f[voff + (size_t)(c * vh + j) * nrhs + r] = make_double2(raw[6 * (size_t)j + 2 * c], raw[6 * (size_t)j + 2 * c + 1]);
}

__global__ void k_b_to_raw(double *raw, const double2 *f, long long voff, int vh, int nrhs, int r)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= vh) return;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double2 z = f[voff + (size_t)(c * vh + j) * nrhs + r];
        raw[6 * (size_t)j + 2 * c] = z.x;
        raw[6 * (size_t)j + 2 * c + 1] = z.y;
    }
}

// FP64 parity block of the library's vector layout (complex e = c*Vh + j)
// <-> slot r of a segment
__global__ void k_b_from_blk(double2 *f, long long voff, int n3, int nrhs, int r, const double2 *v)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n3) f[voff + (size_t)e * nrhs + r] = v[e];
}

__global__ void k_b_to_blk(double2 *v, const double2 *f, long long voff, int n3, int nrhs, int r)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n3) v[e] = f[voff + (size_t)e * nrhs + r];
}

}  // namespace qb

// FP64 <-> FP32 copy of a whole batched field (n complex numbers)
__global__ void k_b_narrow(float2 *dst, const double2 *src, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = make_float2((float)src[i].x, (float)src[i].y);
}
__global__ void k_b_widen(double2 *dst, const float2 *src, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = make_double2((double)src[i].x, (double)src[i].y);
}

// ------------------------------------------------------------------ host --
struct QPHIX_B200_Batch_struct {
    struct Lat {
        int dims[4];
        qb::Geom g;
        qb::LinkSet l64, l32;
    };
    std::vector<Lat> lats;
};

namespace qb {
namespace {

template <typename K>
int resident_blocks(K kernel)
{
    int per_sm = 0, sms = 0, dev = 0;
    QB_CUDA(cudaGetDevice(&dev));
    QB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    QB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, 0));
    return std::max(1, per_sm) * sms;
}

// one lattice of a batched solve: geometry and its FP64 / FP32 link blocks
struct LatRef {
    const Geom *g;
    const LinkSet *l64, *l32;
};

struct SegPlan {
    int lat, nrhs, sys0;
    std::vector<int> user;  // caller's system index of each slot
};

int log2i(int n)
{
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

// Segment sizes: G * 2^k with G = 1..4 right-hand sides per thread, so that
// every kernel's groups per site are a power of two (warp-shuffle sums).
constexpr int kSegSizes[] = {32, 24, 16, 12, 8, 6, 4, 3, 2, 1};

// Systems of each lattice in segments of the largest allowed size first;
// slot_of[k] = batch slot of caller system k.
std::vector<SegPlan> plan_segments(int nlat, int nsys, const int *lat, std::vector<int> &slot_of)
{
    std::vector<SegPlan> plan;
    slot_of.assign(nsys, 0);
    int sys = 0;
    for (int l = 0; l < nlat; ++l) {
        std::vector<int> mine;
        for (int k = 0; k < nsys; ++k)
            if (lat[k] == l) mine.push_back(k);
        size_t pos = 0;
        while (pos < mine.size()) {
            int n = 1;
            for (int sz : kSegSizes)
                if (sz <= (int)(mine.size() - pos)) { n = sz; break; }
            SegPlan p{l, n, sys, {}};
            for (int r = 0; r < n; ++r) {
                p.user.push_back(mine[pos + r]);
                slot_of[mine[pos + r]] = sys + r;
            }
            sys += n;
            pos += n;
            plan.push_back(p);
        }
    }
    if ((int)plan.size() > kBMaxSeg) throw Error("batch: too many segments");
    return plan;
}

// kind 0: FP32 Dslash (G = 3 for multiples of 3, else <= 4; measured: G = 4
// at 2 blocks/SM beats G = 2 at 3 blocks/SM by 4-5 %), 1: FP64 Dslash (G = 3
// for multiples of 3, else <= 2), 2: vector kernels
BTable make_table(const std::vector<SegPlan> &plan, const std::vector<LatRef> &lats, int kind, int gpref = 4)
{
    BTable t{};
    t.nseg = (int)plan.size();
    long long voff = 0;
    int tile = 0;
    for (int s = 0; s < t.nseg; ++s) {
        const SegPlan &p = plan[s];
        const LatRef &L = lats[p.lat];
        const int n = p.nrhs;
        BSeg &g = t.seg[s];
        g.g = *L.g;
        g.nrhs = n;
        g.sys0 = p.sys0;
        g.voff = voff;
        voff += 3LL * L.g->vh * n;
        if (kind == 2) {
            int ngrp = 1;
            while (ngrp < 32 && n % (2 * ngrp) == 0) ngrp *= 2;
            g.G = n / ngrp;
            g.lg_ngrp = log2i(ngrp);
            g.items = 3 * L.g->vh * ngrp;
        } else {
            g.G = (n % 3 == 0) ? 3 : std::min(n, kind == 0 ? gpref : 2);
            g.lg_ngrp = log2i(n / g.G);
            g.items = L.g->vh * (n / g.G);
            const LinkSet &ls = kind == 0 ? *L.l32 : *L.l64;
            g.links[0] = ls.blk[0];
            g.links[1] = ls.blk[1];
        }
        g.tile0 = tile;
        tile += (g.items + kBlock - 1) / kBlock;
    }
    t.ntiles = tile;
    return t;
}

BState *pinned_state()
{
    static BState *h = nullptr;
    if (!h) QB_CUDA(cudaMallocHost(&h, sizeof(BState)));
    return h;
}

// QPHIX_B200_BATCH_G=4|2|1 skips the batched-Dslash tuning and uses that
// many systems per thread where the segment size allows it
int batch_tuning_forced()
{
    const char *e = std::getenv("QPHIX_B200_BATCH_G");
    return (e && (e[0] == '4' || e[0] == '2' || e[0] == '1')) ? e[0] - '0' : 0;
}

int last_batch_g = 0;  // systems per thread of the last batched solve's FP32 Dslash

bool batch_graphs_enabled()
{
    const char *e = std::getenv("QPHIX_B200_GRAPHS");
    return !(e && e[0] == '0');
}

struct BatchRun {
    const BTable *tab_s, *tab_d, *tab_v;
    int grid_s0, grid_s1, grid_d0, grid_d1, grid_v[5];
    int gmax_s;  // largest right-hand sides per thread of the FP32 Dslash table
    BState *st;
    BFields f;
    double *partials;
    int cb, other;
    cudaStream_t stream;

    // R0..R3: x += x_s; r = b - M x in FP64; p = r + b p (flagged systems)
    void reliable_update() const
    {
        k_bvec<kBAccum><<<grid_v[kBAccum], kBlock, 0, stream>>>(tab_v, st, f, partials);
        k_bdslash_d<false><<<grid_d0, kBlock, 0, stream>>>(tab_d, st, f.t64, f.x, f, other, partials);
        k_bdslash_d<true><<<grid_d1, kBlock, 0, stream>>>(tab_d, st, nullptr, f.t64, f, cb, partials);
        k_bvec<kBAxpyRu><<<grid_v[kBAxpyRu], kBlock, 0, stream>>>(tab_v, st, f, partials);
    }
    // K1..K4: one FP32 CG iteration of every active system
    void iteration() const
    {
        if (gmax_s > 2) {
            k_bdslash_s<false, 4><<<grid_s0, kBlock, 0, stream>>>(tab_s, st, f.t32, f.p, f.p, other, partials);
            k_bdslash_s<true, 4><<<grid_s1, kBlock, 0, stream>>>(tab_s, st, f.ap, f.t32, f.p, cb, partials);
        } else if (gmax_s == 2) {
            k_bdslash_s<false, 2><<<grid_s0, kBlock, 0, stream>>>(tab_s, st, f.t32, f.p, f.p, other, partials);
            k_bdslash_s<true, 2><<<grid_s1, kBlock, 0, stream>>>(tab_s, st, f.ap, f.t32, f.p, cb, partials);
        } else {
            k_bdslash_s<false, 1><<<grid_s0, kBlock, 0, stream>>>(tab_s, st, f.t32, f.p, f.p, other, partials);
            k_bdslash_s<true, 1><<<grid_s1, kBlock, 0, stream>>>(tab_s, st, f.ap, f.t32, f.p, cb, partials);
        }
        k_bvec<kBUpdate><<<grid_v[kBUpdate], kBlock, 0, stream>>>(tab_v, st, f, partials);
        k_bvec<kBAxpy><<<grid_v[kBAxpy], kBlock, 0, stream>>>(tab_v, st, f, partials);
    }
};

// One CUDA graph: while (cond_loop) { if (cond_ru) { R0..R3 }; K1..K4 }.
// cond_ru starts at 1 (the first pass forms every system's true residual);
// K3 sets it each iteration, K1 clears cond_loop once the solve stopped.
struct BatchGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphConditionalHandle hloop = 0, hru = 0;
    ~BatchGraph()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
    void build(const BatchRun &R)
    {
        QB_CUDA(cudaGraphCreate(&graph, 0));
        QB_CUDA(cudaGraphConditionalHandleCreate(&hloop, graph, 1, cudaGraphCondAssignDefault));
        QB_CUDA(cudaGraphConditionalHandleCreate(&hru, graph, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams wp = {};
        wp.type = cudaGraphNodeTypeConditional;
        wp.conditional.handle = hloop;
        wp.conditional.type = cudaGraphCondTypeWhile;
        wp.conditional.size = 1;
        cudaGraphNode_t wnode;
        QB_CUDA(cudaGraphAddNode(&wnode, graph, nullptr, 0, &wp));
        cudaGraph_t body = wp.conditional.phGraph_out[0];
        cudaGraphNodeParams ip = {};
        ip.type = cudaGraphNodeTypeConditional;
        ip.conditional.handle = hru;
        ip.conditional.type = cudaGraphCondTypeIf;
        ip.conditional.size = 1;
        cudaGraphNode_t inode;
        QB_CUDA(cudaGraphAddNode(&inode, body, nullptr, 0, &ip));
        cudaGraph_t rbody = ip.conditional.phGraph_out[0];
        capture(R.stream, rbody, nullptr, [&] { R.reliable_update(); });
        capture(R.stream, body, &inode, [&] { R.iteration(); });
        QB_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    }
    template <typename F>
    static void capture(cudaStream_t s, cudaGraph_t g, const cudaGraphNode_t *dep, F enqueue)
    {
        QB_CUDA(cudaStreamBeginCaptureToGraph(s, g, dep, nullptr, dep ? 1 : 0, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue();
        } catch (...) {
            cudaGraph_t dummy;
            cudaStreamEndCapture(s, &dummy);
            throw;
        }
        QB_CUDA(cudaStreamEndCapture(s, &g));
    }
};

void upload(BState *d, const BState *h, cudaStream_t s)
{
    QB_CUDA(cudaMemcpyAsync(d, h, sizeof(BState), cudaMemcpyHostToDevice, s));
}
void download(BState *h, const BState *d, cudaStream_t s)
{
    QB_CUDA(cudaMemcpyAsync(h, d, sizeof(BState), cudaMemcpyDeviceToHost, s));
    sync_check();
}

// device buffers of one batched solve, released on every exit path
struct BatchMem {
    std::vector<void *> ptrs;
    void *get(size_t bytes)
    {
        void *p = dev_alloc(bytes);
        ptrs.push_back(p);
        return p;
    }
    ~BatchMem()
    {
        for (void *p : ptrs) dev_free(p);
    }
};


// One batched solve.  load(f, vtab) fills f.b and f.x (sources and initial
// guesses, vector-table layout); store(f, vtab, h) reads the solutions and
// the per-system results after the run.  m4[s] and resid[s] are per batch
// slot.
template <typename Load, typename Store>
void run_batch(const std::vector<LatRef> &lats, const std::vector<SegPlan> &plan, int nsys, const double *m4,
               const double *resid, int cb, int iter_cap, Load load, Store store)
{
    Context &c = ctx();
    BTable tabs[3] = {make_table(plan, lats, 0), make_table(plan, lats, 1), make_table(plan, lats, 2)};
    long long ncx = 0;
    for (const auto &p : plan) ncx += 3LL * lats[p.lat].g->vh * p.nrhs;

    BatchMem mem;
    BTable *d_tabs = static_cast<BTable *>(mem.get(sizeof(tabs)));
    BState *d_st = static_cast<BState *>(mem.get(sizeof(BState)));
    BFields f{};
    void *mem64 = mem.get((size_t)ncx * 16 * 3);
    void *mem32 = mem.get((size_t)ncx * 8 * 5);
    f.x = static_cast<double2 *>(mem64);
    f.b = f.x + ncx;
    f.t64 = f.b + ncx;
    f.xs = static_cast<float2 *>(mem32);
    f.r = f.xs + ncx;
    f.p = f.r + ncx;
    f.ap = f.p + ncx;
    f.t32 = f.ap + ncx;
    QB_CUDA(cudaMemsetAsync(mem64, 0, (size_t)ncx * 16 * 3, c.stream));
    QB_CUDA(cudaMemsetAsync(mem32, 0, (size_t)ncx * 8 * 5, c.stream));
    QB_CUDA(cudaMemcpyAsync(d_tabs, tabs, sizeof(tabs), cudaMemcpyHostToDevice, c.stream));

    int gmax_s = 1;
    for (int s = 0; s < tabs[0].nseg; ++s) gmax_s = std::max(gmax_s, tabs[0].seg[s].G);
    static int rb_s0 = 0, rb_s1, rb_s0w, rb_s1w, rb_s0n, rb_s1n, rb_d0, rb_d1, rb_v[5];
    if (!rb_s0) {
        rb_s1 = resident_blocks(k_bdslash_s<true, 2>);
        rb_s0w = resident_blocks(k_bdslash_s<false, 4>);
        rb_s1w = resident_blocks(k_bdslash_s<true, 4>);
        rb_s0n = resident_blocks(k_bdslash_s<false, 1>);
        rb_s1n = resident_blocks(k_bdslash_s<true, 1>);
        rb_d0 = resident_blocks(k_bdslash_d<false>);
        rb_d1 = resident_blocks(k_bdslash_d<true>);
        rb_v[0] = resident_blocks(k_bvec<0>);
        rb_v[1] = resident_blocks(k_bvec<1>);
        rb_v[2] = resident_blocks(k_bvec<2>);
        rb_v[3] = resident_blocks(k_bvec<3>);
        rb_v[4] = resident_blocks(k_bvec<4>);
        rb_s0 = resident_blocks(k_bdslash_s<false, 2>);
    }
    auto grid = [](int res_blocks, int ntiles) { return std::max(1, std::min(res_blocks, ntiles)); };
    // resident blocks of the FP32 Dslash kernel for the table's largest G
    auto rb_s = [&](int gm, bool mdagm) {
        return gm > 2 ? (mdagm ? rb_s1w : rb_s0w) : gm == 2 ? (mdagm ? rb_s1 : rb_s0) : (mdagm ? rb_s1n : rb_s0n);
    };
    BatchRun R{};
    R.tab_s = d_tabs;
    R.tab_d = d_tabs + 1;
    R.tab_v = d_tabs + 2;
    R.gmax_s = gmax_s;
    R.grid_s0 = grid(rb_s(gmax_s, false), tabs[0].ntiles);
    R.grid_s1 = grid(rb_s(gmax_s, true), tabs[0].ntiles);
    R.grid_d0 = grid(rb_d0, tabs[1].ntiles);
    R.grid_d1 = grid(rb_d1, tabs[1].ntiles);
    for (int i = 0; i < 5; ++i) R.grid_v[i] = grid(rb_v[i], tabs[2].ntiles);
    const int gmax = std::max({R.grid_s1, R.grid_d1, R.grid_v[0], R.grid_v[1]});
    R.partials = static_cast<double *>(mem.get(sizeof(double) * kBMaxSys * gmax));
    R.st = d_st;
    R.f = f;
    R.cb = cb;
    R.other = 1 - cb;
    R.stream = c.stream;

    load(f, tabs[2], mem);

    BState *h = pinned_state();
    std::memset(h, 0, sizeof(BState));
    h->nsys = nsys;
    // Autotuning of the FP32 batched Dslash: for segments whose size allows
    // it, G = 4, 2 or 1 systems per thread (registers against occupancy).
    // With G = 1 the 16 lanes of a 16-system segment share one site: every
    // colour component is one 128-byte run per site and the kernel fits in
    // 64 registers (4 blocks/SM).
    // Timed once per set of (lattice, segment size) on the solve's own
    // fields, all systems active; the choice is kept for later solves.
    {
        static std::map<std::string, int> chosen;
        std::string key;
        bool choice = false;
        for (const auto &p : plan) {
            key += std::to_string(lats[p.lat].g->vh) + ":" + std::to_string(p.nrhs) + ",";
            choice |= p.nrhs >= 2 && p.nrhs % 3 != 0;
        }
        auto it = chosen.find(key);
        int gpref = 4;
        if (batch_tuning_forced()) {
            gpref = batch_tuning_forced();
        } else if (it != chosen.end()) {
            gpref = it->second;
        } else if (choice) {
            h->active_mask = nsys >= 64 ? ~0ull : ((1ull << nsys) - 1ull);
            upload(d_st, h, c.stream);
            float best = 0;
            for (int g : {4, 2, 1}) {
                const BTable t = make_table(plan, lats, 0, g);
                QB_CUDA(cudaMemcpyAsync(d_tabs, &t, sizeof(BTable), cudaMemcpyHostToDevice, c.stream));
                int gm = 1;
                for (int k = 0; k < t.nseg; ++k) gm = std::max(gm, t.seg[k].G);
                const int gr = grid(rb_s(gm, false), t.ntiles);
                cudaEvent_t e0, e1;
                QB_CUDA(cudaEventCreate(&e0));
                QB_CUDA(cudaEventCreate(&e1));
                for (int r = 0; r < 4; ++r) {
                    if (r == 1) QB_CUDA(cudaEventRecord(e0, c.stream));
                    if (gm > 2) k_bdslash_s<false, 4><<<gr, kBlock, 0, c.stream>>>(d_tabs, d_st, f.t32, f.p, f.p, 1 - cb, R.partials);
                    else if (gm == 2) k_bdslash_s<false, 2><<<gr, kBlock, 0, c.stream>>>(d_tabs, d_st, f.t32, f.p, f.p, 1 - cb, R.partials);
                    else k_bdslash_s<false, 1><<<gr, kBlock, 0, c.stream>>>(d_tabs, d_st, f.t32, f.p, f.p, 1 - cb, R.partials);
                }
                QB_CUDA(cudaEventRecord(e1, c.stream));
                QB_CUDA(cudaEventSynchronize(e1));
                float ms = 0;
                QB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                if (g == 4 || ms < best) {
                    best = ms;
                    gpref = g;
                }
            }
            chosen[key] = gpref;
            h->active_mask = 0;
        }
        last_batch_g = gpref;
        if (gpref != 4) {
            tabs[0] = make_table(plan, lats, 0, gpref);
            gmax_s = 1;
            for (int k = 0; k < tabs[0].nseg; ++k) gmax_s = std::max(gmax_s, tabs[0].seg[k].G);
            R.gmax_s = gmax_s;
            R.grid_s0 = grid(rb_s(gmax_s, false), tabs[0].ntiles);
            R.grid_s1 = grid(rb_s(gmax_s, true), tabs[0].ntiles);
        }
        QB_CUDA(cudaMemcpyAsync(d_tabs, &tabs[0], sizeof(BTable), cudaMemcpyHostToDevice, c.stream));
    }
    h->delta2 = c.reliable_delta * c.reliable_delta;
    h->iter_cap = std::max(1, iter_cap);
    for (int s = 0; s < nsys; ++s) {
        h->sys[s].m4 = m4[s];
        h->sys[s].resid = resid[s];
    }
    upload(d_st, h, c.stream);
    k_bvec<kBNormB><<<R.grid_v[kBNormB], kBlock, 0, c.stream>>>(R.tab_v, d_st, f, R.partials);
    QB_CUDA(cudaGetLastError());
    download(h, d_st, c.stream);

    if (!h->stop) {
        if (batch_graphs_enabled()) {
            BatchGraph G;
            G.build(R);
            h->use_cond = 1;
            h->cond_loop = G.hloop;
            h->cond_ru = G.hru;
            upload(d_st, h, c.stream);
            QB_CUDA(cudaGraphLaunch(G.exec, c.stream));
            download(h, d_st, c.stream);
        } else {
            h->use_cond = 0;
            upload(d_st, h, c.stream);
            int chunk = 16;
            for (;;) {
                for (int i = 0; i < chunk; ++i) {
                    R.reliable_update();
                    R.iteration();
                }
                QB_CUDA(cudaGetLastError());
                download(h, d_st, c.stream);
                if (h->stop && !h->any_flag) break;
                chunk = std::min(chunk * 2, 256);
            }
        }
        // systems stopped by the iteration cap: one last reliable update
        // folds x_s into x and measures their true residual
        if (h->active_mask && !h->nonfinite) {
            h->flag_mask = h->active_mask;
            for (int k = 0; k < h->nsys; ++k) h->sys[k].flag = h->sys[k].active;
            h->any_flag = 1;
            h->use_cond = 0;
            upload(d_st, h, c.stream);
            R.reliable_update();
            download(h, d_st, c.stream);
        }
    }
    if (h->nonfinite == 2) throw Error("batch_invert: CG breakdown (p.Ap <= 0) in a system");
    if (h->nonfinite) throw Error("batch_invert: non-finite source or residual in a system");
    store(f, tabs[2], h, mem);
    sync_check();
    c.stats = Stats{};
    c.stats.iterations = h->iteration;
    c.stats.batch_rhs_per_thread = last_batch_g;
    for (int k = 0; k < h->nsys; ++k) c.stats.reliable_updates += h->sys[k].reliable_updates;
}

void free_batch_links(QPHIX_B200_Batch &B)
{
    for (auto &L : B.lats) {
        free_links(L.l64);
        free_links(L.l32);
    }
}

}  // namespace

// Refinement of several systems (4 m_k^2 - D D) x_k = b on the library's own
// lattice, one batched solve: x_k (FP64 parity blocks) are the initial
// guesses and receive the solutions; each system stops at its own squared
// relative tolerance tol_k on the FP64 true residual.  l32 is the 18-real
// FP32 copy of l64 (the batched kernels' link format).
void batch_refine(const LinkSet &l64, const LinkSet &l32, VecBlock b, const std::vector<VecBlock> &x,
                  const std::vector<double> &mass, const std::vector<double> &tol, int parity, int iter_cap,
                  std::vector<RefineResult> &out)
{
    Context &c = ctx();
    const int nsys = (int)x.size();
    if (nsys < 1 || nsys > kBMaxSys) throw Error("batch_refine: 1.." + std::to_string(kBMaxSys) + " systems");
    std::vector<int> lat(nsys, 0), slot_of;
    const std::vector<SegPlan> plan = plan_segments(1, nsys, lat.data(), slot_of);
    const std::vector<LatRef> lats{LatRef{&c.g, &l64, &l32}};
    std::vector<double> m4(nsys), rs(nsys);
    for (int k = 0; k < nsys; ++k) {
        m4[slot_of[k]] = 4.0 * mass[k] * mass[k];
        rs[slot_of[k]] = tol[k];
    }
    out.assign(nsys, RefineResult{});
    const int n3 = 3 * c.g.vh;
    const Stats keep = c.stats;  // run_batch reports into the context's stats
    run_batch(
        lats, plan, nsys, m4.data(), rs.data(), parity, iter_cap,
        [&](const BFields &f, const BTable &vt, BatchMem &) {
            for (size_t s = 0; s < plan.size(); ++s)
                for (int r = 0; r < plan[s].nrhs; ++r) {
                    const int k = plan[s].user[r];
                    k_b_from_blk<<<grid_for(n3), kBlock, 0, c.stream>>>(f.b, vt.seg[s].voff, n3, plan[s].nrhs, r,
                                                                       static_cast<const double2 *>(b.data));
                    k_b_from_blk<<<grid_for(n3), kBlock, 0, c.stream>>>(f.x, vt.seg[s].voff, n3, plan[s].nrhs, r,
                                                                       static_cast<const double2 *>(x[k].data));
                }
        },
        [&](const BFields &f, const BTable &vt, const BState *h, BatchMem &) {
            for (size_t s = 0; s < plan.size(); ++s)
                for (int r = 0; r < plan[s].nrhs; ++r) {
                    const int k = plan[s].user[r];
                    const BSys &y = h->sys[plan[s].sys0 + r];
                    k_b_to_blk<<<grid_for(n3), kBlock, 0, c.stream>>>(static_cast<double2 *>(x[k].data), f.x,
                                                                     vt.seg[s].voff, n3, plan[s].nrhs, r);
                    out[k].true_rsq_rel = y.bnorm > 0 ? y.true_rsq / y.bnorm : 0.0;
                    out[k].iterations = y.iterations;
                    out[k].reliable_updates = y.reliable_updates;
                }
        });
    c.stats = keep;
}

static QPHIX_B200_Batch *batch_create(int nlat, const int *latsize, double *const *fat, double *const *lng,
                                      double *const *fatback, double *const *lngback)
{
    Context &c = ctx();
    if (!c.initialized) throw Error("batch_create_L: QPhiX library used before QPHIX_init");
    if (nlat < 1 || nlat > kBMaxLat) throw Error("batch_create_L: nlat must be 1.." + std::to_string(kBMaxLat));
    if (!latsize || !fat || !lng || !fatback || !lngback) throw Error("batch_create_L: NULL argument");
    auto *B = new QPHIX_B200_Batch();
    B->lats.reserve(nlat);
    try {
        for (int l = 0; l < nlat; ++l) {
            QPHIX_B200_Batch::Lat L{};
            for (int i = 0; i < 4; ++i) L.dims[i] = latsize[4 * l + i];
            check_lattice(L.dims, "batch_create_L");
            if (!fat[l] || !lng[l] || !fatback[l] || !lngback[l]) throw Error("batch_create_L: NULL link array");
            L.g = make_geom(L.dims[0], L.dims[1], L.dims[2], L.dims[3]);
            B->lats.push_back(L);
            QPHIX_B200_Batch::Lat &H = B->lats.back();
            const Launch ln{c.stream, &H.g, c.d_err};
            H.l64 = alloc_links(Prec::Double, H.g.vh);
            const size_t nraw = (size_t)2 * H.g.vh * 72;
            void *stage = dev_alloc(nraw * sizeof(double));
            const double *raw[4] = {fat[l], fatback[l], lng[l], lngback[l]};  // slots 0..3
            for (int slot = 0; slot < 4; ++slot) {
                h2d_copy(stage, raw[slot], nraw * sizeof(double));
                links_from_raw(Prec::Double, H.l64, stage, true, slot, ln);
            }
            dev_free(stage);
            H.l32 = alloc_links(Prec::Single, H.g.vh);
            links_convert(Prec::Single, H.l32, Prec::Double, H.l64, ln);
            sync_check();
            QB_CUDA(cudaGetLastError());
        }
    } catch (...) {
        free_batch_links(*B);
        delete B;
        throw;
    }
    return B;
}

static void batch_destroy(QPHIX_B200_Batch *B)
{
    if (!B) return;
    free_batch_links(*B);
    sync_check();
    delete B;
}

static int batch_invert(QPHIX_info_t *info, QPHIX_B200_Batch *B, QPHIX_invert_arg_t *inv, QPHIX_resid_arg_t **res,
                        int nsys, const int *lat, const double *mass, double *const *out, double *const *in)
{
    Context &c = ctx();
    if (!c.initialized) throw Error("batch_invert: QPhiX library used before QPHIX_init");
    if (!info || !B || !inv || !res || !lat || !mass || !out || !in) throw Error("batch_invert: NULL argument");
    if (nsys < 1 || nsys > kBMaxSys) throw Error("batch_invert: nsys must be 1.." + std::to_string(kBMaxSys));
    if (inv->parity != QPHIX_EVEN && inv->parity != QPHIX_ODD)
        throw Error("batch_invert: parity must be QPHIX_EVEN or QPHIX_ODD");
    for (int k = 0; k < nsys; ++k) {
        if (lat[k] < 0 || lat[k] >= (int)B->lats.size()) throw Error("batch_invert: lattice index out of range");
        if (!res[k] || !out[k] || !in[k]) throw Error("batch_invert: NULL system argument");
    }
    info->final_sec = wall_seconds();
    const int cb = inv->parity == QPHIX_EVEN ? 0 : 1;
    std::vector<int> slot_of;
    const std::vector<SegPlan> plan = plan_segments((int)B->lats.size(), nsys, lat, slot_of);
    std::vector<LatRef> lats;
    for (const auto &L : B->lats) lats.push_back(LatRef{&L.g, &L.l64, &L.l32});
    std::vector<double> m4(nsys), rs(nsys);
    for (int k = 0; k < nsys; ++k) {
        m4[slot_of[k]] = 4.0 * mass[k] * mass[k];
        rs[slot_of[k]] = res[k]->resid;
    }
    int max_iter = 0;
    double flops = 0;
    run_batch(
        lats, plan, nsys, m4.data(), rs.data(), cb, inv->max * inv->nrestart,
        [&](const BFields &f, const BTable &vt, BatchMem &mem) {
            // sources and initial guesses: parity cb of the callers' raw vectors
            for (size_t s = 0; s < plan.size(); ++s) {
                const SegPlan &p = plan[s];
                const Geom &g = *lats[p.lat].g;
                const size_t n = (size_t)6 * g.vh;
                double *sb = static_cast<double *>(mem.get(sizeof(double) * n * 2 * p.nrhs));
                for (int r = 0; r < p.nrhs; ++r) {
                    const int k = p.user[r];
                    double *bk = sb + 2 * n * r, *xk = bk + n;
                    QB_CUDA(cudaMemcpyAsync(bk, in[k] + cb * n, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream));
                    QB_CUDA(cudaMemcpyAsync(xk, out[k] + cb * n, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream));
                    k_b_from_raw<<<grid_for(g.vh), kBlock, 0, c.stream>>>(f.b, vt.seg[s].voff, g.vh, p.nrhs, r, bk);
                    k_b_from_raw<<<grid_for(g.vh), kBlock, 0, c.stream>>>(f.x, vt.seg[s].voff, g.vh, p.nrhs, r, xk);
                }
            }
        },
        [&](const BFields &f, const BTable &vt, const BState *h, BatchMem &mem) {
            for (size_t s = 0; s < plan.size(); ++s) {
                const SegPlan &p = plan[s];
                const Geom &g = *lats[p.lat].g;
                const size_t n = (size_t)6 * g.vh;
                double *stage = static_cast<double *>(mem.get(sizeof(double) * n));
                for (int r = 0; r < p.nrhs; ++r) {
                    const int k = p.user[r];
                    const BSys &y = h->sys[p.sys0 + r];
                    k_b_to_raw<<<grid_for(g.vh), kBlock, 0, c.stream>>>(stage, f.x, vt.seg[s].voff, g.vh, p.nrhs, r);
                    QB_CUDA(cudaMemcpyAsync(out[k] + cb * n, stage, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                            c.stream));
                    sync_check();
                    res[k]->final_rsq = y.bnorm > 0 ? y.true_rsq / y.bnorm : 0.0;
                    res[k]->size_r = res[k]->final_rsq;
                    res[k]->final_rel = 0;
                    res[k]->size_relr = 0;
                    res[k]->final_iter = y.iterations;
                    res[k]->final_restart = y.reliable_updates;
                    max_iter = std::max(max_iter, y.iterations);
                    flops += 1187.0 * y.iterations * 2.0 * g.vh;
                }
            }
        });
    info->final_sec = wall_seconds() - info->final_sec;
    info->final_flop = flops;
    info->status = QPHIX_SUCCESS;
    return max_iter;
}

// The batched solver's Dslash kernels on caller vectors, one launch each
// (QPHIX_B200_D3_batch_dslash): op 0 out = D in, op 1 out = m4 in - D D in
// (FP32 only); prec 1 FP32 kernels with g systems per thread, 2 the FP64
// kernel of the reliable update.
static void batch_dslash(QPHIX_B200_Batch *B, int nsys, const int *lat, const double *mass, QPHIX_evenodd_t parity,
                         int op, int prec, int g, double *const *out, double *const *in)
{
    Context &c = ctx();
    if (!c.initialized) throw Error("batch_dslash: QPhiX library used before QPHIX_init");
    if (!B || !lat || !out || !in || (op == 1 && !mass)) throw Error("batch_dslash: NULL argument");
    if (nsys < 1 || nsys > kBMaxSys) throw Error("batch_dslash: nsys must be 1.." + std::to_string(kBMaxSys));
    if (parity != QPHIX_EVEN && parity != QPHIX_ODD) throw Error("batch_dslash: parity must be EVEN or ODD");
    if (op != 0 && op != 1) throw Error("batch_dslash: op must be 0 (D) or 1 (4m^2 - D D)");
    if (prec != QPHIX_B200_PREC_SINGLE && prec != QPHIX_B200_PREC_DOUBLE)
        throw Error("batch_dslash: prec must be QPHIX_B200_PREC_SINGLE or _DOUBLE");
    if (prec == QPHIX_B200_PREC_DOUBLE && op != 0) throw Error("batch_dslash: the FP64 batched kernel applies D only");
    if (g == 0) g = 4;
    if (g != 1 && g != 2 && g != 4) throw Error("batch_dslash: rhs_per_thread must be 0, 1, 2 or 4");
    for (int k = 0; k < nsys; ++k) {
        if (lat[k] < 0 || lat[k] >= (int)B->lats.size()) throw Error("batch_dslash: lattice index out of range");
        if (!out[k] || !in[k]) throw Error("batch_dslash: NULL system vector");
    }
    const int cb = parity == QPHIX_EVEN ? 0 : 1;
    const int in_cb = op == 0 ? 1 - cb : cb;
    std::vector<int> slot_of;
    const std::vector<SegPlan> plan = plan_segments((int)B->lats.size(), nsys, lat, slot_of);
    std::vector<LatRef> lats;
    for (const auto &L : B->lats) lats.push_back(LatRef{&L.g, &L.l64, &L.l32});
    const bool dbl = prec == QPHIX_B200_PREC_DOUBLE;
    const BTable tab = make_table(plan, lats, dbl ? 1 : 0, g);
    const BTable vt = make_table(plan, lats, 2);
    long long ncx = 0;
    for (const auto &p : plan) ncx += 3LL * lats[p.lat].g->vh * p.nrhs;

    BatchMem mem;
    BTable *d_tab = static_cast<BTable *>(mem.get(sizeof(BTable)));
    BState *d_st = static_cast<BState *>(mem.get(sizeof(BState)));
    double2 *in64 = static_cast<double2 *>(mem.get((size_t)ncx * 16));
    double2 *out64 = static_cast<double2 *>(mem.get((size_t)ncx * 16));
    QB_CUDA(cudaMemsetAsync(in64, 0, (size_t)ncx * 16, c.stream));
    QB_CUDA(cudaMemsetAsync(out64, 0, (size_t)ncx * 16, c.stream));
    QB_CUDA(cudaMemcpyAsync(d_tab, &tab, sizeof(BTable), cudaMemcpyHostToDevice, c.stream));
    for (size_t s = 0; s < plan.size(); ++s) {
        const SegPlan &p = plan[s];
        const Geom &gm = *lats[p.lat].g;
        const size_t n = (size_t)6 * gm.vh;
        double *stage = static_cast<double *>(mem.get(sizeof(double) * n));
        for (int r = 0; r < p.nrhs; ++r) {
            QB_CUDA(cudaMemcpyAsync(stage, in[p.user[r]] + in_cb * n, sizeof(double) * n, cudaMemcpyHostToDevice,
                                    c.stream));
            k_b_from_raw<<<grid_for(gm.vh), kBlock, 0, c.stream>>>(in64, vt.seg[s].voff, gm.vh, p.nrhs, r, stage);
        }
    }
    BState *h = pinned_state();
    std::memset(h, 0, sizeof(BState));
    h->nsys = nsys;
    h->active_mask = h->flag_mask = nsys >= 64 ? ~0ull : ((1ull << nsys) - 1ull);
    h->any_flag = 1;
    for (int k = 0; k < nsys; ++k) {
        h->sys[slot_of[k]].m4 = op == 1 ? 4.0 * mass[k] * mass[k] : 0.0;
        h->sys[slot_of[k]].active = 1;
        h->sys[slot_of[k]].flag = 1;
    }
    upload(d_st, h, c.stream);
    auto grid = [&](int res_blocks) { return std::max(1, std::min(res_blocks, tab.ntiles)); };
    double *partials = static_cast<double *>(mem.get(sizeof(double) * kBMaxSys * tab.ntiles));
    const unsigned nb = (unsigned)((ncx + kBlock - 1) / kBlock);
    if (dbl) {
        k_bdslash_d<false><<<grid(resident_blocks(k_bdslash_d<false>)), kBlock, 0, c.stream>>>(
            d_tab, d_st, out64, in64, BFields{}, cb, partials);
    } else {
        float2 *in32 = static_cast<float2 *>(mem.get((size_t)ncx * 8));
        float2 *t32 = static_cast<float2 *>(mem.get((size_t)ncx * 8));
        float2 *out32 = static_cast<float2 *>(mem.get((size_t)ncx * 8));
        QB_CUDA(cudaMemsetAsync(t32, 0, (size_t)ncx * 8, c.stream));
        QB_CUDA(cudaMemsetAsync(out32, 0, (size_t)ncx * 8, c.stream));
        k_b_narrow<<<nb, kBlock, 0, c.stream>>>(in32, in64, ncx);
        int gmax = 1;
        for (int k = 0; k < tab.nseg; ++k) gmax = std::max(gmax, tab.seg[k].G);
        auto run = [&](auto k0, auto k1) {
            if (op == 0) {
                k0<<<grid(resident_blocks(k0)), kBlock, 0, c.stream>>>(d_tab, d_st, out32, in32, in32, cb, partials);
            } else {
                k0<<<grid(resident_blocks(k0)), kBlock, 0, c.stream>>>(d_tab, d_st, t32, in32, in32, 1 - cb,
                                                                        partials);
                k1<<<grid(resident_blocks(k1)), kBlock, 0, c.stream>>>(d_tab, d_st, out32, t32, in32, cb, partials);
            }
        };
        if (gmax > 2) run(k_bdslash_s<false, 4>, k_bdslash_s<true, 4>);
        else if (gmax == 2) run(k_bdslash_s<false, 2>, k_bdslash_s<true, 2>);
        else run(k_bdslash_s<false, 1>, k_bdslash_s<true, 1>);
        k_b_widen<<<nb, kBlock, 0, c.stream>>>(out64, out32, ncx);
    }
    QB_CUDA(cudaGetLastError());
    for (size_t s = 0; s < plan.size(); ++s) {
        const SegPlan &p = plan[s];
        const Geom &gm = *lats[p.lat].g;
        const size_t n = (size_t)6 * gm.vh;
        double *stage = static_cast<double *>(mem.get(sizeof(double) * n));
        for (int r = 0; r < p.nrhs; ++r) {
            k_b_to_raw<<<grid_for(gm.vh), kBlock, 0, c.stream>>>(stage, out64, vt.seg[s].voff, gm.vh, p.nrhs, r);
            QB_CUDA(cudaMemcpyAsync(out[p.user[r]] + cb * n, stage, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                    c.stream));
            sync_check();
        }
    }
    sync_check();
}

}  // namespace qb

// ------------------------------------------------------------- C ABI --
namespace {
template <typename F>
QPHIX_status_t batch_guarded(F f)
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

QPHIX_B200_Batch *QPHIX_B200_D3_batch_create_L(int nlat, const int *latsize, double *const *fat, double *const *lng,
                                               double *const *fatback, double *const *lngback)
{
    QPHIX_B200_Batch *B = nullptr;
    batch_guarded([&] { B = qb::batch_create(nlat, latsize, fat, lng, fatback, lngback); });
    return B;
}

void QPHIX_B200_D3_batch_destroy_L(QPHIX_B200_Batch *B)
{
    batch_guarded([&] { qb::batch_destroy(B); });
}

int QPHIX_B200_D3_batch_invert(QPHIX_info_t *info, QPHIX_B200_Batch *B, QPHIX_invert_arg_t *inv_arg,
                               QPHIX_resid_arg_t **res_arg, int nsys, const int *lat, const double *mass,
                               double *const *out, double *const *in)
{
    int it = 0;
    const QPHIX_status_t s =
        batch_guarded([&] { it = qb::batch_invert(info, B, inv_arg, res_arg, nsys, lat, mass, out, in); });
    if (s != QPHIX_SUCCESS && info) info->status = s;
    return it;
}

QPHIX_status_t QPHIX_B200_D3_batch_dslash(QPHIX_B200_Batch *B, int nsys, const int *lat, const double *mass,
                                          QPHIX_evenodd_t parity, int op, QPHIX_B200_precision_t prec,
                                          int rhs_per_thread, double *const *out, double *const *in)
{
    return batch_guarded(
        [&] { qb::batch_dslash(B, nsys, lat, mass, parity, op, (int)prec, rhs_per_thread, out, in); });
}

}  // extern "C"
#pragma GCC visibility pop
