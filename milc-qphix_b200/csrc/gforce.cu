// Symanzik one-loop gauge force: QPHIX_{F3,D3}_symanzik_1loop_gauge_force
// and the gauge-field / momentum objects it works on
// (QPHIX_*_create_G_from_raw, _create_F_from_raw, extract, destroy).
//
// Reference: gauge_force_imp.cpp:136-199 passes the gauge field, the
// momenta, coeffs->plaquette / rectangle / parallelogram and eps to per-site
// bodies (gforce_imp_body, update_mg_body) that live in the unvendored
// milc-qphix-codegen; the host layout code (create_G_from_raw,
// create_F_from_raw, qphix_f3.cpp:160-470) fixes the raw formats: 72 reals
// per site, the four forward links (or the four momenta, full 3x3
// anti-Hermitian matrices) of the site, even sites first.  The arithmetic
// is the one-loop Symanzik force as MILC defines it (imp_gauge_force; eps
// carries beta/3):
//
//   A_mu(x) <- A_mu(x) + eps TA( U_mu(x) sum_loops c_loop S_loop(x, mu) ),
//   TA(M) = (M - M^dag)/2 - tr(M - M^dag)/6,
//
// over the 6 plaquettes, 18 1x2 rectangles and 24 six-link parallelograms
// through each link, S_loop the product of the loop's other links from
// x + mu back to x; it is the derivative of S = -1/3 sum c Re tr U_loop
// (restated independently in oracle/gauge_force_oracle.py, which the tests
// also check against finite differences of that action).  As in the
// reference, one call updates the links of one checkerboard: the objects'
// parity, EVENODD meaning EVEN (qphix_f3.cpp:178-179, 347-348).
//
// One thread owns one link (site of the parity, direction mu) and walks the
// 48 staple paths of a constant table; the links it gathers come from
// L1/L2 (every link is read by ~200 threads).  FP64 for D3, FP32 for F3.
#include <cstring>
#include <type_traits>
#include <vector>

#include "context.h"
#include "device_common.cuh"

namespace qb {

namespace {

// staple paths of a forward link mu: steps 2*axis (forward) or 2*axis+1
// (backward) from x + mu back to x; type 0 plaquette, 1 rectangle, 2
// parallelogram
struct GfPath {
    unsigned char n, type, s[5];
};
constexpr int kGfPaths = 48;
__constant__ GfPath c_gf_paths[4][kGfPaths];

std::vector<GfPath> staple_table(int mu)
{
    std::vector<GfPath> out;
    int others[3], k = 0;
    for (int d = 0; d < 4; ++d)
        if (d != mu) others[k++] = d;
    auto st = [](int axis, int sign) { return (unsigned char)(2 * axis + (sign < 0 ? 1 : 0)); };
    for (int i = 0; i < 3; ++i)
        for (int s : {1, -1}) {
            const int nu = others[i];
            out.push_back(GfPath{3, 0, {st(nu, s), st(mu, -1), st(nu, -s), 0, 0}});
        }
    for (int i = 0; i < 3; ++i)
        for (int s : {1, -1}) {
            const int nu = others[i];
            out.push_back(GfPath{5, 1, {st(mu, 1), st(nu, s), st(mu, -1), st(mu, -1), st(nu, -s)}});
            out.push_back(GfPath{5, 1, {st(nu, s), st(mu, -1), st(mu, -1), st(nu, -s), st(mu, 1)}});
            out.push_back(GfPath{5, 1, {st(nu, s), st(nu, s), st(mu, -1), st(nu, -s), st(nu, -s)}});
        }
    for (int i = 0; i < 3; ++i)
        for (int i2 = 0; i2 < 3; ++i2) {
            if (i2 == i) continue;
            for (int s : {1, -1})
                for (int r : {1, -1}) {
                    const int nu = others[i], rho = others[i2];
                    out.push_back(GfPath{5, 2, {st(nu, s), st(rho, r), st(mu, -1), st(nu, -s), st(rho, -r)}});
                }
        }
    return out;
}

// 3x3 complex products on row-major reals (u[6 r + 2 c] + i u[6 r + 2 c + 1])
template <typename R>
__device__ __forceinline__ void mm(const R a[18], const R b[18], R c[18], bool adj_b)
{
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            R re = 0, im = 0;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const R ar = a[6 * r + 2 * j], ai = a[6 * r + 2 * j + 1];
                // b_jk, or conj(b_kj) for b^dag
                const R br = adj_b ? b[6 * k + 2 * j] : b[6 * j + 2 * k];
                const R bi = adj_b ? -b[6 * k + 2 * j + 1] : b[6 * j + 2 * k + 1];
                re += ar * br - ai * bi;
                im += ar * bi + ai * br;
            }
            c[6 * r + 2 * k] = re;
            c[6 * r + 2 * k + 1] = im;
        }
}

template <typename R>
struct GaugeView {
    const cx_t<R> *b[2];
    Geom g;
    // link of direction d at full coordinates y (already wrapped)
    __device__ __forceinline__ void load(const int y[4], int d, R u[18]) const
    {
        const int cb = (y[0] + y[1] + y[2] + y[3]) & 1;
        const int j = ((y[3] * g.nz + y[2]) * g.ny + y[1]) * g.nxh + (y[0] >> 1);
        const cx_t<R> *p = b[cb] + (size_t)d * 9 * g.vh + j;
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            const cx_t<R> z = __ldg(p + (size_t)e * g.vh);
            u[2 * e] = z.x;
            u[2 * e + 1] = z.y;
        }
    }
};

// M <- M U or M U^dag, one row at a time (row r of the product needs only
// row r of M), with mm's arithmetic order
template <typename R>
__device__ __forceinline__ void mm_inplace(R a[18], const R b[18], bool adj_b)
{
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        R t[6];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            R re = 0, im = 0;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const R ar = a[6 * r + 2 * j], ai = a[6 * r + 2 * j + 1];
                const R br = adj_b ? b[6 * k + 2 * j] : b[6 * j + 2 * k];
                const R bi = adj_b ? -b[6 * k + 2 * j + 1] : b[6 * j + 2 * k + 1];
                re += ar * br - ai * bi;
                im += ar * bi + ai * br;
            }
            t[2 * k] = re;
            t[2 * k + 1] = im;
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) a[6 * r + i] = t[i];
    }
}

// One thread per link (direction-major: a warp's threads share the path
// table entry and gather consecutive sites).  In FP64 the path product is
// formed in place, one row at a time, under a register cap of four blocks per
// SM: 15.6 ms against 16.2 ms per 32^3x64 checkerboard.  In FP32 both were
// slower (9.7 ms with the cap, 10.6 ms in place without it, against 9.3 ms),
// so FP32 keeps the product in a third matrix.  Moving the staple sum to
// shared memory and interleaving the four directions of a site over adjacent
// threads was slower in both (17.4 / 11.8 ms).
constexpr int kGfThreads = 128;
template <typename R> struct GfMinBlocks { static constexpr int value = 1; };
template <> struct GfMinBlocks<double> { static constexpr int value = 4; };

template <typename R>
__global__ void __launch_bounds__(kGfThreads, GfMinBlocks<R>::value)
k_gauge_force(GaugeView<R> U, cx_t<R> *mom, int cb, R eps, R c0, R c1, R c2)
{
    const Geom &g = U.g;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 4 * g.vh) return;
    const int mu = idx / g.vh, j = idx - mu * g.vh;
    const SiteCoords s = decode(g, cb, j);
    const int x0[4] = {2 * s.xh + s.xodd, s.y, s.z, s.t};
    const int L[4] = {g.nx, g.ny, g.nz, g.nt};
    const R coef[3] = {c0, c1, c2};
    R acc[18];
#pragma unroll
    for (int i = 0; i < 18; ++i) acc[i] = R(0);
#pragma unroll 1
    for (int p = 0; p < kGfPaths; ++p) {
        const GfPath P = c_gf_paths[mu][p];
        const R c = coef[P.type];
        if (c == R(0)) continue;
        int y[4] = {x0[0], x0[1], x0[2], x0[3]};
        y[mu] = y[mu] + 1 == L[mu] ? 0 : y[mu] + 1;
        R M[18], Lk[18];
#pragma unroll 1
        for (int k = 0; k < P.n; ++k) {
            const int a = P.s[k] >> 1;
            const bool back = P.s[k] & 1;
            if (back) y[a] = y[a] == 0 ? L[a] - 1 : y[a] - 1;
            U.load(y, a, Lk);
            if (!back) y[a] = y[a] + 1 == L[a] ? 0 : y[a] + 1;
            if (k == 0) {
                if (back) {
#pragma unroll
                    for (int r = 0; r < 3; ++r)
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            M[6 * r + 2 * q] = Lk[6 * q + 2 * r];
                            M[6 * r + 2 * q + 1] = -Lk[6 * q + 2 * r + 1];
                        }
                } else {
#pragma unroll
                    for (int i = 0; i < 18; ++i) M[i] = Lk[i];
                }
            } else if constexpr (std::is_same<R, double>::value) {
                mm_inplace(M, Lk, back);
            } else {
                R T[18];
                mm(M, Lk, T, back);
#pragma unroll
                for (int i = 0; i < 18; ++i) M[i] = T[i];
            }
        }
#pragma unroll
        for (int i = 0; i < 18; ++i) acc[i] += c * M[i];
    }
    R Um[18], W[18];
    U.load(x0, mu, Um);
    mm(Um, acc, W, false);
    // TA(W) = (W - W^dag)/2 - tr(W - W^dag)/6
    const R tr = (W[1] + W[9] + W[17]) * (R(1) / R(3));  // imaginary part of tr(W - W^dag)/2 / 3
    cx_t<R> *m = mom + (size_t)mu * 9 * g.vh + j;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            R fr = R(0.5) * (W[6 * r + 2 * q] - W[6 * q + 2 * r]);
            R fi = R(0.5) * (W[6 * r + 2 * q + 1] + W[6 * q + 2 * r + 1]);
            if (r == q) fi -= tr;
            cx_t<R> z = m[(size_t)(3 * r + q) * g.vh];
            z.x += eps * fr;
            z.y += eps * fi;
            m[(size_t)(3 * r + q) * g.vh] = z;
        }
}

// raw (72 reals per site, site cb*vh + j) <-> blocks [dir][9][vh] of the
// parities in mask (bit cb)
template <typename D, typename RAW>
__global__ void k_gf_from_raw(D *b0, D *b1, const RAW *raw, int vh, int mask)
{
    const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (idx >= (size_t)2 * vh * 36) return;
    const int e = idx % 9, d = (idx / 9) % 4;
    const size_t s = idx / 36;
    const int cb = s >= (size_t)vh;
    if (!((mask >> cb) & 1)) return;
    const int j = (int)(s - (size_t)cb * vh);
    D z;
    z.x = raw[2 * idx];
    z.y = raw[2 * idx + 1];
    (cb ? b1 : b0)[((size_t)d * 9 + e) * vh + j] = z;
}

template <typename S, typename RAW>
__global__ void k_gf_to_raw(RAW *raw, const S *b0, const S *b1, int vh, int mask)
{
    const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (idx >= (size_t)2 * vh * 36) return;
    const int e = idx % 9, d = (idx / 9) % 4;
    const size_t s = idx / 36;
    const int cb = s >= (size_t)vh;
    if (!((mask >> cb) & 1)) return;
    const int j = (int)(s - (size_t)cb * vh);
    const S z = (cb ? b1 : b0)[((size_t)d * 9 + e) * vh + j];
    raw[2 * idx] = (RAW)z.x;
    raw[2 * idx + 1] = (RAW)z.y;
}

template <typename R> struct GfApi;
template <> struct GfApi<float> {
    using G = QPHIX_F3_GaugeField;
    using F = QPHIX_F3_Force;
};
template <> struct GfApi<double> {
    using G = QPHIX_D3_GaugeField;
    using F = QPHIX_D3_Force;
};

int parity_mask(QPHIX_evenodd_t eo) { return ((eo & QPHIX_EVEN) ? 1 : 0) | ((eo & QPHIX_ODD) ? 2 : 0); }

template <typename F>
QPHIX_status_t gf_guarded(F f)
{
    try {
        f();
        ctx().last_error.clear();
        return QPHIX_SUCCESS;
    } catch (const Error &e) {
        ctx().last_error = e.what();
        return e.status;
    } catch (const std::exception &e) {
        ctx().last_error = e.what();
        return QPHIX_FAIL;
    }
}

void require(bool ok, const char *msg)
{
    if (!ok) throw Error(msg);
}

// both parity blocks of a field, raw -> device, parities of `mask`
template <typename R>
void upload_blocks(void *blk[2], const R *raw, int mask)
{
    Context &c = ctx();
    const int vh = c.g.vh;
    const size_t bytes = (size_t)36 * vh * sizeof(cx_t<R>);
    for (int cb = 0; cb < 2; ++cb) {
        blk[cb] = dev_alloc(bytes);
        QB_CUDA(cudaMemsetAsync(blk[cb], 0, bytes, c.stream));
    }
    const size_t nraw = (size_t)2 * vh * 72;
    R *stage = static_cast<R *>(dev_alloc(nraw * sizeof(R)));
    QB_CUDA(cudaMemsetAsync(stage, 0, nraw * sizeof(R), c.stream));
    if (mask & 1) h2d_copy(stage, raw, nraw / 2 * sizeof(R));
    if (mask & 2) h2d_copy(stage + nraw / 2, raw + nraw / 2, nraw / 2 * sizeof(R));
    const int grid = (int)(((size_t)2 * vh * 36 + kBlock - 1) / kBlock);
    k_gf_from_raw<cx_t<R>, R><<<grid, kBlock, 0, c.stream>>>(static_cast<cx_t<R> *>(blk[0]),
                                                             static_cast<cx_t<R> *>(blk[1]), stage, vh, mask);
    dev_free(stage);
    sync_check();
    QB_CUDA(cudaGetLastError());
}

template <typename R>
void download_blocks(R *raw, void *const blk[2], int mask)
{
    Context &c = ctx();
    const int vh = c.g.vh;
    const size_t nraw = (size_t)2 * vh * 72;
    R *stage = static_cast<R *>(dev_alloc(nraw * sizeof(R)));
    const int grid = (int)(((size_t)2 * vh * 36 + kBlock - 1) / kBlock);
    k_gf_to_raw<cx_t<R>, R><<<grid, kBlock, 0, c.stream>>>(stage, static_cast<const cx_t<R> *>(blk[0]),
                                                           static_cast<const cx_t<R> *>(blk[1]), vh, mask);
    if (mask & 1) d2h_copy(raw, stage, nraw / 2 * sizeof(R));
    if (mask & 2) d2h_copy(raw + nraw / 2, stage + nraw / 2, nraw / 2 * sizeof(R));
    dev_free(stage);
    sync_check();
    QB_CUDA(cudaGetLastError());
}

template <typename H>
void free_blocks(H *h)
{
    for (auto &b : h->blk) {
        dev_free(b);
        b = nullptr;
    }
}

void check_evenodd(QPHIX_evenodd_t eo, const char *who)
{
    if (eo != QPHIX_EVEN && eo != QPHIX_ODD && eo != QPHIX_EVENODD) throw Error(std::string(who) + ": bad evenodd");
}

void check_single_rank(const char *who)
{
    const Context &c = ctx();
    if (c.halo.on && c.halo.nranks > 1) throw Error(std::string(who) + ": not available with several ranks");
}

template <typename R>
typename GfApi<R>::G *create_G(R *raw, QPHIX_evenodd_t evenodd)
{
    using G = typename GfApi<R>::G;
    G *h = nullptr;
    const QPHIX_status_t st = gf_guarded([&] {
        require(ctx().initialized, "create_G_from_raw: QPhiX library used before QPHIX_init");
        require(raw != nullptr, "create_G_from_raw: NULL source");
        check_evenodd(evenodd, "create_G_from_raw");
        check_single_rank("create_G_from_raw");
        h = new G();
        h->parity = evenodd == QPHIX_EVENODD ? QPHIX_EVEN : evenodd;
        h->compress12 = 0;
        // the staples reach links of both parities: the reference reads the
        // whole raw field whatever evenodd says (qphix_f3.cpp:184)
        upload_blocks<R>(h->blk, raw, 3);
        h->geo = h->blk[0];
    });
    if (st != QPHIX_SUCCESS && h) {
        free_blocks(h);
        delete h;
        h = nullptr;
    }
    return h;
}

template <typename R>
void extract_G(R *dest, typename GfApi<R>::G *h, QPHIX_evenodd_t evenodd)
{
    gf_guarded([&] {
        require(ctx().initialized, "extract_G_to_raw: QPhiX library used before QPHIX_init");
        require(dest && h, "extract_G_to_raw: NULL argument");
        check_evenodd(evenodd, "extract_G_to_raw");
        download_blocks<R>(dest, h->blk, parity_mask(evenodd));
    });
}

template <typename R>
typename GfApi<R>::F *create_F(R *raw, QPHIX_evenodd_t evenodd)
{
    using F = typename GfApi<R>::F;
    F *h = nullptr;
    const QPHIX_status_t st = gf_guarded([&] {
        require(ctx().initialized, "create_F_from_raw: QPhiX library used before QPHIX_init");
        require(raw != nullptr, "create_F_from_raw: NULL source");
        check_evenodd(evenodd, "create_F_from_raw");
        check_single_rank("create_F_from_raw");
        h = new F();
        h->parity = evenodd == QPHIX_EVENODD ? QPHIX_EVEN : evenodd;
        upload_blocks<R>(h->blk, raw, parity_mask(evenodd));
        h->heo = h->blk[0];
        h->htmp = h->blk[1];
    });
    if (st != QPHIX_SUCCESS && h) {
        free_blocks(h);
        delete h;
        h = nullptr;
    }
    return h;
}

template <typename R>
void extract_F(R *dest, typename GfApi<R>::F *h, QPHIX_evenodd_t evenodd)
{
    gf_guarded([&] {
        require(ctx().initialized, "extract_F_to_raw: QPhiX library used before QPHIX_init");
        require(dest && h, "extract_F_to_raw: NULL argument");
        check_evenodd(evenodd, "extract_F_to_raw");
        download_blocks<R>(dest, h->blk, parity_mask(evenodd));
    });
}

template <typename H>
void destroy(H *h)
{
    if (!h) return;
    gf_guarded([&] {
        free_blocks(h);
        if (ctx().initialized) sync_check();
    });
    delete h;
}

bool g_table_ready[64] = {false};

void upload_table()
{
    int dev = 0;
    QB_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && g_table_ready[dev]) return;
    GfPath t[4][kGfPaths];
    for (int mu = 0; mu < 4; ++mu) {
        const std::vector<GfPath> p = staple_table(mu);
        if ((int)p.size() != kGfPaths) throw Error("gauge force: staple table has the wrong size");
        for (int i = 0; i < kGfPaths; ++i) t[mu][i] = p[i];
    }
    QB_CUDA(cudaMemcpyToSymbol(c_gf_paths, t, sizeof(t)));
    if (dev >= 0 && dev < 64) g_table_ready[dev] = true;
}

// flops of one link's force: (steps - 1) 3x3 complex products per path
// (198 flops each), its weighted sum (36), U times the sum (198), TA and the
// update (54)
double flops_per_link(const QPHIX_gauge_coeffs_t &co)
{
    const double c[3] = {co.plaquette, co.rectangle, co.parallelogram};
    const std::vector<GfPath> p = staple_table(0);
    double f = 198 + 54;
    for (const auto &q : p)
        if (c[q.type] != 0.0) f += 198.0 * (q.n - 1) + 36;
    return f;
}

template <typename R>
void gauge_force(QPHIX_info_t *info, typename GfApi<R>::G *G, typename GfApi<R>::F *F,
                 QPHIX_gauge_coeffs_t *coeffs, R eps)
{
    Context &c = ctx();
    QPHIX_status_t s = gf_guarded([&] {
        require(c.initialized, "symanzik_1loop_gauge_force: QPhiX library used before QPHIX_init");
        require(info && G && F && coeffs, "symanzik_1loop_gauge_force: NULL argument");
        // gauge_force_imp.cpp:142
        require(F->parity == G->parity, "symanzik_1loop_gauge_force: force and gauge field parities differ");
        check_single_rank("symanzik_1loop_gauge_force");
        info->final_sec = wall_seconds();
        upload_table();
        const int cb = G->parity == QPHIX_EVEN ? 0 : 1;
        GaugeView<R> U;
        U.b[0] = static_cast<const cx_t<R> *>(G->blk[0]);
        U.b[1] = static_cast<const cx_t<R> *>(G->blk[1]);
        U.g = c.g;
        QB_CUDA(cudaEventRecord(c.ev_solve[0], c.stream));
        const int grid = (4 * c.g.vh + kGfThreads - 1) / kGfThreads;
        k_gauge_force<R><<<grid, kGfThreads, 0, c.stream>>>(U, static_cast<cx_t<R> *>(F->blk[cb]), cb, eps,
                                                     (R)coeffs->plaquette, (R)coeffs->rectangle,
                                                     (R)coeffs->parallelogram);
        QB_CUDA(cudaGetLastError());
        QB_CUDA(cudaEventRecord(c.ev_solve[1], c.stream));
        sync_check();
        float ms = 0.f;
        QB_CUDA(cudaEventElapsedTime(&ms, c.ev_solve[0], c.ev_solve[1]));
        c.stats = Stats{};
        c.stats.solve_ms = ms;
        info->final_sec = wall_seconds() - info->final_sec;
        info->final_flop = flops_per_link(*coeffs) * 4.0 * c.g.vh;
        info->status = QPHIX_SUCCESS;
    });
    if (s != QPHIX_SUCCESS && info) info->status = s;
}

}  // namespace
}  // namespace qb

using namespace qb;

#pragma GCC visibility push(default)
extern "C" {

QPHIX_F3_GaugeField *QPHIX_F3_create_G_from_raw(QPHIX_F_Real *raw, QPHIX_evenodd_t eo) { return create_G<float>(raw, eo); }
void QPHIX_F3_extract_G_to_raw(QPHIX_F_Real *dest, QPHIX_F3_GaugeField *G, QPHIX_evenodd_t eo) { extract_G<float>(dest, G, eo); }
void QPHIX_F3_destroy_G(QPHIX_F3_GaugeField *G) { destroy(G); }
QPHIX_F3_Force *QPHIX_F3_create_F_from_raw(QPHIX_F_Real *raw, QPHIX_evenodd_t eo) { return create_F<float>(raw, eo); }
void QPHIX_F3_extract_F_to_raw(QPHIX_F_Real *dest, QPHIX_F3_Force *F, QPHIX_evenodd_t eo) { extract_F<float>(dest, F, eo); }
void QPHIX_F3_destroy_F(QPHIX_F3_Force *F) { destroy(F); }
void QPHIX_F3_symanzik_1loop_gauge_force(QPHIX_info_t *info, QPHIX_F3_GaugeField *G, QPHIX_F3_Force *F,
                                         QPHIX_gauge_coeffs_t *coeffs, QPHIX_F_Real eps)
{
    gauge_force<float>(info, G, F, coeffs, eps);
}

QPHIX_D3_GaugeField *QPHIX_D3_create_G_from_raw(QPHIX_D_Real *raw, QPHIX_evenodd_t eo) { return create_G<double>(raw, eo); }
void QPHIX_D3_extract_G_to_raw(QPHIX_D_Real *dest, QPHIX_D3_GaugeField *G, QPHIX_evenodd_t eo) { extract_G<double>(dest, G, eo); }
void QPHIX_D3_destroy_G(QPHIX_D3_GaugeField *G) { destroy(G); }
QPHIX_D3_Force *QPHIX_D3_create_F_from_raw(QPHIX_D_Real *raw, QPHIX_evenodd_t eo) { return create_F<double>(raw, eo); }
void QPHIX_D3_extract_F_to_raw(QPHIX_D_Real *dest, QPHIX_D3_Force *F, QPHIX_evenodd_t eo) { extract_F<double>(dest, F, eo); }
void QPHIX_D3_destroy_F(QPHIX_D3_Force *F) { destroy(F); }
void QPHIX_D3_symanzik_1loop_gauge_force(QPHIX_info_t *info, QPHIX_D3_GaugeField *G, QPHIX_D3_Force *F,
                                         QPHIX_gauge_coeffs_t *coeffs, QPHIX_D_Real eps)
{
    gauge_force<double>(info, G, F, coeffs, eps);
}

}  // extern "C"
#pragma GCC visibility pop
