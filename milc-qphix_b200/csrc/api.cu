// The C ABI: QPHIX_* entry points of qphix_int.h / qphix_f3.h / qphix_d3.h
// and the QPHIX_B200_* additions of qphix_b200.h.
//
// Error behaviour: where the reference asserts and exits (MYASSERT,
// ks_boundary.h:35, and assert() in the solvers) this library returns
// QPHIX_FAIL (through the return value or info->status), or NULL from a
// create call, and records a message for QPHIX_B200_last_error().  Nothing
// exits, aborts or traps.
#include <climits>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "context.h"
#include "device_common.cuh"

using namespace qb;

namespace {

template <typename F>
QPHIX_status_t guarded(F f)
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

void require_init()
{
    if (!ctx().initialized) throw Error("QPhiX library used before QPHIX_init");
}

int env_precision(int dflt)
{
    const char *e = std::getenv("QPHIX_GPU_PRECISION");
    if (!e) return dflt;
    if (!strcmp(e, "double") || !strcmp(e, "fp64")) return QPHIX_B200_PREC_DOUBLE;
    if (!strcmp(e, "single") || !strcmp(e, "fp32") || !strcmp(e, "mixed")) return QPHIX_B200_PREC_SINGLE;
    if (!strcmp(e, "half") || !strcmp(e, "fp16")) return QPHIX_B200_PREC_HALF;
    if (!strcmp(e, "half-links")) return QPHIX_B200_PREC_HALF_LINKS;
    return dflt;
}

// Lattice checks of QPHIX_init (qphix_misc.cpp:455-469, 494-497)
void init_context(QPHIX_layout_t *layout)
{
    Context &c = ctx();
    if (!layout || !layout->latsize) throw Error("QPHIX_init: layout or latsize is NULL");
    if (layout->machdim != layout->latdim) throw Error("QPHIX_init: machine dimension must equal lattice dimension");
    if (layout->latdim != 4) throw Error("QPHIX_init: only 4-dimensional lattices are supported");
    // Decomposition: t slabs only, one per process and GPU
    // (QPHIX_B200_comm_init); machsize = {1, 1, 1, P}
    int P = 1;
    if (layout->machsize) {
        for (int i = 0; i < 3; ++i)
            if (layout->machsize[i] != 1)
                throw Error("QPHIX_init: the lattice may be cut along t only (machsize {1,1,1,P})");
        P = layout->machsize[3];
    }
    if (P < 1) throw Error("QPHIX_init: bad machsize");
    if (P != comm_nranks())
        throw Error("QPHIX_init: machsize[3] = " + std::to_string(P) + " but the communicator has " +
                    std::to_string(comm_nranks()) + " ranks (QPHIX_B200_comm_init)");
    if (P > 1 && layout->this_node != comm_rank())
        throw Error("QPHIX_init: this_node differs from the communicator's rank");
    const int *G = layout->latsize;
    if (G[3] % P) throw Error("QPHIX_init: Nt is not a multiple of machsize[3]");
    const int Lloc[4] = {G[0], G[1], G[2], G[3] / P};
    const int *L = Lloc;
    check_lattice(L, "QPHIX_init");
    if (layout->node_number) {
        const int orig[4] = {0, 0, 0, 0};
        (void)layout->node_number(orig);  // the reference calls it (qphix_misc.cpp:489)
    }
    if (c.initialized) {
        if (c.dims[0] == L[0] && c.dims[1] == L[1] && c.dims[2] == L[2] && c.dims[3] == L[3] &&
            c.global_dims[3] == G[3])
            return;
        throw Error("QPHIX_init: already initialised with another lattice; call QPHIX_finalize first");
    }
    const char *dev = std::getenv("QPHIX_GPU_DEVICE");
    c.device = dev ? std::atoi(dev) : 0;
    QB_CUDA(cudaSetDevice(c.device));
    QB_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    cudaMemPool_t pool;
    QB_CUDA(cudaDeviceGetDefaultMemPool(&pool, c.device));
    uint64_t thr = UINT64_MAX;
    QB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    for (int i = 0; i < 4; ++i) c.dims[i] = L[i];
    for (int i = 0; i < 4; ++i) c.global_dims[i] = G[i];
    c.g = make_geom(L[0], L[1], L[2], L[3]);
    halo_setup(c, P, comm_rank(), 2LL * c.g.vh * P);
    QB_CUDA(cudaMalloc(&c.d_state, sizeof(SolverState)));
    QB_CUDA(cudaMemset(c.d_state, 0, sizeof(SolverState)));
    QB_CUDA(cudaMallocHost(&c.h_state, sizeof(SolverState)));
    std::memset(c.h_state, 0, sizeof(SolverState));
    QB_CUDA(cudaMalloc(&c.d_partials, sizeof(double) * 4 * kMaxPartials));
    QB_CUDA(cudaMalloc(&c.d_scalars, sizeof(double) * 64));
    QB_CUDA(cudaMalloc(&c.d_err, sizeof(int)));
    QB_CUDA(cudaMemset(c.d_err, 0, sizeof(int)));
    QB_CUDA(cudaMallocHost(&c.h_scalars, sizeof(double) * 64));
    for (int i = 0; i < 2; ++i) {
        QB_CUDA(cudaEventCreate(&c.ev_solve[i]));
        QB_CUDA(cudaEventCreate(&c.ev_user[i]));
    }
    c.inner_mode = env_precision(QPHIX_B200_PREC_DOUBLE);
    // compressed Naik links for the FP32 inner solves without code changes
    const char *lc = std::getenv("QPHIX_GPU_LINK_COMPRESSION");
    c.link_compression = (lc && lc[0] == '1') ? 1 : 0;
    c.verbose = std::getenv("QPHIX_B200_VERBOSE") ? std::atoi(std::getenv("QPHIX_B200_VERBOSE")) : 0;
    c.initialized = true;
}

void finalize_context()
{
    Context &c = ctx();
    if (!c.initialized) return;
    cudaStreamSynchronize(c.stream);
    cudaFree(c.d_state);
    cudaFreeHost(c.h_state);
    cudaFree(c.d_partials);
    cudaFree(c.d_scalars);
    cudaFree(c.d_err);
    c.d_err = nullptr;
    cudaFreeHost(c.h_scalars);
    for (int i = 0; i < 2; ++i) {
        cudaEventDestroy(c.ev_solve[i]);
        cudaEventDestroy(c.ev_user[i]);
    }
    for (auto e : c.ktimer.ev) cudaEventDestroy(e);
    c.ktimer.ev.clear();
    free_staging();
    halo_free(c);
    cudaStreamDestroy(c.stream);
    c.stream = nullptr;
    c.d_state = nullptr;
    c.h_state = nullptr;
    c.initialized = false;
    for (int i = 0; i < 4; ++i) c.dims[i] = c.global_dims[i] = 0;
}

// ---------------------------------------------------------------------------
// precision-generic API bodies
// ---------------------------------------------------------------------------
template <typename Real> struct Api;
template <> struct Api<float> {
    using CV = QPHIX_F3_ColorVector;
    using FL = QPHIX_F3_FermionLinksAsqtad;
    static constexpr Prec prec = Prec::Single;
};
template <> struct Api<double> {
    using CV = QPHIX_D3_ColorVector;
    using FL = QPHIX_D3_FermionLinksAsqtad;
    static constexpr Prec prec = Prec::Double;
};

template <typename Real>
typename Api<Real>::CV *create_V(Real *src, QPHIX_evenodd_t evenodd)
{
    using CV = typename Api<Real>::CV;
    CV *V = nullptr;
    QPHIX_status_t s = guarded([&] {
        require_init();
        Context &c = ctx();
        if (!src) throw Error("create_V_from_raw: NULL source");
        if ((evenodd & QPHIX_EVENODD) == 0) throw Error("create_V_from_raw: bad evenodd");
        V = new CV();
        V->parity = evenodd;
        const size_t nblk = (size_t)c.g.vh * 6;
        void *stage = dev_alloc(nblk * sizeof(Real));
        for (int cb = 0; cb < 2; ++cb) {
            const int want = cb == 0 ? (evenodd & QPHIX_EVEN) : (evenodd & QPHIX_ODD);
            if (!want) continue;
            V->blk[cb] = alloc_vec(Api<Real>::prec);
            h2d_copy(stage, src + cb * nblk, nblk * sizeof(Real));
            vec_from_raw(Api<Real>::prec, V->blk[cb], stage, sizeof(Real) == 8, c.launch());
        }
        dev_free(stage);
        sync_check();
        QB_CUDA(cudaGetLastError());
        V->even = V->blk[0].data;
        V->odd = V->blk[1].data;
    });
    if (s != QPHIX_SUCCESS && V) {
        for (auto &b : V->blk) free_vec(b);
        delete V;
        V = nullptr;
    }
    return V;
}

template <typename Real>
void extract_V(Real *dest, typename Api<Real>::CV *V)
{
    guarded([&] {
        require_init();
        Context &c = ctx();
        if (!dest || !V) throw Error("extract_V_to_raw: NULL argument");
        const size_t nblk = (size_t)c.g.vh * 6;
        void *stage = dev_alloc(nblk * sizeof(Real));
        for (int cb = 0; cb < 2; ++cb) {
            const int have = cb == 0 ? (V->parity & QPHIX_EVEN) : (V->parity & QPHIX_ODD);
            if (!have) continue;
            vec_to_raw(Api<Real>::prec, stage, sizeof(Real) == 8, V->blk[cb], c.launch());
            d2h_copy(dest + cb * nblk, stage, nblk * sizeof(Real));
        }
        dev_free(stage);
        sync_check();
        QB_CUDA(cudaGetLastError());
    });
}

template <typename Real>
void destroy_V(typename Api<Real>::CV *V)
{
    if (!V) return;
    guarded([&] {
        for (auto &b : V->blk) free_vec(b);
        if (ctx().initialized) sync_check();
    });
    delete V;
}

template <typename FL>
void free_link_handle(FL *L)
{
    free_links(L->links);
    free_links(L->sloppy_half);
    if constexpr (std::is_same<FL, QPHIX_D3_FermionLinksAsqtad>::value) {
        free_links(L->sloppy_single);
        free_links(L->sloppy_recon);
    }
}

template <typename Real>
typename Api<Real>::FL *create_L(Real *fat, Real *lng, Real *fatback, Real *lngback, QPHIX_evenodd_t evenodd)
{
    using FL = typename Api<Real>::FL;
    FL *H = nullptr;
    QPHIX_status_t s = guarded([&] {
        require_init();
        Context &c = ctx();
        if (!fat || !lng || !fatback || !lngback) throw Error("asqtad_create_L_from_raw: NULL link array");
        H = new FL();
        H->links = alloc_links(Api<Real>::prec);
        const size_t nhalf = (size_t)c.g.vh * 72;
        Real *stage = static_cast<Real *>(dev_alloc(2 * nhalf * sizeof(Real)));
        Real *raw[4] = {fat, fatback, lng, lngback};  // slots 0..3
        for (int slot = 0; slot < 4; ++slot) {
            QB_CUDA(cudaMemsetAsync(stage, 0, 2 * nhalf * sizeof(Real), c.stream));
            // only the parities asked for are read, as in qphix_f3.cpp:976-1063
            if ((evenodd & QPHIX_EVENODD) == QPHIX_EVENODD) {
                h2d_copy(stage, raw[slot], 2 * nhalf * sizeof(Real));
            } else {
                if (evenodd & QPHIX_EVEN) h2d_copy(stage, raw[slot], nhalf * sizeof(Real));
                if (evenodd & QPHIX_ODD) h2d_copy(stage + nhalf, raw[slot] + nhalf, nhalf * sizeof(Real));
            }
            links_from_raw(Api<Real>::prec, H->links, stage, sizeof(Real) == 8, slot, c.launch());
        }
        dev_free(stage);
        sync_check();
        QB_CUDA(cudaGetLastError());
        // fat and Naik links of an output parity share one block (grouped by
        // direction), so both pointer pairs name the same blocks
        H->fateven = H->lngeven = H->links.blk[0];
        H->fatodd = H->lngodd = H->links.blk[1];
    });
    if (s != QPHIX_SUCCESS && H) {
        free_link_handle(H);
        delete H;
        H = nullptr;
    }
    return H;
}

template <typename Real>
void extract_L(Real *fat, Real *lng, typename Api<Real>::FL *H, QPHIX_evenodd_t evenodd)
{
    guarded([&] {
        require_init();
        Context &c = ctx();
        if (!fat || !lng || !H) throw Error("asqtad_extract_L_to_raw: NULL argument");
        const size_t nhalf = (size_t)c.g.vh * 72;
        Real *stage = static_cast<Real *>(dev_alloc(2 * nhalf * sizeof(Real)));
        Real *dst[2] = {fat, lng};
        const int slots[2] = {0, 2};  // forward links only (qphix_f3.cpp:1125-1143)
        for (int f = 0; f < 2; ++f) {
            links_to_raw(Api<Real>::prec, stage, sizeof(Real) == 8, H->links, slots[f], c.launch());
            if (evenodd & QPHIX_EVEN) d2h_copy(dst[f], stage, nhalf * sizeof(Real));
            if (evenodd & QPHIX_ODD) d2h_copy(dst[f] + nhalf, stage + nhalf, nhalf * sizeof(Real));
            sync_check();
        }
        dev_free(stage);
        sync_check();
        QB_CUDA(cudaGetLastError());
    });
}

template <typename Real>
void destroy_L(typename Api<Real>::FL *H)
{
    if (!H) return;
    guarded([&] {
        free_link_handle(H);
        if (ctx().initialized) sync_check();
    });
    delete H;
}

// QPHIX_*_asqtad_dslash (qphix_f3.cpp:1233-1245)
template <typename Real>
QPHIX_status_t asqtad_dslash(typename Api<Real>::FL *H, typename Api<Real>::CV *out, typename Api<Real>::CV *in,
                             QPHIX_evenodd_t parity)
{
    return guarded([&] {
        require_init();
        Context &c = ctx();
        if (!H || !out || !in) throw Error("asqtad_dslash: NULL argument");
        if (parity != QPHIX_EVEN && parity != QPHIX_ODD) throw Error("asqtad_dslash: parity must be EVEN or ODD");
        const int cb = parity == QPHIX_EVEN ? 0 : 1;
        const int need_in = cb == 0 ? QPHIX_ODD : QPHIX_EVEN;
        if (!(out->parity & parity) || !(in->parity & need_in))
            throw Error("asqtad_dslash: vectors lack the parities the operator needs");
        dslash(Api<Real>::prec, c.launch(), out->blk[cb], in->blk[1 - cb], H->links, cb);
        sync_check();
        QB_CUDA(cudaGetLastError());
    });
}

// FP32 and 16-bit copies of a D3 link set, made on first use
const LinkSet &single_links(QPHIX_D3_FermionLinksAsqtad *H)
{
    if (!H->sloppy_single.valid) {
        H->sloppy_single = alloc_links(Prec::Single);
        links_convert(Prec::Single, H->sloppy_single, Prec::Double, H->links, ctx().launch());
    }
    return H->sloppy_single;
}

const LinkSet &half_links(QPHIX_D3_FermionLinksAsqtad *H)
{
    if (!H->sloppy_half.valid) {
        H->sloppy_half = alloc_links(Prec::Half);
        links_absmax(Prec::Double, H->links, H->sloppy_half, ctx().launch(), ctx().d_partials);
        links_convert(Prec::Half, H->sloppy_half, Prec::Double, H->links, ctx().launch());
    }
    return H->sloppy_half;
}

// inner solve of a mixed-precision D3 call: vector precision, link set, and
// the FP32 links a stalled 16-bit solve continues with
struct SloppyCfg {
    Prec vec;
    const LinkSet *links;
    const LinkSet *up;
};

// FP32 links with 12-real or 13-real Naik links when compression is on and
// the field has a form they need; otherwise the 18-real FP32 copy
const LinkSet &single_inner_links(QPHIX_D3_FermionLinksAsqtad *H)
{
    Context &c = ctx();
    if (!c.link_compression) return single_links(H);
    if (!H->recon_checked) {
        double dev[5];
        H->recon_checked = 1;
        const int mode = links_compress(H->sloppy_recon, H->links, c.launch(), dev);
        if (c.verbose)
            std::fprintf(stderr,
                         "qphix_b200: Naik links %s (|ratio| %.6e spread %.2e imag %.2e residual %.2e / %.2e)\n",
                         mode == 1 ? "12-real" : mode == 2 ? "13-real" : "keep 18 reals", dev[0], dev[1], dev[2],
                         dev[3], dev[4]);
    }
    return H->sloppy_recon.valid ? H->sloppy_recon : single_links(H);
}

bool refine_batched_env()
{
    const char *e = std::getenv("QPHIX_B200_MS_REFINE");
    return e && std::strcmp(e, "batched") == 0;
}

SloppyCfg sloppy_cfg(QPHIX_D3_FermionLinksAsqtad *H, int mode)
{
    switch (mode) {
    case QPHIX_B200_PREC_SINGLE: return {Prec::Single, &single_inner_links(H), nullptr};
    case QPHIX_B200_PREC_HALF: return {Prec::Half, &half_links(H), &single_inner_links(H)};
    case QPHIX_B200_PREC_HALF_LINKS: return {Prec::Single, &half_links(H), &single_inner_links(H)};
    default: throw Error("unknown inner precision");
    }
}

// ---------------------------------------------------------------------------
// Inner-solve operators on FP64 handles (QPHIX_B200_D3_*_inner)
// ---------------------------------------------------------------------------
// vector precision and link copy of an inner-operator storage; a compressed
// copy of a form the solver has not cached is made for the call only
struct InnerOp {
    Prec vec = Prec::Single;
    const LinkSet *links = nullptr;
    LinkSet temp;
    std::vector<VecBlock> vecs;
    InnerOp() = default;
    InnerOp(const InnerOp &) = delete;
    InnerOp &operator=(const InnerOp &) = delete;
    ~InnerOp()
    {
        for (auto &v : vecs) free_vec(v);
        if (temp.valid) free_links(temp);
    }
    VecBlock vec_tmp()
    {
        vecs.push_back(alloc_vec(vec));
        return vecs.back();
    }
};

void inner_setup(QPHIX_D3_FermionLinksAsqtad *H, int storage, InnerOp &op)
{
    Context &c = ctx();
    switch (storage) {
    case QPHIX_B200_STORE_F32:
        op.vec = Prec::Single;
        op.links = &single_links(H);
        break;
    case QPHIX_B200_STORE_F32_R12:
    case QPHIX_B200_STORE_F32_R13: {
        const int want = storage == QPHIX_B200_STORE_F32_R12 ? 1 : 2;
        op.vec = Prec::Single;
        if (H->recon_checked && H->sloppy_recon.valid && H->sloppy_recon.recon == want) {
            op.links = &H->sloppy_recon;  // the copy the solvers use
        } else {
            double dev[5];
            if (links_compress(op.temp, H->links, c.launch(), dev, want) != want)
                throw Error(std::string("inner operator: the Naik links do not have the ") +
                            (want == 1 ? "12-real" : "13-real") + " form");
            op.links = &op.temp;
        }
        break;
    }
    case QPHIX_B200_STORE_HALF_LINKS:
        op.vec = Prec::Single;
        op.links = &half_links(H);
        break;
    case QPHIX_B200_STORE_HALF:
        op.vec = Prec::Half;
        op.links = &half_links(H);
        break;
    default: throw Error("inner operator: unknown storage");
    }
}

QPHIX_status_t dslash_inner(QPHIX_D3_FermionLinksAsqtad *H, QPHIX_D3_ColorVector *out, QPHIX_D3_ColorVector *in,
                            QPHIX_evenodd_t parity, int storage)
{
    return guarded([&] {
        require_init();
        Context &c = ctx();
        if (!H || !out || !in) throw Error("asqtad_dslash_inner: NULL argument");
        if (parity != QPHIX_EVEN && parity != QPHIX_ODD)
            throw Error("asqtad_dslash_inner: parity must be EVEN or ODD");
        const int cb = parity == QPHIX_EVEN ? 0 : 1;
        if (!out->blk[cb].data || !in->blk[1 - cb].data)
            throw Error("asqtad_dslash_inner: vectors lack the parities the operator needs");
        InnerOp op;
        inner_setup(H, storage, op);
        const Launch L = c.launch();
        VecBlock tin = op.vec_tmp(), tout = op.vec_tmp();
        vec_copy(op.vec, tin, Prec::Double, in->blk[1 - cb], L);
        dslash(op.vec, L, tout, tin, *op.links, cb);
        vec_copy(Prec::Double, out->blk[cb], op.vec, tout, L);
        sync_check();
        QB_CUDA(cudaGetLastError());
    });
}

QPHIX_status_t mdagm_inner(QPHIX_D3_FermionLinksAsqtad *H, QPHIX_D3_ColorVector *out, QPHIX_D3_ColorVector *in,
                           double mass, QPHIX_evenodd_t parity, int storage, double *in_dot_out)
{
    return guarded([&] {
        require_init();
        Context &c = ctx();
        if (!H || !out || !in) throw Error("asqtad_mdagm_inner: NULL argument");
        if (parity != QPHIX_EVEN && parity != QPHIX_ODD)
            throw Error("asqtad_mdagm_inner: parity must be EVEN or ODD");
        const int cb = parity == QPHIX_EVEN ? 0 : 1;
        if (!out->blk[cb].data || !in->blk[cb].data)
            throw Error("asqtad_mdagm_inner: in and out must hold the requested parity");
        InnerOp op;
        inner_setup(H, storage, op);
        const Launch L = c.launch();
        VecBlock p = op.vec_tmp(), tmp = op.vec_tmp(), ttt = op.vec_tmp();
        vec_copy(op.vec, p, Prec::Double, in->blk[cb], L);
        // the inner CG's K1 and K2: tmp = D p; ttt = D tmp - 4 m^2 p, p.ttt
        SolverState &S = *c.h_state;
        S.counter = S.counter2 = 0;
        S.stop_at = INT_MAX;
        S.iteration = 0;
        S.rsq = 1.0;
        S.prec_single = 0;
        upload_state();
        dslash_gated(op.vec, L, tmp, p, *op.links, 1 - cb, c.d_state, -1);
        dslash_mdagm_dot(op.vec, L, ttt, tmp, *op.links, p, -4.0 * mass * mass, cb, c.d_state, c.d_partials, -1, 0);
        vec_copy(Prec::Double, out->blk[cb], op.vec, ttt, L);
        download_state();
        if (in_dot_out) *in_dot_out = S.pkp;
        QB_CUDA(cudaGetLastError());
    });
}

template <typename Real>
int asqtad_invert(QPHIX_info_t *info, typename Api<Real>::FL *H, QPHIX_invert_arg_t *inv, QPHIX_resid_arg_t *res,
                  Real mass, typename Api<Real>::CV *out, typename Api<Real>::CV *in)
{
    int iters = 0;
    QPHIX_status_t s = guarded([&] {
        require_init();
        Context &c = ctx();
        if (!info || !H || !inv || !res || !out || !in) throw Error("asqtad_invert: NULL argument");
        // ks_d_congrad_fn.cpp:233
        if (!(in->parity == out->parity && in->parity == inv->parity))
            throw Error("asqtad_invert: in, out and inv_arg parities differ");
        if (inv->max <= 0 || inv->nrestart < 0) throw Error("asqtad_invert: bad iteration limits");
        c.stats = Stats();
        SolveArgs a{info, inv, res, (double)mass, {out->blk[0], out->blk[1]}, {in->blk[0], in->blk[1]}};
        QB_CUDA(cudaEventRecord(c.ev_solve[0], c.stream));
        if constexpr (std::is_same<Real, double>::value) {
            if (c.inner_mode == QPHIX_B200_PREC_DOUBLE) {
                iters = cg_reference(Prec::Double, H->links, a);
            } else {
                const SloppyCfg s = sloppy_cfg(H, c.inner_mode);
                iters = cg_mixed(s.vec, H->links, *s.links, s.up, a);
                c.stats.links_compressed = s.links->recon;
            }
        } else {
            iters = cg_reference(Prec::Single, H->links, a);
        }
        QB_CUDA(cudaEventRecord(c.ev_solve[1], c.stream));
        QB_CUDA(cudaEventSynchronize(c.ev_solve[1]));
        sync_check();
        float ms = 0;
        QB_CUDA(cudaEventElapsedTime(&ms, c.ev_solve[0], c.ev_solve[1]));
        c.stats.solve_ms = ms;
        QB_CUDA(cudaGetLastError());
    });
    if (s != QPHIX_SUCCESS && info) info->status = s;
    return iters;
}

template <typename Real>
int asqtad_invert_multi(QPHIX_info_t *info, typename Api<Real>::FL *H, QPHIX_invert_arg_t *inv,
                        QPHIX_resid_arg_t *res[], Real *mass, int n, typename Api<Real>::CV *out[],
                        typename Api<Real>::CV *in)
{
    int iters = 0;
    if (n == 0) return 0;  // ks_multicg_offset.cpp:218-225
    QPHIX_status_t s = guarded([&] {
        require_init();
        Context &c = ctx();
        if (!info || !H || !inv || !res || !mass || !out || !in || n < 0) throw Error("asqtad_invert_multi: bad argument");
        if (!(in->parity == out[0]->parity && in->parity == inv->parity))  // :232
            throw Error("asqtad_invert_multi: in, out[0] and inv_arg parities differ");
        if (inv->max <= 0 || inv->nrestart < 0) throw Error("asqtad_invert_multi: bad iteration limits");
        c.stats = Stats();
        MultiArgs a;
        a.info = info;
        a.inv = inv;
        a.res = res;
        std::vector<double> m(mass, mass + n);
        a.mass = m.data();
        a.n = n;
        for (int j = 0; j < n; ++j) {
            if (!out[j] || !res[j]) throw Error("asqtad_invert_multi: NULL out or res entry");
            a.out[0].push_back(out[j]->blk[0]);
            a.out[1].push_back(out[j]->blk[1]);
        }
        a.in[0] = in->blk[0];
        a.in[1] = in->blk[1];
        QB_CUDA(cudaEventRecord(c.ev_solve[0], c.stream));
        if constexpr (std::is_same<Real, double>::value) {
            if (c.inner_mode == QPHIX_B200_PREC_DOUBLE) {
                iters = multishift_reference(Prec::Double, H->links, a);
            } else {
                const SloppyCfg s = sloppy_cfg(H, c.inner_mode);
                // FP32 inner vectors on one GPU: the shifts are refined
                // together by the batched solver, on the 18-real FP32 links
                const LinkSet *l32 =
                    s.vec == Prec::Single && !c.halo.on && refine_batched_env() ? &single_links(H) : nullptr;
                // The per-shift refinements need a few digits per reliable
                // update: with FP32 vectors they run on the 16-bit links,
                // and a refinement that stagnates there continues on the
                // FP32 links (multishift_mixed).  At 32^3x64 the
                // refinements take 247 ms against 295 ms on FP32 links.
                // QPHIX_B200_MS_REFINE_STORAGE=single|half-links|half
                // overrides the choice.
                const char *e = std::getenv("QPHIX_B200_MS_REFINE_STORAGE");
                const std::string rs = e ? e : (s.vec == Prec::Single ? "half-links" : "single");
                RefineOp rop{s.vec, s.links, s.up};
                if (rs == "half-links") rop = {Prec::Single, &half_links(H), &single_inner_links(H)};
                else if (rs == "half") rop = {Prec::Half, &half_links(H), &single_inner_links(H)};
                else if (rs != "single") throw Error("QPHIX_B200_MS_REFINE_STORAGE: single, half-links or half");
                iters = multishift_mixed(s.vec, H->links, *s.links, s.up, a, l32, &rop);
                c.stats.links_compressed = s.links->recon;
            }
        } else {
            iters = multishift_reference(Prec::Single, H->links, a);
        }
        QB_CUDA(cudaEventRecord(c.ev_solve[1], c.stream));
        QB_CUDA(cudaEventSynchronize(c.ev_solve[1]));
        sync_check();
        float ms = 0;
        QB_CUDA(cudaEventElapsedTime(&ms, c.ev_solve[0], c.ev_solve[1]));
        c.stats.solve_ms = ms;
        QB_CUDA(cudaGetLastError());
    });
    if (s != QPHIX_SUCCESS && info) info->status = s;
    return iters;
}

template <typename Real>
QPHIX_status_t dslash_timed(void *links, void *out, void *in, QPHIX_evenodd_t parity, int reps, double *ms)
{
    return guarded([&] {
        require_init();
        Context &c = ctx();
        auto *H = static_cast<typename Api<Real>::FL *>(links);
        auto *O = static_cast<typename Api<Real>::CV *>(out);
        auto *I = static_cast<typename Api<Real>::CV *>(in);
        if (!H || !O || !I || !ms || reps <= 0) throw Error("dslash_timed: bad argument");
        if (parity != QPHIX_EVEN && parity != QPHIX_ODD) throw Error("dslash_timed: parity must be EVEN or ODD");
        const int cb = parity == QPHIX_EVEN ? 0 : 1;
        if (!O->blk[cb].data || !I->blk[1 - cb].data) throw Error("dslash_timed: vectors lack the needed parity");
        // one untimed launch first: module loading and one-time kernel set-up
        dslash(Api<Real>::prec, c.launch(), O->blk[cb], I->blk[1 - cb], H->links, cb);
        QB_CUDA(cudaEventRecord(c.ev_user[0], c.stream));
        for (int r = 0; r < reps; ++r)
            dslash(Api<Real>::prec, c.launch(), O->blk[cb], I->blk[1 - cb], H->links, cb);
        QB_CUDA(cudaEventRecord(c.ev_user[1], c.stream));
        QB_CUDA(cudaEventSynchronize(c.ev_user[1]));
        sync_check();
        float t = 0;
        QB_CUDA(cudaEventElapsedTime(&t, c.ev_user[0], c.ev_user[1]));
        *ms = t / reps;
        QB_CUDA(cudaGetLastError());
    });
}

// autotuner report of kernel 0 (Dslash) / 1 (fused M^dag M) for the
// precision codes of QPHIX_B200_dslash_variant
int variant_report(int kernel, int p, double *us, int n)
{
    Prec pv;
    int slot;
    switch (p) {
    case QPHIX_B200_PREC_HALF: pv = Prec::Half; slot = (int)Prec::Half; break;
    case QPHIX_B200_PREC_SINGLE: pv = Prec::Single; slot = (int)Prec::Single; break;
    case QPHIX_B200_PREC_DOUBLE: pv = Prec::Double; slot = (int)Prec::Double; break;
    case QPHIX_B200_PREC_HALF_LINKS: pv = Prec::Single; slot = (int)Prec::Half; break;
    case QPHIX_B200_TUNE_F32_R12: pv = Prec::Single; slot = 3; break;
    case QPHIX_B200_TUNE_F32_R13: pv = Prec::Single; slot = 4; break;
    default: return -1;
    }
    float t[kDslashVariants] = {0, 0, 0, 0};
    const int v = dslash_variant(kernel, pv, slot, t);
    if (us)
        for (int i = 0; i < n && i < kDslashVariants; ++i) us[i] = t[i];
    return v;
}

}  // namespace

#pragma GCC visibility push(default)
extern "C" {

// ----------------------------------------------------------- init/finalize --
QPHIX_status_t QPHIX_init_F(QPHIX_layout_t *layout) { return guarded([&] { init_context(layout); }); }
QPHIX_status_t QPHIX_init_D(QPHIX_layout_t *layout) { return guarded([&] { init_context(layout); }); }
QPHIX_status_t QPHIX_init(QPHIX_layout_t *layout)
{
    return (QPHIX_status_t)(QPHIX_init_F(layout) | QPHIX_init_D(layout));
}
QPHIX_status_t QPHIX_finalize_F() { return guarded([&] { finalize_context(); }); }
QPHIX_status_t QPHIX_finalize_D() { return guarded([&] { finalize_context(); }); }
QPHIX_status_t QPHIX_finalize() { return (QPHIX_status_t)(QPHIX_finalize_F() | QPHIX_finalize_D()); }

// ------------------------------------------------------------------- F3 --
QPHIX_F3_ColorVector *QPHIX_F3_create_V_from_raw(QPHIX_F_Real *src, QPHIX_evenodd_t evenodd) { return create_V<float>(src, evenodd); }
void QPHIX_F3_extract_V_to_raw(QPHIX_F_Real *dest, QPHIX_F3_ColorVector *src, QPHIX_evenodd_t) { extract_V<float>(dest, src); }
void QPHIX_F3_destroy_V(QPHIX_F3_ColorVector *V) { destroy_V<float>(V); }
QPHIX_F3_FermionLinksAsqtad *QPHIX_F3_asqtad_create_L_from_raw(QPHIX_F_Real *fat, QPHIX_F_Real *lng, QPHIX_F_Real *fatback,
                                                               QPHIX_F_Real *lngback, QPHIX_evenodd_t evenodd)
{
    return create_L<float>(fat, lng, fatback, lngback, evenodd);
}
void QPHIX_F3_asqtad_extract_L_to_raw(QPHIX_F_Real *fat, QPHIX_F_Real *lng, QPHIX_F3_FermionLinksAsqtad *src,
                                      QPHIX_evenodd_t evenodd)
{
    extract_L<float>(fat, lng, src, evenodd);
}
void QPHIX_F3_asqtad_destroy_L(QPHIX_F3_FermionLinksAsqtad *L) { destroy_L<float>(L); }
void QPHIX_F3_asqtad_dslash(QPHIX_F3_FermionLinksAsqtad *L, QPHIX_F3_ColorVector *out, QPHIX_F3_ColorVector *in,
                            QPHIX_evenodd_t parity)
{
    asqtad_dslash<float>(L, out, in, parity);
}
int QPHIX_F3_asqtad_invert(QPHIX_info_t *info, QPHIX_F3_FermionLinksAsqtad *L, QPHIX_invert_arg_t *inv,
                           QPHIX_resid_arg_t *res, QPHIX_F_Real mass, QPHIX_F3_ColorVector *out, QPHIX_F3_ColorVector *in)
{
    return asqtad_invert<float>(info, L, inv, res, mass, out, in);
}
int QPHIX_F3_asqtad_invert_multi(QPHIX_info_t *info, QPHIX_F3_FermionLinksAsqtad *L, QPHIX_invert_arg_t *inv,
                                 QPHIX_resid_arg_t *res[], QPHIX_F_Real *mass, int n, QPHIX_F3_ColorVector *out[],
                                 QPHIX_F3_ColorVector *in)
{
    return asqtad_invert_multi<float>(info, L, inv, res, mass, n, out, in);
}

// ------------------------------------------------------------------- D3 --
QPHIX_D3_ColorVector *QPHIX_D3_create_V_from_raw(QPHIX_D_Real *src, QPHIX_evenodd_t evenodd) { return create_V<double>(src, evenodd); }
void QPHIX_D3_extract_V_to_raw(QPHIX_D_Real *dest, QPHIX_D3_ColorVector *src, QPHIX_evenodd_t) { extract_V<double>(dest, src); }
void QPHIX_D3_destroy_V(QPHIX_D3_ColorVector *V) { destroy_V<double>(V); }
QPHIX_D3_FermionLinksAsqtad *QPHIX_D3_asqtad_create_L_from_raw(QPHIX_D_Real *fat, QPHIX_D_Real *lng, QPHIX_D_Real *fatback,
                                                               QPHIX_D_Real *lngback, QPHIX_evenodd_t evenodd)
{
    return create_L<double>(fat, lng, fatback, lngback, evenodd);
}
void QPHIX_D3_asqtad_extract_L_to_raw(QPHIX_D_Real *fat, QPHIX_D_Real *lng, QPHIX_D3_FermionLinksAsqtad *src,
                                      QPHIX_evenodd_t evenodd)
{
    extract_L<double>(fat, lng, src, evenodd);
}
void QPHIX_D3_asqtad_destroy_L(QPHIX_D3_FermionLinksAsqtad *L) { destroy_L<double>(L); }
void QPHIX_D3_asqtad_dslash(QPHIX_D3_FermionLinksAsqtad *L, QPHIX_D3_ColorVector *out, QPHIX_D3_ColorVector *in,
                            QPHIX_evenodd_t parity)
{
    asqtad_dslash<double>(L, out, in, parity);
}
int QPHIX_D3_asqtad_invert(QPHIX_info_t *info, QPHIX_D3_FermionLinksAsqtad *L, QPHIX_invert_arg_t *inv,
                           QPHIX_resid_arg_t *res, QPHIX_D_Real mass, QPHIX_D3_ColorVector *out, QPHIX_D3_ColorVector *in)
{
    return asqtad_invert<double>(info, L, inv, res, mass, out, in);
}
int QPHIX_D3_asqtad_invert_multi(QPHIX_info_t *info, QPHIX_D3_FermionLinksAsqtad *L, QPHIX_invert_arg_t *inv,
                                 QPHIX_resid_arg_t *res[], QPHIX_D_Real *mass, int n, QPHIX_D3_ColorVector *out[],
                                 QPHIX_D3_ColorVector *in)
{
    return asqtad_invert_multi<double>(info, L, inv, res, mass, n, out, in);
}

// --------------------------------------------------------------- B200 API --
QPHIX_status_t QPHIX_B200_set_inner_precision(QPHIX_B200_precision_t p)
{
    return guarded([&] {
        if (p != QPHIX_B200_PREC_HALF && p != QPHIX_B200_PREC_SINGLE && p != QPHIX_B200_PREC_DOUBLE &&
            p != QPHIX_B200_PREC_HALF_LINKS)
            throw Error("set_inner_precision: unknown precision");
        ctx().inner_mode = p;
    });
}
QPHIX_B200_precision_t QPHIX_B200_get_inner_precision(void) { return static_cast<QPHIX_B200_precision_t>(ctx().inner_mode); }
QPHIX_status_t QPHIX_B200_set_link_compression(int on)
{
    return guarded([&] { ctx().link_compression = on ? 1 : 0; });
}
QPHIX_status_t QPHIX_B200_set_reliable_delta(double delta)
{
    return guarded([&] {
        if (!(delta > 0 && delta < 1)) throw Error("set_reliable_delta: delta must lie in (0, 1)");
        ctx().reliable_delta = delta;
    });
}
QPHIX_status_t QPHIX_B200_get_last_stats(QPHIX_B200_stats_t *s)
{
    return guarded([&] {
        if (!s) throw Error("get_last_stats: NULL");
        const Stats &t = ctx().stats;
        s->solve_ms = t.solve_ms;
        s->iterations = t.iterations;
        s->reliable_updates = t.reliable_updates;
        s->dslash_launches = t.dslash_launches;
        s->dslash_ms = t.dslash_ms;
        s->mdagm_launches = t.mdagm_launches;
        s->mdagm_ms = t.mdagm_ms;
        s->true_rsq = t.true_rsq;
        s->links_compressed = t.links_compressed;
        s->batch_rhs_per_thread = t.batch_rhs_per_thread;
        s->escalated = t.escalated;
    });
}
QPHIX_status_t QPHIX_B200_set_kernel_timing(int on) { return guarded([&] { ctx().kernel_timing = on ? 1 : 0; }); }
QPHIX_status_t QPHIX_B200_timer_start(void)
{
    return guarded([&] {
        require_init();
        QB_CUDA(cudaEventRecord(ctx().ev_user[0], ctx().stream));
    });
}
QPHIX_status_t QPHIX_B200_timer_stop(double *ms)
{
    return guarded([&] {
        require_init();
        if (!ms) throw Error("timer_stop: NULL");
        Context &c = ctx();
        QB_CUDA(cudaEventRecord(c.ev_user[1], c.stream));
        QB_CUDA(cudaEventSynchronize(c.ev_user[1]));
        float t = 0;
        QB_CUDA(cudaEventElapsedTime(&t, c.ev_user[0], c.ev_user[1]));
        *ms = t;
    });
}
QPHIX_status_t QPHIX_B200_F3_dslash_timed(void *links, void *out, void *in, QPHIX_evenodd_t parity, int reps, double *ms)
{
    return dslash_timed<float>(links, out, in, parity, reps, ms);
}
QPHIX_status_t QPHIX_B200_D3_dslash_timed(void *links, void *out, void *in, QPHIX_evenodd_t parity, int reps, double *ms)
{
    return dslash_timed<double>(links, out, in, parity, reps, ms);
}
long QPHIX_B200_neighbor_index(const int L[4], int cb, long site, int k)
{
    if (!L || k < 0 || k > 15 || (cb & ~1)) return -1;
    const Geom g = make_geom(L[0], L[1], L[2], L[3]);
    if (site < 0 || site >= g.vh) return -1;
    const SiteCoords s = decode(g, cb, (int)site);
    return neighbor(g, s, k);
}
QPHIX_status_t QPHIX_B200_D3_asqtad_dslash_inner(QPHIX_D3_FermionLinksAsqtad *L, QPHIX_D3_ColorVector *out,
                                                 QPHIX_D3_ColorVector *in, QPHIX_evenodd_t parity,
                                                 QPHIX_B200_storage_t storage)
{
    return dslash_inner(L, out, in, parity, (int)storage);
}
QPHIX_status_t QPHIX_B200_D3_asqtad_mdagm_inner(QPHIX_D3_FermionLinksAsqtad *L, QPHIX_D3_ColorVector *out,
                                                QPHIX_D3_ColorVector *in, QPHIX_D_Real mass, QPHIX_evenodd_t parity,
                                                QPHIX_B200_storage_t storage, double *in_dot_out)
{
    return mdagm_inner(L, out, in, mass, parity, (int)storage, in_dot_out);
}
QPHIX_status_t QPHIX_B200_comm_unique_id(void *id128)
{
    return guarded([&] {
        if (!id128) throw Error("comm_unique_id: NULL");
        nccl_unique_id(id128);
    });
}
QPHIX_status_t QPHIX_B200_comm_init(const void *id128, int nranks, int rank)
{
    return guarded([&] { comm_init(id128, nranks, rank); });
}
QPHIX_status_t QPHIX_B200_comm_finalize(void) { return guarded([&] { comm_finalize(); }); }
QPHIX_status_t QPHIX_B200_set_loopback_halo(int on)
{
    return guarded([&] {
        Context &c = ctx();
        if (c.initialized && c.halo.nranks > 1) throw Error("set_loopback_halo: several ranks are in use");
        set_loopback(on != 0);
        if (c.initialized) {
            QB_CUDA(cudaStreamSynchronize(c.stream));
            halo_setup(c, 1, 0, 2LL * c.g.vh);
        }
    });
}
int QPHIX_B200_dslash_variant(int p, double us[3]) { return variant_report(0, p, us, 3); }
int QPHIX_B200_mdagm_variant(int p, double us[3]) { return variant_report(1, p, us, 3); }
int QPHIX_B200_tuning(int kernel, int p, double *us, int n)
{
    return (kernel == 0 || kernel == 1) ? variant_report(kernel, p, us, n) : -1;
}
QPHIX_status_t QPHIX_B200_set_dslash_variant(int variant) { return guarded([&] { set_forced_variant(variant); }); }
QPHIX_status_t QPHIX_B200_set_wait_limit(long polls) { return guarded([&] { set_wait_limit(polls); }); }

const char *QPHIX_B200_last_error(void) { return ctx().last_error.c_str(); }
int QPHIX_B200_version(void) { return 100; }

}  // extern "C"
#pragma GCC visibility pop
