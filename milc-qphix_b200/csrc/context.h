// Process-wide state of libqphix_b200 and the handle structures behind the
// QPhiX opaque types.
//
// The reference keeps its lattice geometry, neighbour tables and thread
// scheduler in process globals per precision (ks_globals.h:14-43), set by
// QPHIX_init (qphix_misc.cpp:427-547) and cleared by QPHIX_finalize
// (:549-578).  Here the process globals are one Context: geometry, the CUDA
// stream every call runs on, the device-resident solver scalars, reduction
// scratch and the solver settings.  Like the reference, the library serves
// one caller thread; every entry point is synchronous on return.
#pragma once

#include <chrono>
#include <climits>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "halo.h"
#include "internal.h"
#include "qphix.h"
#include "qphix_b200.h"

namespace qb {

struct Error : std::runtime_error {
    QPHIX_status_t status;
    Error(const std::string &m, QPHIX_status_t s = QPHIX_FAIL) : std::runtime_error(m), status(s) {}
};

#define QB_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            throw ::qb::Error(std::string(#call) + ": " + cudaGetErrorString(e_),              \
                              e_ == cudaErrorMemoryAllocation ? QPHIX_MEM_ERROR : QPHIX_FAIL); \
    } while (0)

struct Stats {
    double solve_ms = 0;
    int iterations = 0;
    int reliable_updates = 0;
    int dslash_launches = 0;
    double dslash_ms = 0;
    int mdagm_launches = 0;
    double mdagm_ms = 0;
    double true_rsq = 0;
    int escalated = 0;
    int links_compressed = 0;
    int batch_rhs_per_thread = 0;
};

// CUDA-event timing of individual kernel launches inside a solve
struct KernelTimer {
    std::vector<cudaEvent_t> ev;
    size_t used = 0;
    std::vector<std::pair<int, size_t>> marks;  // (kind, first event index); kind 0 = K1, 1 = K2
    void reset() { used = 0; marks.clear(); }
    cudaEvent_t next()
    {
        if (used == ev.size()) {
            cudaEvent_t e;
            QB_CUDA(cudaEventCreate(&e));
            ev.push_back(e);
        }
        return ev[used++];
    }
};

// Pinned staging for host -> device copies from pageable memory (h2d_copy):
// one CUDA stream and two pinned slots per host worker thread.
struct HostStaging {
    int workers = 0;
    std::vector<cudaStream_t> streams;
    std::vector<char *> slots;
    std::vector<cudaEvent_t> done;
};

struct Context {
    bool initialized = false;
    int dims[4] = {0, 0, 0, 0};
    Geom g{};
    int device = 0;
    cudaStream_t stream = nullptr;
    SolverState *d_state = nullptr;
    SolverState *h_state = nullptr;  // pinned mirror
    double *d_partials = nullptr;    // reduction partials
    double *d_scalars = nullptr;     // device scalar outputs
    double *h_scalars = nullptr;     // pinned mirror of d_scalars
    cudaEvent_t ev_solve[2] = {nullptr, nullptr};
    cudaEvent_t ev_user[2] = {nullptr, nullptr};
    // settings (qphix_b200.h)
    int inner_mode = QPHIX_B200_PREC_DOUBLE;  // QPHIX_B200_precision_t of D3 solves
    int link_compression = 0;                 // FP32 inner solves with 12-/13-real Naik links
    double reliable_delta = 0.2;
    int kernel_timing = 0;
    int max_chunk = 64;
    int verbose = 0;
    Stats stats;
    KernelTimer ktimer;
    std::string last_error;

    int *d_err = nullptr;            // kernel failure word (bounded waits)
    HostStaging staging;             // made on the first large pageable upload
    Halo halo;                       // domain decomposition along t (halo.h)
    int global_dims[4] = {0, 0, 0, 0};  // the whole lattice (dims: this GPU's slab)

    Launch launch() const { return Launch{stream, &g, d_err, halo.on ? &halo : nullptr}; }
};

Context &ctx();

// domain decomposition (halo.cu)
void comm_init(const void *id128, int nranks, int rank);
void comm_finalize();
int comm_nranks();
int comm_rank();
void set_loopback(bool on);
bool loopback();
void halo_setup(Context &c, int nranks, int rank, long long global_sites);
void halo_free(Context &c);

// device memory from the stream-ordered pool (cached, no device-wide sync)
void *dev_alloc(size_t bytes);
void dev_free(void *p);

// Host -> device copy that has completed on return.  Pinned or small
// sources go by one cudaMemcpyAsync on the library stream; large pageable
// ones are split across host threads, each copying its part through two
// pinned slots while the copy engine moves the previous slot.
void h2d_copy(void *dst, const void *src, size_t bytes);
// the same for device -> host (completed on return)
void d2h_copy(void *dst, const void *src, size_t bytes);
void free_staging();

VecBlock alloc_vec(Prec p);
void free_vec(VecBlock &b);
LinkSet alloc_links(Prec p);          // for the QPHIX_init lattice
LinkSet alloc_links(Prec p, int vh);  // for a lattice of vh sites per parity
void free_links(LinkSet &ls);

void upload_state();    // h_state -> d_state (async)
void download_state();  // d_state -> h_state, waits
void sync_check();      // waits for the stream; throws if a kernel reported a failed wait

double wall_seconds();

// lattice extents the library accepts (the reference's asserts,
// qphix_misc.cpp:455-469,494-497); throws Error("<who>: ...") otherwise
void check_lattice(const int L[4], const char *who);

}  // namespace qb

// ---- handle structures behind the opaque QPhiX types ----------------------
// The first members keep the reference's struct layout
// (qphix_f3_internal.h:9-32): even/odd/parity for vectors, and
// lngeven/lngodd/fateven/fatodd for links -- here device pointers.
struct QPHIX_F3_ColorVector_struct {
    void *even;
    void *odd;
    int parity;
    qb::VecBlock blk[2];
};
struct QPHIX_D3_ColorVector_struct {
    void *even;
    void *odd;
    int parity;
    qb::VecBlock blk[2];
};
struct QPHIX_F3_FermionLinksAsqtad_struct {
    void *lngeven, *lngodd, *fateven, *fatodd;
    qb::LinkSet links;       // 16-matrix blocks of both output parities (FP32)
    qb::LinkSet sloppy_half;  // derived 16-bit copy (created on demand)
};
struct QPHIX_D3_FermionLinksAsqtad_struct {
    void *lngeven, *lngodd, *fateven, *fatodd;
    qb::LinkSet links;         // FP64
    qb::LinkSet sloppy_single;  // derived FP32 copy for mixed-precision solves
    qb::LinkSet sloppy_half;    // derived 16-bit copy
    qb::LinkSet sloppy_recon;   // derived FP32 copy with 12-real or 13-real Naik links
    int recon_checked = 0;      // 1: compression was tried (sloppy_recon valid if it applied)
};
// Gauge fields and momenta of the gauge force (gforce.cu): both parity
// blocks on the device, per block [dir][9 complex][Vh] (site-minor), FP32
// for F3 and FP64 for D3.  `parity` is the checkerboard whose links the
// force updates (the reference's rule: EVENODD works on EVEN).
struct QPHIX_F3_GaugeField_struct {
    void *geo;
    int parity;
    int compress12;
    void *blk[2];
};
struct QPHIX_D3_GaugeField_struct {
    void *geo;
    int parity;
    int compress12;
    void *blk[2];
};
struct QPHIX_F3_Force_struct {
    void *heo;
    void *htmp;
    int parity;
    void *blk[2];
};
struct QPHIX_D3_Force_struct {
    void *heo;
    void *htmp;
    int parity;
    void *blk[2];
};

namespace qb {

// solver drivers (solvers.cu)
struct SolveArgs {
    QPHIX_info_t *info;
    QPHIX_invert_arg_t *inv;
    QPHIX_resid_arg_t *res;
    double mass;
    VecBlock out[2];
    VecBlock in[2];
};

// CG with the reference's control flow (ks_d_congrad_fn.cpp:221-619) in
// precision p (Single for the F3 API, Double for D3)
int cg_reference(Prec p, const LinkSet &ls, SolveArgs &a);
// mixed precision: sloppy p_s inner CG, FP64 reliable updates
int cg_mixed(Prec ps, const LinkSet &ls64, const LinkSet &ls_s, const LinkSet *ls_up, SolveArgs &a);

struct MultiArgs {
    QPHIX_info_t *info;
    QPHIX_invert_arg_t *inv;
    QPHIX_resid_arg_t **res;
    const double *mass;
    int n;
    std::vector<VecBlock> out[2];
    VecBlock in[2];
};
int multishift_reference(Prec p, const LinkSet &ls, MultiArgs &a);
// ls32: the 18-real FP32 links for refining all shifts in one batched solve
// (nullptr: the shifts are refined one after the other); rop: the inner
// operator of the per-shift refinements (nullptr: the sloppy recurrence's)
struct RefineOp {
    Prec vec;
    const LinkSet *links;
    const LinkSet *up;
};
int multishift_mixed(Prec ps, const LinkSet &ls64, const LinkSet &ls_s, const LinkSet *ls_up, MultiArgs &a,
                     const LinkSet *ls32 = nullptr, const RefineOp *rop = nullptr);

}  // namespace qb
