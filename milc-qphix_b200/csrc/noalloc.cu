// Allocation-free application of the CG operator: QPHIX_B200_D3_asqtad_mdagm_noalloc.
//
// Some callers cannot allocate GPU memory at the point where they need the
// operator: code running under a fixed memory budget that was reserved up
// front, code driven from inside another framework's allocator, or code
// that must not pay the synchronisation a cudaMalloc/cudaFree may cost.
// This entry point needs, besides the caller's input and output vectors
// and the link handle, scratch for the intermediate vector D in, the
// reduction partials and a small scalar block.  That scratch lives in the
// file-scope device array below, so the call itself allocates nothing.
//
// Limits and sharing:
//  * at most kNoAllocMaxSites sites per parity (e.g. a 16^3x32 or 32^3x16
//    lattice); larger lattices are refused with QPHIX_FAIL;
//  * the array (about 12.6 MB) is part of the library image: every GPU on
//    which the library's kernels are loaded holds it until the process exits;
//  * every call uses the same array and it keeps the previous call's
//    contents; the reduction counter is cleared at the start of each call.
//    Calls whose work overlaps on the GPU (from several host threads or
//    several streams) race on the array and give wrong results;
//  * the call runs on the library's device (QPHIX_GPU_DEVICE at QPHIX_init)
//    whatever device the calling thread has current, and restores the
//    caller's current device before it returns;
//  * the device address of the array is looked up (cudaGetSymbolAddress)
//    on the first call made for each device, with that device current; make
//    that first call before any stream capture begins.
#include <cstring>
#include <mutex>

#include "context.h"
#include "device_common.cuh"

namespace qb {

namespace {

constexpr int kNoAllocMaxSites = 1 << 18;           // sites per parity block
constexpr size_t kStateBytes = 16384;               // SolverState (rounded up)
constexpr size_t kPartialBytes = 16384;             // one double per block of 256 sites
constexpr size_t kVecBytes = (size_t)3 * kNoAllocMaxSites * sizeof(double2);
constexpr size_t kScratchBytes = kStateBytes + kPartialBytes + kVecBytes;
static_assert(sizeof(SolverState) <= kStateBytes, "scalar block too small");
static_assert((kNoAllocMaxSites / kBlock) * sizeof(double) <= kPartialBytes, "partials too small");

// The scratch.  In host code the name is only a stand-in for the symbol,
// never a device address: kernels get the address from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
unsigned char *g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;  // first lookups from several host threads

// Device address of the scratch on `dev`, which must be the current device
// (a symbol's address is per device).
unsigned char *scratch_for_device(int dev)
{
    if (dev < 0 || dev >= kMaxDevices) throw Error("mdagm_noalloc: device index out of range");
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            throw Error(std::string("mdagm_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<unsigned char *>(p);
    }
    return g_scratch_addr[dev];
}

// makes `dev` current for the scope and restores the caller's device
struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int dev)
    {
        QB_CUDA(cudaGetDevice(&prev));
        if (prev != dev) QB_CUDA(cudaSetDevice(dev));
    }
    ~DeviceScope()
    {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace
}  // namespace qb

using namespace qb;

#pragma GCC visibility push(default)
extern "C" QPHIX_status_t QPHIX_B200_D3_asqtad_mdagm_noalloc(QPHIX_D3_FermionLinksAsqtad *L, QPHIX_D3_ColorVector *out,
                                                             QPHIX_D3_ColorVector *in, QPHIX_D_Real mass,
                                                             QPHIX_evenodd_t parity, double *in_dot_out)
{
    Context &c = ctx();
    try {
        if (!c.initialized) throw Error("mdagm_noalloc: QPhiX library used before QPHIX_init");
        if (c.g.vh > kNoAllocMaxSites)
            throw Error("mdagm_noalloc: lattice has " + std::to_string(c.g.vh) +
                        " sites per parity; the allocation-free path holds at most " +
                        std::to_string(kNoAllocMaxSites));
        if (c.halo.on) throw Error("mdagm_noalloc: not available with the decomposed (halo) path");
        if (!L || !out || !in) throw Error("mdagm_noalloc: NULL argument");
        if (parity != QPHIX_EVEN && parity != QPHIX_ODD)
            throw Error("mdagm_noalloc: parity must be QPHIX_EVEN or QPHIX_ODD");
        const int cb = parity == QPHIX_EVEN ? 0 : 1;
        if (!(out->parity & parity) || !(in->parity & parity) || !in->blk[cb].data || !out->blk[cb].data)
            throw Error("mdagm_noalloc: in and out must hold the requested parity");
        // the stream and the links belong to the library's device
        DeviceScope on_device(c.device);
        unsigned char *base = scratch_for_device(c.device);
        SolverState *st = reinterpret_cast<SolverState *>(base);
        double *partials = reinterpret_cast<double *>(base + kStateBytes);
        VecBlock tmp{base + kStateBytes + kPartialBytes};
        const Launch Lh = c.launch();
        // the grid reduction needs its arrival counter at zero; clear the whole
        // scalar block so nothing of an earlier call is read
        QB_CUDA(cudaMemsetAsync(st, 0, sizeof(SolverState), c.stream));
        // tmp[1-cb] = D in[cb];  out[cb] = D tmp - 4 m^2 in, with in . out reduced
        dslash_fixed_d(Lh, tmp, in->blk[cb], L->links, 1 - cb);
        dslash_mdagm_fixed_d(Lh, out->blk[cb], tmp, L->links, in->blk[cb], -4.0 * (double)mass * (double)mass, cb,
                             st, partials);
        double pkp = 0;
        QB_CUDA(cudaMemcpyAsync(&pkp, &st->pkp, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        QB_CUDA(cudaStreamSynchronize(c.stream));
        QB_CUDA(cudaGetLastError());
        if (in_dot_out) *in_dot_out = pkp;
        c.last_error.clear();
        return QPHIX_SUCCESS;
    } catch (const Error &e) {
        c.last_error = e.what();
        return e.status;
    } catch (const std::exception &e) {
        c.last_error = e.what();
        return QPHIX_FAIL;
    }
}
#pragma GCC visibility pop
