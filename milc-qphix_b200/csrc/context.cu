// Context, device memory and state transfer helpers.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <thread>

#include "context.h"
#include "device_common.cuh"

namespace qb {

Context &ctx()
{
    static Context c;
    return c;
}

double wall_seconds()
{
    using namespace std::chrono;
    return duration<double>(system_clock::now().time_since_epoch()).count();
}

void *dev_alloc(size_t bytes)
{
    void *p = nullptr;
    if (bytes == 0) return nullptr;
    QB_CUDA(cudaMallocAsync(&p, bytes, ctx().stream));
    return p;
}

void dev_free(void *p)
{
    if (p) cudaFreeAsync(p, ctx().stream);
}

namespace {

constexpr size_t kStageBytes = 8u << 20;      // one pinned slot
constexpr size_t kStageMinBytes = 16u << 20;  // smaller copies go in one call

void make_staging(Context &c)
{
    HostStaging &h = c.staging;
    if (h.workers) return;
    const unsigned hw = std::thread::hardware_concurrency();
    const int w = (int)std::max(1u, std::min(8u, hw / 2));
    for (int i = 0; i < w; ++i) {
        cudaStream_t s;
        QB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        h.streams.push_back(s);
        for (int k = 0; k < 2; ++k) {
            void *p = nullptr;
            QB_CUDA(cudaHostAlloc(&p, kStageBytes, cudaHostAllocDefault));
            h.slots.push_back(static_cast<char *>(p));
            cudaEvent_t e;
            QB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            h.done.push_back(e);
        }
        h.workers = i + 1;
    }
}

}  // namespace

void free_staging()
{
    HostStaging &h = ctx().staging;
    for (auto s : h.streams) cudaStreamDestroy(s);
    for (auto p : h.slots) cudaFreeHost(p);
    for (auto e : h.done) cudaEventDestroy(e);
    h = HostStaging{};
}

void h2d_copy(void *dst, const void *src, size_t bytes)
{
    Context &c = ctx();
    if (bytes == 0) return;
    // only plain pageable host memory is staged; pinned, managed or device
    // memory goes by one copy (direction from the unified address space)
    cudaPointerAttributes at{};
    const bool pageable = cudaPointerGetAttributes(&at, src) != cudaSuccess || at.type == cudaMemoryTypeUnregistered;
    cudaGetLastError();  // an unregistered pointer is not an error here
    if (!pageable || bytes < kStageMinBytes) {
        QB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, c.stream));
        QB_CUDA(cudaStreamSynchronize(c.stream));
        return;
    }
    make_staging(c);
    // work already queued on the library stream (e.g. a memset of dst)
    // finishes before the worker streams write dst
    QB_CUDA(cudaStreamSynchronize(c.stream));
    HostStaging &h = c.staging;
    const int W = h.workers;
    std::atomic<int> failed{0};
    std::vector<std::thread> th;
    for (int w = 0; w < W; ++w) {
        th.emplace_back([&, w] {
            if (cudaSetDevice(c.device) != cudaSuccess) { failed = 1; return; }
            // contiguous part of the source, 4 KiB aligned
            const size_t lo = (bytes * w / W) & ~(size_t)4095, hi = w + 1 == W ? bytes : (bytes * (w + 1) / W) & ~(size_t)4095;
            int k = 0;
            for (size_t off = lo; off < hi; off += kStageBytes, ++k) {
                const size_t n = std::min(kStageBytes, hi - off);
                const int sl = 2 * w + (k & 1);
                if (k >= 2 && cudaEventSynchronize(h.done[sl]) != cudaSuccess) { failed = 1; break; }
                std::memcpy(h.slots[sl], static_cast<const char *>(src) + off, n);
                if (cudaMemcpyAsync(static_cast<char *>(dst) + off, h.slots[sl], n, cudaMemcpyHostToDevice,
                                    h.streams[w]) != cudaSuccess ||
                    cudaEventRecord(h.done[sl], h.streams[w]) != cudaSuccess) {
                    failed = 1;
                    break;
                }
            }
            if (cudaStreamSynchronize(h.streams[w]) != cudaSuccess) failed = 1;
        });
    }
    for (auto &t : th) t.join();
    if (failed) throw Error("host to device copy through pinned staging failed");
}

void d2h_copy(void *dst, const void *src, size_t bytes)
{
    Context &c = ctx();
    if (bytes == 0) return;
    cudaPointerAttributes at{};
    const bool pageable = cudaPointerGetAttributes(&at, dst) != cudaSuccess || at.type == cudaMemoryTypeUnregistered;
    cudaGetLastError();  // an unregistered pointer is not an error here
    if (!pageable || bytes < kStageMinBytes) {
        QB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, c.stream));
        QB_CUDA(cudaStreamSynchronize(c.stream));
        return;
    }
    make_staging(c);
    // the kernels that produce src finish before the worker streams read it
    QB_CUDA(cudaStreamSynchronize(c.stream));
    HostStaging &h = c.staging;
    const int W = h.workers;
    std::atomic<int> failed{0};
    std::vector<std::thread> th;
    for (int w = 0; w < W; ++w) {
        th.emplace_back([&, w] {
            if (cudaSetDevice(c.device) != cudaSuccess) { failed = 1; return; }
            const size_t lo = (bytes * w / W) & ~(size_t)4095, hi = w + 1 == W ? bytes : (bytes * (w + 1) / W) & ~(size_t)4095;
            // chunk k goes device -> slot k&1 while the host copies chunk k-1 out of the other slot
            size_t prev_off = 0, prev_n = 0;
            int k = 0;
            auto drain = [&](int slot) {
                if (cudaEventSynchronize(h.done[slot]) != cudaSuccess) { failed = 1; return false; }
                std::memcpy(static_cast<char *>(dst) + prev_off, h.slots[slot], prev_n);
                return true;
            };
            for (size_t off = lo; off < hi; off += kStageBytes, ++k) {
                const size_t n = std::min(kStageBytes, hi - off);
                const int sl = 2 * w + (k & 1);
                if (cudaMemcpyAsync(h.slots[sl], static_cast<const char *>(src) + off, n, cudaMemcpyDeviceToHost,
                                    h.streams[w]) != cudaSuccess ||
                    cudaEventRecord(h.done[sl], h.streams[w]) != cudaSuccess) {
                    failed = 1;
                    break;
                }
                if (k > 0 && !drain(2 * w + ((k - 1) & 1))) break;
                prev_off = off;
                prev_n = n;
            }
            if (!failed && k > 0) drain(2 * w + ((k - 1) & 1));
            if (cudaStreamSynchronize(h.streams[w]) != cudaSuccess) failed = 1;
        });
    }
    for (auto &t : th) t.join();
    if (failed) throw Error("device to host copy through pinned staging failed");
}

void check_lattice(const int L[4], const char *who)
{
    const std::string w(who);
    for (int i = 0; i < 4; ++i)
        if (L[i] <= 0) throw Error(w + ": non-positive lattice extent");
    if (L[0] % 2) throw Error(w + ": Nx must be even");
    if ((L[0] / 2) % 2 != 0) throw Error(w + ": Nx/2 must be even");
    if (L[1] % 4 || L[2] % 4 || L[3] % 4) throw Error(w + ": Ny, Nz and Nt must be multiples of 4");
    const long long V = (long long)L[0] * L[1] * L[2] * L[3];
    if (V / 2 > (1LL << 30)) throw Error(w + ": lattice too large for 32-bit site indices");
    if (2LL * ((V / 2 + kBlock - 1) / kBlock) > 4LL * kMaxPartials)
        throw Error(w + ": lattice too large for one GPU's reduction scratch");
}

static size_t cx_bytes(Prec p) { return p == Prec::Double ? 16 : (p == Prec::Single ? 8 : 4); }

VecBlock alloc_vec(Prec p)
{
    Context &c = ctx();
    VecBlock b;
    b.data = dev_alloc(vec_bytes(p, c.g.vh));
    QB_CUDA(cudaMemsetAsync(b.data, 0, vec_bytes(p, c.g.vh), c.stream));
    return b;
}

void free_vec(VecBlock &b)
{
    dev_free(b.data);
    b.data = nullptr;
}

LinkSet alloc_links(Prec p) { return alloc_links(p, ctx().g.vh); }

LinkSet alloc_links(Prec p, int vh)
{
    Context &c = ctx();
    LinkSet ls;
    const size_t bytes = (size_t)kMats * 9 * vh * cx_bytes(p);
    for (int cb = 0; cb < 2; ++cb) {
        ls.blk[cb] = dev_alloc(bytes);
        QB_CUDA(cudaMemsetAsync(ls.blk[cb], 0, bytes, c.stream));
    }
    ls.prec = p;
    ls.valid = true;
    return ls;
}

void free_links(LinkSet &ls)
{
    for (int cb = 0; cb < 2; ++cb) {
        dev_free(ls.blk[cb]);
        dev_free(ls.sign[cb]);
        dev_free(ls.lam[cb]);
        ls.blk[cb] = nullptr;
        ls.sign[cb] = nullptr;
        ls.lam[cb] = nullptr;
    }
    ls.valid = false;
    ls.recon = 0;
}

void upload_state()
{
    Context &c = ctx();
    QB_CUDA(cudaMemcpyAsync(c.d_state, c.h_state, sizeof(SolverState), cudaMemcpyHostToDevice, c.stream));
    // the pinned mirror is edited again right after; let the copy land first
    QB_CUDA(cudaStreamSynchronize(c.stream));
}

void download_state()
{
    Context &c = ctx();
    QB_CUDA(cudaMemcpyAsync(c.h_state, c.d_state, sizeof(SolverState), cudaMemcpyDeviceToHost, c.stream));
    sync_check();
}

void sync_check()
{
    Context &c = ctx();
    QB_CUDA(cudaStreamSynchronize(c.stream));
    if (!c.d_err) return;
    int e = 0;
    QB_CUDA(cudaMemcpy(&e, c.d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        QB_CUDA(cudaMemset(c.d_err, 0, sizeof(int)));
        throw Error("a Dslash pipeline wait timed out on the GPU; the call's results are invalid");
    }
}

}  // namespace qb
