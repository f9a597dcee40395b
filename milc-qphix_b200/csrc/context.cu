// Context, device memory and state transfer helpers.
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
