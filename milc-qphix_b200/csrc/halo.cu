// Set-up of the domain-decomposed path (halo.h): the communicator, the
// decomposition of the QPHIX_init lattice and the ghost buffers.
#include <cstdlib>
#include <string>

#include "context.h"
#include "halo.h"

namespace qb {

namespace {

// the NCCL communicator outlives QPHIX_init / QPHIX_finalize cycles, as an
// MPI communicator does for the reference
struct CommState {
    void *comm = nullptr;
    int nranks = 1, rank = 0;
};
CommState g_comm;
bool g_loopback = false;

// bytes per site of one parity-block vector in precision pi (Prec index)
size_t site_bytes(int pi) { return pi == (int)Prec::Double ? 48 : (pi == (int)Prec::Single ? 24 : 16); }

}  // namespace

void comm_init(const void *id128, int nranks, int rank)
{
    if (!id128) throw Error("comm_init: NULL unique id");
    if (nranks < 1 || rank < 0 || rank >= nranks) throw Error("comm_init: bad nranks / rank");
    if (ctx().initialized) throw Error("comm_init: call before QPHIX_init");
    if (g_comm.comm) throw Error("comm_init: a communicator exists; call QPHIX_B200_comm_finalize first");
    const char *dev = std::getenv("QPHIX_GPU_DEVICE");
    QB_CUDA(cudaSetDevice(dev ? std::atoi(dev) : 0));
    if (nranks > 1) g_comm.comm = nccl_comm_init(id128, nranks, rank);
    g_comm.nranks = nranks;
    g_comm.rank = rank;
}

void comm_finalize()
{
    if (ctx().initialized) throw Error("comm_finalize: call after QPHIX_finalize");
    nccl_comm_destroy(g_comm.comm);
    g_comm = CommState{};
}

int comm_nranks() { return g_comm.nranks; }
int comm_rank() { return g_comm.rank; }
void set_loopback(bool on) { g_loopback = on; }
bool loopback() { return g_loopback; }

void halo_free(Context &c)
{
    Halo &h = c.halo;
    for (int p = 0; p < 3; ++p) {
        if (h.gback[p]) cudaFree(h.gback[p]);
        if (h.nranks > 1) {
            if (h.sback[p]) cudaFree(h.sback[p]);
        }
    }
    if (h.comm_stream) cudaStreamDestroy(h.comm_stream);
    if (h.ev_packed) cudaEventDestroy(h.ev_packed);
    if (h.ev_recv) cudaEventDestroy(h.ev_recv);
    h = Halo{};
}

// Ghost and send buffers for the lattice c.g cut along t into `nranks`
// slabs.  One allocation per precision holds the backward and forward
// ghosts (and, with several GPUs, the two send buffers); with one GPU the
// send buffers are the ghosts themselves (loopback).
void halo_setup(Context &c, int nranks, int rank, long long global_sites)
{
    halo_free(c);
    Halo &h = c.halo;
    if (nranks == 1 && !g_loopback) return;
    h.nranks = nranks;
    h.rank = rank;
    h.prev = (rank + nranks - 1) % nranks;
    h.next = (rank + 1) % nranks;
    h.comm = g_comm.comm;
    h.global_sites = global_sites;
    for (int p = 0; p < 3; ++p) {
        h.face_bytes[p] = (size_t)3 * c.g.st * site_bytes(p);
        char *g = nullptr;
        QB_CUDA(cudaMalloc(&g, 2 * h.face_bytes[p]));
        QB_CUDA(cudaMemset(g, 0, 2 * h.face_bytes[p]));
        h.gback[p] = g;
        h.gfwd[p] = g + h.face_bytes[p];
        if (nranks > 1) {
            char *sb = nullptr;
            QB_CUDA(cudaMalloc(&sb, 2 * h.face_bytes[p]));
            h.sback[p] = sb;
            h.sfwd[p] = sb + h.face_bytes[p];
        } else {
            // the rank is its own t neighbour: its first slices are its
            // forward ghost, its last slices its backward ghost
            h.sback[p] = h.gfwd[p];
            h.sfwd[p] = h.gback[p];
        }
    }
    if (nranks > 1) {
        QB_CUDA(cudaStreamCreateWithFlags(&h.comm_stream, cudaStreamNonBlocking));
        QB_CUDA(cudaEventCreateWithFlags(&h.ev_packed, cudaEventDisableTiming));
        QB_CUDA(cudaEventCreateWithFlags(&h.ev_recv, cudaEventDisableTiming));
    }
    h.on = true;
}

}  // namespace qb
