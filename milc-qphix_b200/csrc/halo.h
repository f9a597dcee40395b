// Domain decomposition over several GPUs: the lattice cut into slabs along
// t, one slab per process and GPU.
//
// The reference runs one MPI rank per node.  Before each Dslash it packs the
// depth-3 faces of the input parity into send buffers (pack_face,
// ks_boundary.cpp:440-557), exchanges them with its neighbours
// (:694-825), computes the interior while the messages travel and
// finishes the boundary sites from the received faces (unpack_face,
// :559-690); every dot product is summed over ranks (g_doublesum,
// ks_blas_utils_c.cpp:101-107).
//
// Here each GPU keeps, per vector precision, a ghost buffer of the three
// t-slices before and after its slab (input parity only).  A Dslash with
// the halo on
//   1. packs its own first and last three t-slices into send buffers (one
//      small kernel),
//   2. sends them to the t-neighbours and receives theirs straight into its
//      ghost buffer (NCCL send/recv over NVLink, on a communication stream),
//   3. meanwhile computes the interior sites (3 <= t < Nt-3),
//   4. then the boundary sites, whose t-neighbours come from the ghost
//      buffer.
// The reductions of the solvers end in one ncclAllReduce of their FP64
// totals and a one-thread kernel that takes the solver's scalar step.
// With one process and the loopback switch the same path runs on one GPU:
// every send buffer is the matching receive buffer (the rank is its own t
// neighbour), as in the reference's ASSUME_MULTINODE
// (ks_boundary.cpp:196-200, 250-256), so the pack -> ghost -> boundary path
// reproduces the periodic Dslash.  No TMA or bulk copy reads another GPU's
// memory, and no library kernel is given a peer pointer: faces arrive in
// each GPU's own memory through NCCL.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace qb {

struct Halo {
    bool on = false;         // t faces go through the ghost buffers
    int nranks = 1, rank = 0;
    int prev = 0, next = 0;  // ranks of the t-neighbours
    void *comm = nullptr;    // ncclComm_t (nranks > 1)
    cudaStream_t comm_stream = nullptr;
    cudaEvent_t ev_packed = nullptr, ev_recv = nullptr;
    // per vector precision (Prec index): ghost of t = -3..-1 and t = Nt..Nt+2,
    // and the send buffers (aliases of the ghosts in loopback)
    void *gback[3] = {nullptr, nullptr, nullptr}, *gfwd[3] = {nullptr, nullptr, nullptr};
    void *sback[3] = {nullptr, nullptr, nullptr}, *sfwd[3] = {nullptr, nullptr, nullptr};
    size_t face_bytes[3] = {0, 0, 0};  // bytes of three t-slices of one parity
    long long global_sites = 0;        // sites of the whole lattice
};

// NCCL, loaded at run time (libnccl.so.2) so linking the library needs no
// NCCL; throws when it is missing
bool nccl_available();
void nccl_unique_id(void *id128);
void *nccl_comm_init(const void *id128, int nranks, int rank);
void nccl_comm_destroy(void *comm);
// in-place sum of n doubles over the ranks, on `stream`
void nccl_allreduce_sum(void *comm, double *dev, int n, cudaStream_t stream);
// grouped face exchange: send sback to prev and sfwd to next, receive the
// next rank's into gfwd and the previous rank's into gback
void nccl_exchange(void *comm, const void *sback, const void *sfwd, void *gback, void *gfwd, size_t bytes,
                   int prev, int next, cudaStream_t stream);

}  // namespace qb
