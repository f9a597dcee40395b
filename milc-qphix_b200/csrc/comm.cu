// NCCL for the domain-decomposed path (halo.h), loaded at run time.
//
// The library is linked without NCCL so a single-GPU MILC build needs
// nothing more than before; the first multi-GPU call opens libnccl.so.2
// (the system's, or the one already loaded into the process).
#include <dlfcn.h>
#include <nccl.h>

#include <cstring>
#include <mutex>
#include <string>

#include "context.h"
#include "halo.h"

namespace qb {

namespace {

struct NcclApi {
    ncclResult_t (*get_unique_id)(ncclUniqueId *) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    ncclResult_t (*group_start)() = nullptr;
    ncclResult_t (*group_end)() = nullptr;
    ncclResult_t (*send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*all_reduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                               cudaStream_t) = nullptr;
    const char *(*error_string)(ncclResult_t) = nullptr;
    bool ok = false;
    std::string why;
};

NcclApi &api()
{
    static NcclApi a;
    static std::once_flag once;
    std::call_once(once, [] {
        void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
        if (!h) {
            a.why = std::string("NCCL (libnccl.so.2) could not be loaded: ") + dlerror();
            return;
        }
        auto sym = [&](const char *n) { return dlsym(h, n); };
        a.get_unique_id = reinterpret_cast<decltype(a.get_unique_id)>(sym("ncclGetUniqueId"));
        a.comm_init_rank = reinterpret_cast<decltype(a.comm_init_rank)>(sym("ncclCommInitRank"));
        a.comm_destroy = reinterpret_cast<decltype(a.comm_destroy)>(sym("ncclCommDestroy"));
        a.group_start = reinterpret_cast<decltype(a.group_start)>(sym("ncclGroupStart"));
        a.group_end = reinterpret_cast<decltype(a.group_end)>(sym("ncclGroupEnd"));
        a.send = reinterpret_cast<decltype(a.send)>(sym("ncclSend"));
        a.recv = reinterpret_cast<decltype(a.recv)>(sym("ncclRecv"));
        a.all_reduce = reinterpret_cast<decltype(a.all_reduce)>(sym("ncclAllReduce"));
        a.error_string = reinterpret_cast<decltype(a.error_string)>(sym("ncclGetErrorString"));
        a.ok = a.get_unique_id && a.comm_init_rank && a.comm_destroy && a.group_start && a.group_end && a.send &&
               a.recv && a.all_reduce && a.error_string;
        if (!a.ok) a.why = "libnccl.so.2 lacks a symbol the library needs";
    });
    return a;
}

const NcclApi &need()
{
    const NcclApi &a = api();
    if (!a.ok) throw Error(a.why);
    return a;
}

void check(ncclResult_t r, const char *what)
{
    if (r != ncclSuccess) throw Error(std::string(what) + ": " + api().error_string(r));
}

}  // namespace

bool nccl_available() { return api().ok; }

void nccl_unique_id(void *id128)
{
    static_assert(sizeof(ncclUniqueId) == 128, "ncclUniqueId is 128 bytes");
    ncclUniqueId id;
    check(need().get_unique_id(&id), "ncclGetUniqueId");
    std::memcpy(id128, &id, sizeof(id));
}

void *nccl_comm_init(const void *id128, int nranks, int rank)
{
    ncclUniqueId id;
    std::memcpy(&id, id128, sizeof(id));
    ncclComm_t comm = nullptr;
    check(need().comm_init_rank(&comm, nranks, id, rank), "ncclCommInitRank");
    return comm;
}

void nccl_comm_destroy(void *comm)
{
    if (comm && api().ok) api().comm_destroy(static_cast<ncclComm_t>(comm));
}

void nccl_allreduce_sum(void *comm, double *dev, int n, cudaStream_t stream)
{
    check(need().all_reduce(dev, dev, (size_t)n, ncclDouble, ncclSum, static_cast<ncclComm_t>(comm), stream),
          "ncclAllReduce");
}

void nccl_exchange(void *comm, const void *sback, const void *sfwd, void *gback, void *gfwd, size_t bytes, int prev,
                   int next, cudaStream_t stream)
{
    const NcclApi &a = need();
    ncclComm_t c = static_cast<ncclComm_t>(comm);
    // Between a pair of ranks NCCL matches sends and receives in issue
    // order.  Every rank issues (send to prev, receive from next, send to
    // next, receive from prev); with two ranks prev == next, and the first
    // send (our first slices) meets the peer's first receive (its forward
    // ghost), the second send (our last slices) its backward ghost.
    check(a.group_start(), "ncclGroupStart");
    check(a.send(sback, bytes, ncclUint8, prev, c, stream), "ncclSend");
    check(a.recv(gfwd, bytes, ncclUint8, next, c, stream), "ncclRecv");
    check(a.send(sfwd, bytes, ncclUint8, next, c, stream), "ncclSend");
    check(a.recv(gback, bytes, ncclUint8, prev, c, stream), "ncclRecv");
    check(a.group_end(), "ncclGroupEnd");
}

}  // namespace qb
