// Single-rank MPI shim implementation -- TEST INFRASTRUCTURE ONLY.
// See mpi.h in this directory for the semantics provided.
#include "mpi.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

int g_initialized = 0;
int g_finalized = 0;

struct CartComm {
    int periods[3];
};
std::vector<CartComm> g_carts;  // communicator id = 2 + index

struct Pending {
    bool isSend;
    const void* sendBuf;
    void* recvBuf;
    std::size_t bytes;
    int tag;
    bool done;
};
std::vector<Pending> g_pending;

std::size_t typeSize(MPI_Datatype t) {
    switch (t) {
        case MPI_DOUBLE: return sizeof(double);
        case MPI_INT: return sizeof(int);
        default: return 0;
    }
}

}  // namespace

extern "C" {

int MPI_Init(int*, char***) { g_initialized = 1; return MPI_SUCCESS; }
int MPI_Initialized(int* flag) { *flag = g_initialized; return MPI_SUCCESS; }
int MPI_Finalize(void) { g_finalized = 1; return MPI_SUCCESS; }
int MPI_Finalized(int* flag) { *flag = g_finalized; return MPI_SUCCESS; }

int MPI_Abort(MPI_Comm, int code) {
    std::fprintf(stderr, "MPI_Abort(%d) called in single-rank shim\n", code);
    std::exit(code);
}

int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
int MPI_Comm_free(MPI_Comm* comm) { *comm = MPI_COMM_NULL; return MPI_SUCCESS; }

int MPI_Dims_create(int, int ndims, int dims[]) {
    for (int d = 0; d < ndims; ++d)
        if (dims[d] == 0) dims[d] = 1;
    return MPI_SUCCESS;
}

int MPI_Cart_create(MPI_Comm, int ndims, const int[], const int periods[], int,
                    MPI_Comm* cart) {
    CartComm c{{0, 0, 0}};
    for (int d = 0; d < ndims && d < 3; ++d) c.periods[d] = periods[d];
    g_carts.push_back(c);
    *cart = 2 + static_cast<int>(g_carts.size()) - 1;
    return MPI_SUCCESS;
}

int MPI_Cart_coords(MPI_Comm, int, int maxdims, int coords[]) {
    for (int d = 0; d < maxdims; ++d) coords[d] = 0;
    return MPI_SUCCESS;
}

int MPI_Cart_shift(MPI_Comm comm, int direction, int, int* source, int* dest) {
    int idx = comm - 2;
    int periodic = 0;
    if (idx >= 0 && idx < static_cast<int>(g_carts.size()) && direction >= 0 && direction < 3)
        periodic = g_carts[idx].periods[direction];
    *source = periodic ? 0 : MPI_PROC_NULL;
    *dest = periodic ? 0 : MPI_PROC_NULL;
    return MPI_SUCCESS;
}

int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type,
                  MPI_Op, MPI_Comm) {
    if (sendbuf != MPI_IN_PLACE)
        std::memcpy(recvbuf, sendbuf, typeSize(type) * static_cast<std::size_t>(count));
    return MPI_SUCCESS;
}

int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
               int, MPI_Datatype, int, MPI_Comm) {
    if (sendbuf != MPI_IN_PLACE)
        std::memcpy(recvbuf, sendbuf, typeSize(sendtype) * static_cast<std::size_t>(sendcount));
    return MPI_SUCCESS;
}

int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm,
              MPI_Request* req) {
    if (dest == MPI_PROC_NULL) { *req = -1; return MPI_SUCCESS; }
    g_pending.push_back({true, buf, nullptr, typeSize(type) * static_cast<std::size_t>(count), tag, false});
    *req = static_cast<int>(g_pending.size()) - 1;
    return MPI_SUCCESS;
}

int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm,
              MPI_Request* req) {
    if (source == MPI_PROC_NULL) { *req = -1; return MPI_SUCCESS; }
    g_pending.push_back({false, nullptr, buf, typeSize(type) * static_cast<std::size_t>(count), tag, false});
    *req = static_cast<int>(g_pending.size()) - 1;
    return MPI_SUCCESS;
}

int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status*) {
    // Match every receive with the first unmatched send of the same tag.
    for (int r = 0; r < count; ++r) {
        if (reqs[r] < 0) continue;
        Pending& rv = g_pending[reqs[r]];
        if (rv.isSend || rv.done) continue;
        for (int s = 0; s < count; ++s) {
            if (reqs[s] < 0) continue;
            Pending& sd = g_pending[reqs[s]];
            if (!sd.isSend || sd.done || sd.tag != rv.tag) continue;
            std::memcpy(rv.recvBuf, sd.sendBuf, rv.bytes < sd.bytes ? rv.bytes : sd.bytes);
            sd.done = true;
            rv.done = true;
            break;
        }
        if (!rv.done) {
            std::fprintf(stderr, "single-rank MPI shim: unmatched receive (tag %d)\n", rv.tag);
            std::abort();
        }
    }
    g_pending.clear();
    return MPI_SUCCESS;
}

}  // extern "C"
