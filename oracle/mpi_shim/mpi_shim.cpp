// MPI shim implementation -- TEST INFRASTRUCTURE ONLY.
// See mpi.h in this directory for the semantics provided.
//
// Two modes.  By default the process is one rank (MPI_COMM_WORLD of size
// 1).  Inside sifv_mpi_shim_run(nranks, fn, user) the world has nranks
// ranks, each a thread of this process running fn(user, rank): the
// reference keeps no mutable static state, so one process holds every
// rank's objects and messages are copies between the threads' buffers.
#include "mpi.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

namespace {

int g_initialized = 0;
int g_finalized = 0;

// Waits on other ranks give up after this long (a rank that died or a
// protocol mismatch), printing where, instead of hanging the process.
constexpr auto kWaitLimit = std::chrono::seconds(900);

struct CartComm {
    int ndims;
    int dims[3];
    int periods[3];
};

struct Message {
    int src;
    int tag;
    std::vector<char> data;
};

// The world shared by the rank threads of one sifv_mpi_shim_run call.
struct World {
    int size = 1;
    std::mutex m;
    std::condition_variable cv;
    std::vector<std::deque<Message>> inbox;   // per destination rank
    // collectives: contributions of the current round, the result of the
    // last completed round, and the round counter
    int arrived = 0;
    long long round = 0;
    std::vector<std::vector<char>> contrib;
    std::vector<char> result;
};

World* g_world = nullptr;          // set while sifv_mpi_shim_run runs
thread_local int t_rank = 0;
thread_local std::vector<CartComm> t_carts;   // communicator id = 2 + index (per rank, same order on every rank)

struct Pending {
    bool isSend;
    const void* sendBuf;
    void* recvBuf;
    std::size_t bytes;
    int peer;
    int tag;
    bool done;
};
thread_local std::vector<Pending> t_pending;

std::size_t typeSize(MPI_Datatype t) {
    switch (t) {
        case MPI_DOUBLE: return sizeof(double);
        case MPI_INT: return sizeof(int);
        default: return 0;
    }
}

int worldSize() { return g_world ? g_world->size : 1; }

[[noreturn]] void die(const char* what) {
    std::fprintf(stderr, "MPI shim (rank %d of %d): %s\n", t_rank, worldSize(), what);
    std::abort();
}

template <typename T>
void reduceInto(T* acc, const T* x, int count, MPI_Op op) {
    for (int i = 0; i < count; ++i) {
        switch (op) {
            case MPI_MIN: acc[i] = (x[i] < acc[i]) ? x[i] : acc[i]; break;
            case MPI_MAX: acc[i] = (x[i] > acc[i]) ? x[i] : acc[i]; break;
            default: acc[i] = acc[i] + x[i]; break;
        }
    }
}

// One collective round: every rank deposits `mine`; the last to arrive
// builds the result with `combine` (contributions in rank order, so the
// result does not depend on arrival order) and wakes the others, who copy
// it out before any rank can complete the next round.
template <typename Combine>
std::vector<char> collective(const void* mine, std::size_t bytes, Combine combine) {
    World& w = *g_world;
    std::unique_lock<std::mutex> lock(w.m);
    w.contrib[t_rank].assign(static_cast<const char*>(mine), static_cast<const char*>(mine) + bytes);
    if (++w.arrived == w.size) {
        w.result = combine(w.contrib);
        w.arrived = 0;
        ++w.round;
        w.cv.notify_all();
        return w.result;
    }
    const long long r = w.round;
    if (!w.cv.wait_for(lock, kWaitLimit, [&] { return w.round != r; })) die("collective timed out");
    return w.result;
}

}  // namespace

extern "C" {

int MPI_Init(int*, char***) { g_initialized = 1; return MPI_SUCCESS; }
int MPI_Initialized(int* flag) { *flag = g_initialized; return MPI_SUCCESS; }
int MPI_Finalize(void) { g_finalized = 1; return MPI_SUCCESS; }
int MPI_Finalized(int* flag) { *flag = g_finalized; return MPI_SUCCESS; }

int MPI_Abort(MPI_Comm, int code) {
    std::fprintf(stderr, "MPI_Abort(%d) called (MPI shim, rank %d)\n", code, t_rank);
    std::exit(code);
}

int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = t_rank; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int* size) { *size = worldSize(); return MPI_SUCCESS; }
int MPI_Comm_free(MPI_Comm* comm) { *comm = MPI_COMM_NULL; return MPI_SUCCESS; }

// Balanced factorisation of nnodes over the dimensions left at 0, in
// non-increasing order (the behaviour MPI specifies for MPI_Dims_create):
// prime factors, largest first, each to the currently smallest free
// dimension.
int MPI_Dims_create(int nnodes, int ndims, int dims[]) {
    int fixed = 1, nfree = 0;
    for (int d = 0; d < ndims; ++d) {
        if (dims[d] > 0) fixed *= dims[d];
        else ++nfree;
    }
    if (nfree == 0) return MPI_SUCCESS;
    int rest = (fixed > 0 && nnodes % fixed == 0) ? nnodes / fixed : 1;
    std::vector<int> primes;
    for (int p = 2; p * p <= rest; ++p)
        while (rest % p == 0) { primes.push_back(p); rest /= p; }
    if (rest > 1) primes.push_back(rest);
    std::sort(primes.rbegin(), primes.rend());
    std::vector<int> f(nfree, 1);
    for (int p : primes) *std::min_element(f.begin(), f.end()) *= p;
    std::sort(f.rbegin(), f.rend());
    for (int d = 0, k = 0; d < ndims; ++d)
        if (dims[d] <= 0) dims[d] = f[k++];
    return MPI_SUCCESS;
}

int MPI_Cart_create(MPI_Comm, int ndims, const int dims[], const int periods[], int, MPI_Comm* cart) {
    CartComm c{ndims < 3 ? ndims : 3, {1, 1, 1}, {0, 0, 0}};
    for (int d = 0; d < c.ndims; ++d) {
        c.dims[d] = dims[d];
        c.periods[d] = periods[d];
    }
    t_carts.push_back(c);
    *cart = 2 + static_cast<int>(t_carts.size()) - 1;
    return MPI_SUCCESS;
}

static const CartComm* cartOf(MPI_Comm comm) {
    int idx = comm - 2;
    if (idx >= 0 && idx < static_cast<int>(t_carts.size())) return &t_carts[idx];
    return nullptr;
}

// Row-major rank order (the last dimension varies fastest), no reordering.
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int coords[]) {
    const CartComm* c = cartOf(comm);
    for (int d = 0; d < maxdims; ++d) coords[d] = 0;
    if (!c) return MPI_SUCCESS;
    int r = rank;
    for (int d = c->ndims - 1; d >= 0; --d) {
        if (d < maxdims) coords[d] = r % c->dims[d];
        r /= c->dims[d];
    }
    return MPI_SUCCESS;
}

int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int* source, int* dest) {
    const CartComm* c = cartOf(comm);
    if (!c || direction < 0 || direction >= c->ndims) {
        *source = *dest = MPI_PROC_NULL;
        return MPI_SUCCESS;
    }
    int coords[3] = {0, 0, 0};
    MPI_Cart_coords(comm, t_rank, 3, coords);
    auto rankAt = [&](int shift) -> int {
        int cc[3] = {coords[0], coords[1], coords[2]};
        int n = c->dims[direction];
        int v = cc[direction] + shift;
        if (v < 0 || v >= n) {
            if (!c->periods[direction]) return MPI_PROC_NULL;
            v = ((v % n) + n) % n;
        }
        cc[direction] = v;
        int r = 0;
        for (int d = 0; d < c->ndims; ++d) r = r * c->dims[d] + cc[d];
        return r;
    };
    *source = rankAt(-disp);
    *dest = rankAt(disp);
    return MPI_SUCCESS;
}

int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm) {
    const std::size_t bytes = typeSize(type) * static_cast<std::size_t>(count);
    const void* mine = (sendbuf == MPI_IN_PLACE) ? recvbuf : sendbuf;
    if (!g_world) {
        if (sendbuf != MPI_IN_PLACE) std::memcpy(recvbuf, sendbuf, bytes);
        return MPI_SUCCESS;
    }
    std::vector<char> r = collective(mine, bytes, [&](const std::vector<std::vector<char>>& all) {
        std::vector<char> acc = all[0];
        for (std::size_t k = 1; k < all.size(); ++k) {
            if (type == MPI_DOUBLE)
                reduceInto(reinterpret_cast<double*>(acc.data()), reinterpret_cast<const double*>(all[k].data()),
                           count, op);
            else
                reduceInto(reinterpret_cast<int*>(acc.data()), reinterpret_cast<const int*>(all[k].data()), count,
                           op);
        }
        return acc;
    });
    std::memcpy(recvbuf, r.data(), bytes);
    return MPI_SUCCESS;
}

int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int, MPI_Datatype, int root,
               MPI_Comm) {
    const std::size_t bytes = typeSize(sendtype) * static_cast<std::size_t>(sendcount);
    if (!g_world) {
        if (sendbuf != MPI_IN_PLACE) std::memcpy(recvbuf, sendbuf, bytes);
        return MPI_SUCCESS;
    }
    std::vector<char> r = collective(sendbuf, bytes, [&](const std::vector<std::vector<char>>& all) {
        std::vector<char> cat;
        for (const auto& a : all) cat.insert(cat.end(), a.begin(), a.end());
        return cat;
    });
    if (t_rank == root) std::memcpy(recvbuf, r.data(), r.size());
    return MPI_SUCCESS;
}

// Sends are buffered: the data is copied into the destination's inbox at
// once, so a send completes without waiting for its receive.
int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm, MPI_Request* req) {
    if (dest == MPI_PROC_NULL) { *req = -1; return MPI_SUCCESS; }
    const std::size_t bytes = typeSize(type) * static_cast<std::size_t>(count);
    if (g_world) {
        if (dest < 0 || dest >= g_world->size) die("send to a rank outside the world");
        Message msg{t_rank, tag, std::vector<char>(static_cast<const char*>(buf), static_cast<const char*>(buf) + bytes)};
        {
            std::lock_guard<std::mutex> lock(g_world->m);
            g_world->inbox[dest].push_back(std::move(msg));
        }
        g_world->cv.notify_all();
        *req = -1;
        return MPI_SUCCESS;
    }
    t_pending.push_back({true, buf, nullptr, bytes, dest, tag, false});
    *req = static_cast<int>(t_pending.size()) - 1;
    return MPI_SUCCESS;
}

int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm, MPI_Request* req) {
    if (source == MPI_PROC_NULL) { *req = -1; return MPI_SUCCESS; }
    t_pending.push_back({false, nullptr, buf, typeSize(type) * static_cast<std::size_t>(count), source, tag, false});
    *req = static_cast<int>(t_pending.size()) - 1;
    return MPI_SUCCESS;
}

int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status*) {
    if (g_world) {
        // every receive takes the oldest message of its (source, tag)
        World& w = *g_world;
        std::unique_lock<std::mutex> lock(w.m);
        for (int r = 0; r < count; ++r) {
            if (reqs[r] < 0) continue;
            Pending& rv = t_pending[reqs[r]];
            if (rv.isSend || rv.done) continue;
            auto& box = w.inbox[t_rank];
            auto match = [&] {
                return std::find_if(box.begin(), box.end(),
                                    [&](const Message& m) { return m.src == rv.peer && m.tag == rv.tag; });
            };
            if (!w.cv.wait_for(lock, kWaitLimit, [&] { return match() != box.end(); }))
                die("receive timed out");
            auto it = match();
            std::memcpy(rv.recvBuf, it->data.data(), std::min(rv.bytes, it->data.size()));
            box.erase(it);
            rv.done = true;
        }
        t_pending.clear();
        return MPI_SUCCESS;
    }
    // one rank: every receive is matched with the first unmatched send of
    // the same tag (the periodic self-exchange)
    for (int r = 0; r < count; ++r) {
        if (reqs[r] < 0) continue;
        Pending& rv = t_pending[reqs[r]];
        if (rv.isSend || rv.done) continue;
        for (int s = 0; s < count; ++s) {
            if (reqs[s] < 0) continue;
            Pending& sd = t_pending[reqs[s]];
            if (!sd.isSend || sd.done || sd.tag != rv.tag) continue;
            std::memcpy(rv.recvBuf, sd.sendBuf, rv.bytes < sd.bytes ? rv.bytes : sd.bytes);
            sd.done = true;
            rv.done = true;
            break;
        }
        if (!rv.done) die("unmatched receive");
    }
    t_pending.clear();
    return MPI_SUCCESS;
}

int sifv_mpi_shim_run(int nranks, void (*fn)(void* user, int rank), void* user) {
    if (nranks < 1 || g_world) return -1;
    World w;
    w.size = nranks;
    w.inbox.resize(nranks);
    w.contrib.resize(nranks);
    g_world = &w;
    g_initialized = 1;
    std::vector<std::thread> threads;
    threads.reserve(nranks);
    for (int r = 0; r < nranks; ++r)
        threads.emplace_back([=] {
            t_rank = r;
            t_carts.clear();
            t_pending.clear();
            fn(user, r);
            t_carts.clear();
        });
    for (auto& t : threads) t.join();
    g_world = nullptr;
    t_rank = 0;
    return 0;
}

}  // extern "C"
