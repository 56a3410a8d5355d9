// Thread-rank MPI stand-in — TEST INFRASTRUCTURE ONLY (see mpi.h).
//
// Ranks are threads; a communicator holds a generation barrier, a slot table
// for collectives and a mailbox for point-to-point messages.  Datatypes are
// either a basic element (double / int) or a 2-D C-order subarray of doubles,
// which is all the reference's CPU libraries construct.

#include "mpi.h"

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <list>
#include <mutex>
#include <stdexcept>
#include <vector>

struct shim_type {
    int elem;          // element size in bytes
    bool subarray;     // false: contiguous run of `count` elements
    int sizes[2], subsizes[2], starts[2];
};

struct shim_type shim_type_double = {8, false, {0, 0}, {0, 0}, {0, 0}};
struct shim_type shim_type_int = {4, false, {0, 0}, {0, 0}, {0, 0}};

namespace {

struct Msg {
    int src, dst, tag;
    const void* buf;
    int count;
    MPI_Datatype type;
    bool consumed;
};

}  // namespace

struct shim_req {
    bool is_send;
    bool done;
    int peer, tag;
    void* rbuf;
    int count;
    MPI_Datatype type;
    Msg* msg;  // for sends
    MPI_Comm comm;
};

struct shim_comm {
    int size;
    std::mutex mu;
    std::condition_variable cv;
    int bar_count = 0;
    long bar_gen = 0;
    // collective publication slots (one per rank)
    std::vector<const void*> c_sbuf;
    std::vector<const int*> c_scount, c_sdispl;
    std::vector<const MPI_Datatype*> c_stype;
    std::vector<int> c_int;
    std::list<Msg*> mailbox;
};

namespace {

thread_local int tl_rank = -1;

void barrier(MPI_Comm c) {
    std::unique_lock<std::mutex> lk(c->mu);
    long gen = c->bar_gen;
    if (++c->bar_count == c->size) {
        c->bar_count = 0;
        ++c->bar_gen;
        c->cv.notify_all();
    } else {
        c->cv.wait(lk, [&] { return c->bar_gen != gen; });
    }
}

// Byte offsets (relative to the buffer start) of every element described by
// (count, type), in MPI type-map order.
void type_offsets(MPI_Datatype t, int count, std::vector<size_t>& off) {
    off.clear();
    if (!t->subarray) {
        for (int k = 0; k < count; ++k) off.push_back((size_t)k * t->elem);
        return;
    }
    size_t extent = (size_t)t->sizes[0] * t->sizes[1] * t->elem;
    for (int k = 0; k < count; ++k)
        for (int i = 0; i < t->subsizes[0]; ++i)
            for (int j = 0; j < t->subsizes[1]; ++j)
                off.push_back(k * extent +
                              ((size_t)(t->starts[0] + i) * t->sizes[1] +
                               (t->starts[1] + j)) * t->elem);
}

// Copy (sbuf, scount, stype) into (rbuf, rcount, rtype) element by element.
void transfer(const void* sbuf, int scount, MPI_Datatype stype,
              void* rbuf, int rcount, MPI_Datatype rtype) {
    std::vector<size_t> so, ro;
    type_offsets(stype, scount, so);
    type_offsets(rtype, rcount, ro);
    if (stype->elem != rtype->elem || so.size() > ro.size())
        throw std::runtime_error("mpi shim: type signature mismatch");
    const char* s = static_cast<const char*>(sbuf);
    char* r = static_cast<char*>(rbuf);
    for (size_t k = 0; k < so.size(); ++k) std::memcpy(r + ro[k], s + so[k], stype->elem);
}

}  // namespace

extern "C" {

MPI_Comm shim_comm_create(int size) {
    shim_comm* c = new shim_comm();
    c->size = size;
    c->c_sbuf.assign(size, nullptr);
    c->c_scount.assign(size, nullptr);
    c->c_sdispl.assign(size, nullptr);
    c->c_stype.assign(size, nullptr);
    c->c_int.assign(size, 0);
    return c;
}

void shim_comm_destroy(MPI_Comm c) {
    for (Msg* m : c->mailbox) delete m;
    delete c;
}

void shim_bind_rank(MPI_Comm, int rank) { tl_rank = rank; }

int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype,
                  void* recvbuf, int, MPI_Datatype, MPI_Comm comm) {
    if (sendcount != 1) throw std::runtime_error("mpi shim: Allgather supports one int");
    {
        std::lock_guard<std::mutex> lk(comm->mu);
        comm->c_int[tl_rank] = *static_cast<const int*>(sendbuf);
    }
    barrier(comm);
    {
        std::lock_guard<std::mutex> lk(comm->mu);
        std::memcpy(recvbuf, comm->c_int.data(), sizeof(int) * comm->size);
    }
    barrier(comm);
    return MPI_SUCCESS;
}

int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[],
                             const int starts[], int order, MPI_Datatype oldtype,
                             MPI_Datatype* newtype) {
    if (ndims != 2 || order != MPI_ORDER_C)
        throw std::runtime_error("mpi shim: only 2-D C-order subarrays");
    shim_type* t = new shim_type();
    t->elem = oldtype->elem;
    t->subarray = true;
    for (int d = 0; d < 2; ++d) {
        t->sizes[d] = sizes[d];
        t->subsizes[d] = subsizes[d];
        t->starts[d] = starts[d];
    }
    *newtype = t;
    return MPI_SUCCESS;
}

int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }

int MPI_Type_free(MPI_Datatype* type) {
    if (*type && *type != MPI_DOUBLE && *type != MPI_INT) delete *type;
    *type = MPI_DATATYPE_NULL;
    return MPI_SUCCESS;
}

int MPI_Ialltoallw(const void* sendbuf, const int sendcounts[], const int sdispls[],
                   const MPI_Datatype sendtypes[], void* recvbuf,
                   const int recvcounts[], const int rdispls[],
                   const MPI_Datatype recvtypes[], MPI_Comm comm,
                   MPI_Request* request) {
    const int me = tl_rank;
    {
        std::lock_guard<std::mutex> lk(comm->mu);
        comm->c_sbuf[me] = sendbuf;
        comm->c_scount[me] = sendcounts;
        comm->c_sdispl[me] = sdispls;
        comm->c_stype[me] = sendtypes;
    }
    barrier(comm);
    for (int p = 0; p < comm->size; ++p) {
        const char* s = static_cast<const char*>(comm->c_sbuf[p]) + comm->c_sdispl[p][me];
        char* r = static_cast<char*>(recvbuf) + rdispls[p];
        transfer(s, comm->c_scount[p][me], comm->c_stype[p][me], r, recvcounts[p], recvtypes[p]);
    }
    barrier(comm);  // senders may reuse their buffers only after every copy
    *request = nullptr;
    return MPI_SUCCESS;
}

int MPI_Isend(const void* buf, int count, MPI_Datatype datatype, int dest,
              int tag, MPI_Comm comm, MPI_Request* request) {
    shim_req* r = new shim_req{true, dest == MPI_PROC_NULL, dest, tag, nullptr, count, datatype, nullptr, comm};
    if (!r->done) {
        Msg* m = new Msg{tl_rank, dest, tag, buf, count, datatype, false};
        r->msg = m;
        std::lock_guard<std::mutex> lk(comm->mu);
        comm->mailbox.push_back(m);
        comm->cv.notify_all();
    }
    *request = r;
    return MPI_SUCCESS;
}

int MPI_Irecv(void* buf, int count, MPI_Datatype datatype, int source,
              int tag, MPI_Comm comm, MPI_Request* request) {
    *request = new shim_req{false, source == MPI_PROC_NULL, source, tag, buf, count, datatype, nullptr, comm};
    return MPI_SUCCESS;
}

}  // extern "C"

namespace {

void complete(MPI_Comm comm, shim_req* r) {
    if (r->done) return;
    std::unique_lock<std::mutex> lk(comm->mu);
    if (r->is_send) {
        comm->cv.wait(lk, [&] { return r->msg->consumed; });
        comm->mailbox.remove(r->msg);
        delete r->msg;
        r->msg = nullptr;
    } else {
        Msg* hit = nullptr;
        comm->cv.wait(lk, [&] {
            for (Msg* m : comm->mailbox)
                if (!m->consumed && m->dst == tl_rank && m->src == r->peer && m->tag == r->tag) {
                    hit = m;
                    return true;
                }
            return false;
        });
        transfer(hit->buf, hit->count, hit->type, r->rbuf, r->count, r->type);
        hit->consumed = true;
        comm->cv.notify_all();
    }
    r->done = true;
}

}  // namespace

extern "C" {

int MPI_Wait(MPI_Request* request, MPI_Status*) {
    shim_req* r = *request;
    if (!r) return MPI_SUCCESS;
    complete(r->comm, r);
    delete r;
    *request = nullptr;
    return MPI_SUCCESS;
}

int MPI_Waitall(int count, MPI_Request requests[], MPI_Status*) {
    // Receives first: every send was posted at MPI_Isend time, so each receive
    // can complete, after which every send has been consumed.
    for (int pass = 0; pass < 2; ++pass)
        for (int k = 0; k < count; ++k) {
            shim_req* r = requests[k];
            if (r && r->is_send == (pass == 1)) MPI_Wait(&requests[k], nullptr);
        }
    return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm) {
    barrier(comm);
    return MPI_SUCCESS;
}

double MPI_Wtime(void) {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

int MPI_Allreduce(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm) {
    throw std::runtime_error("mpi shim: MPI_Allreduce is not provided");
}

int MPI_Alltoall(const void*, int, MPI_Datatype, void*, int, MPI_Datatype, MPI_Comm) {
    throw std::runtime_error("mpi shim: MPI_Alltoall is not provided");
}

int MPI_Alltoallv(const void*, const int[], const int[], MPI_Datatype, void*, const int[],
                  const int[], MPI_Datatype, MPI_Comm) {
    throw std::runtime_error("mpi shim: MPI_Alltoallv is not provided");
}

int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) {
    throw std::runtime_error("mpi shim: MPI_Bcast is not provided");
}

}  // extern "C"

