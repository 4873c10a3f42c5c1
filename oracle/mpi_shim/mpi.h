/*
 * Single-rank stand-in for the MPI surface that parallel-RA's sources call.
 *
 * TEST INFRASTRUCTURE ONLY: this header exists so that the reference's own
 * C++ sources (src/comm, src/IO, src/RAM, src/lie, ...) compile unchanged into
 * oracle/_ref when no MPI installation is present.  It implements every MPI
 * call those sources make for a communicator of exactly one rank:
 *   - collectives (Allreduce, Reduce, Bcast, Allgather, Alltoall, Alltoallv)
 *     degenerate to copies from the send buffer to the receive buffer;
 *   - point-to-point Isend/Irecv/Waitall are self-messages: Isend copies the
 *     payload into a FIFO, Irecv takes the oldest message of the same tag
 *     (immediately, or at Waitall when posted before the matching send);
 *   - MPI-IO maps to POSIX pread/pwrite on one file descriptor.
 * Nothing here is shipped with, linked into, or called by the product library.
 */
#pragma once

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <deque>
#include <vector>
#include <chrono>
#include <fcntl.h>
#include <unistd.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_File;
typedef long MPI_Offset;
typedef int MPI_Request;
struct MPI_Status { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; };

#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_SUCCESS 0

/* datatype handles encode their byte size */
#define MPI_INT ((MPI_Datatype)4)
#define MPI_UNSIGNED_LONG_LONG ((MPI_Datatype)8)
#define MPI_LONG_LONG ((MPI_Datatype)(8 | 0x100))
#define MPI_DOUBLE ((MPI_Datatype)(8 | 0x200))
#define MPI_BYTE ((MPI_Datatype)1)

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_BAND 4

#define MPI_MODE_RDONLY 1
#define MPI_MODE_WRONLY 2
#define MPI_MODE_CREATE 4

namespace mpi_shim {
inline size_t type_size(MPI_Datatype t) { return (size_t)(t & 0xff); }

struct message { int tag; std::vector<unsigned char> bytes; };
struct pending_recv { void* buf; size_t bytes; int tag; bool done; };

inline std::deque<message>& mailbox() { static std::deque<message> q; return q; }
inline std::vector<pending_recv>& pending() { static std::vector<pending_recv> p; return p; }

inline bool take(int tag, void* buf, size_t cap) {
    auto& q = mailbox();
    for (auto it = q.begin(); it != q.end(); ++it) {
        if (it->tag == tag) {
            size_t n = it->bytes.size() < cap ? it->bytes.size() : cap;
            if (n) std::memcpy(buf, it->bytes.data(), n);
            q.erase(it);
            return true;
        }
    }
    return false;
}
}  // namespace mpi_shim

inline int MPI_Init(int*, char***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_size(MPI_Comm, int* n) { *n = 1; return 0; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Abort(MPI_Comm, int code) { std::fflush(stdout); std::exit(code == 0 ? 1 : code & 0xff); }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline double MPI_Wtime() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    if (s != r) std::memmove(r, s, (size_t)n * mpi_shim::type_size(t));
    return 0;
}
inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    if (s != r) std::memmove(r, s, (size_t)n * mpi_shim::type_size(t));
    return 0;
}
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Allgather(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) {
    if (s != r) std::memmove(r, s, (size_t)sn * mpi_shim::type_size(st));
    return 0;
}
inline int MPI_Alltoall(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) {
    if (s != r) std::memmove(r, s, (size_t)sn * mpi_shim::type_size(st));
    return 0;
}
inline int MPI_Alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st,
                         void* r, const int*, const int* rd, MPI_Datatype, MPI_Comm) {
    size_t e = mpi_shim::type_size(st);
    if (sc[0]) std::memmove((char*)r + (size_t)rd[0] * e, (const char*)s + (size_t)sd[0] * e, (size_t)sc[0] * e);
    return 0;
}

inline int MPI_Isend(const void* buf, int n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* req) {
    mpi_shim::message m;
    m.tag = tag;
    m.bytes.resize((size_t)n * mpi_shim::type_size(t));
    if (!m.bytes.empty()) std::memcpy(m.bytes.data(), buf, m.bytes.size());
    mpi_shim::mailbox().push_back(std::move(m));
    *req = -1;
    return 0;
}
inline int MPI_Irecv(void* buf, int n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* req) {
    size_t cap = (size_t)n * mpi_shim::type_size(t);
    if (mpi_shim::take(tag, buf, cap)) { *req = -1; return 0; }
    mpi_shim::pending().push_back({buf, cap, tag, false});
    *req = (int)mpi_shim::pending().size() - 1;
    return 0;
}
inline int MPI_Waitall(int n, MPI_Request* reqs, MPI_Status*) {
    for (int i = 0; i < n; i++) {
        if (reqs[i] < 0) continue;
        auto& p = mpi_shim::pending()[(size_t)reqs[i]];
        if (!p.done && !mpi_shim::take(p.tag, p.buf, p.bytes)) {
            std::fprintf(stderr, "mpi shim: receive with tag %d has no matching send\n", p.tag);
            std::abort();
        }
        p.done = true;
    }
    bool all_done = true;
    for (auto& p : mpi_shim::pending()) all_done = all_done && p.done;
    if (all_done) mpi_shim::pending().clear();
    return 0;
}

inline int MPI_Info_create(MPI_Info* i) { *i = 0; return 0; }
inline int MPI_Info_set(MPI_Info, const char*, const char*) { return 0; }
inline int MPI_Info_free(MPI_Info*) { return 0; }

inline int MPI_File_open(MPI_Comm, const char* name, int mode, MPI_Info, MPI_File* f) {
    int flags = (mode & MPI_MODE_RDONLY) ? O_RDONLY : O_WRONLY;
    if (mode & MPI_MODE_CREATE) flags |= O_CREAT;
    *f = open(name, flags, 0644);
    return *f < 0 ? 1 : 0;
}
inline int MPI_File_read_at_all(MPI_File f, MPI_Offset off, void* buf, int n, MPI_Datatype t, MPI_Status*) {
    ssize_t want = (ssize_t)n * (ssize_t)mpi_shim::type_size(t);
    return pread(f, buf, (size_t)want, off) == want ? 0 : 1;
}
inline int MPI_File_write_at_all(MPI_File f, MPI_Offset off, const void* buf, int n, MPI_Datatype t, MPI_Status*) {
    ssize_t want = (ssize_t)n * (ssize_t)mpi_shim::type_size(t);
    return pwrite(f, buf, (size_t)want, off) == want ? 0 : 1;
}
inline int MPI_File_close(MPI_File* f) { close(*f); *f = -1; return 0; }
