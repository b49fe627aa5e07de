// Single-rank implementation of the MPI subset declared in mpi.h.
// Test infrastructure for the CPU oracle build; see mpi.h for semantics.
#include "mpi.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

// A datatype is a list of (byte offset, byte length) runs plus an extent.
struct TypeDesc {
    std::vector<std::pair<long, long>> runs;
    long extent = 0;
};

std::vector<TypeDesc> &types() {
    static std::vector<TypeDesc> t;
    if (t.empty()) {
        t.resize(4);
        t[MPI_DOUBLE].runs = {{0, 8}};
        t[MPI_DOUBLE].extent = 8;
        t[MPI_INT].runs = {{0, 4}};
        t[MPI_INT].extent = 4;
        t[MPI_BYTE].runs = {{0, 1}};
        t[MPI_BYTE].extent = 1;
    }
    return t;
}

const TypeDesc &desc(MPI_Datatype t) {
    if (t < 0 || t >= (int)types().size()) {
        std::fprintf(stderr, "mpi shim: bad datatype %d\n", t);
        std::abort();
    }
    return types()[t];
}

int add_type(TypeDesc d) {
    // merge adjacent runs so packing is a handful of memcpy calls
    TypeDesc m;
    m.extent = d.extent;
    for (auto &r : d.runs) {
        if (!m.runs.empty() && m.runs.back().first + m.runs.back().second == r.first)
            m.runs.back().second += r.second;
        else
            m.runs.push_back(r);
    }
    types().push_back(m);
    return (int)types().size() - 1;
}

void pack(const void *buf, int count, MPI_Datatype t, std::vector<char> &out) {
    const TypeDesc &d = desc(t);
    const char *b = static_cast<const char *>(buf);
    for (int c = 0; c < count; ++c)
        for (auto &r : d.runs)
            out.insert(out.end(), b + c * d.extent + r.first, b + c * d.extent + r.first + r.second);
}

void unpack(const std::vector<char> &in, void *buf, int count, MPI_Datatype t) {
    const TypeDesc &d = desc(t);
    char *b = static_cast<char *>(buf);
    size_t pos = 0;
    for (int c = 0; c < count && pos < in.size(); ++c)
        for (auto &r : d.runs) {
            if (pos >= in.size()) break;
            size_t n = (size_t)r.second;
            if (pos + n > in.size()) n = in.size() - pos;
            std::memcpy(b + c * d.extent + r.first, in.data() + pos, n);
            pos += n;
        }
}

struct PendingSend { int tag; std::vector<char> data; };
struct PendingRecv { int tag; void *buf; int count; MPI_Datatype type; };

std::vector<PendingSend> g_sends;
std::vector<PendingRecv> g_recvs;
int g_periods[3] = {0, 0, 0};

}  // namespace

extern "C" {

int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code) { std::exit(code); }
int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }

int MPI_Cart_create(MPI_Comm, int ndims, const int *, const int *periods, int, MPI_Comm *cart) {
    for (int d = 0; d < ndims && d < 3; ++d) g_periods[d] = periods[d];
    *cart = 1;
    return MPI_SUCCESS;
}

int MPI_Cart_coords(MPI_Comm, int, int maxdims, int *coords) {
    for (int d = 0; d < maxdims; ++d) coords[d] = 0;
    return MPI_SUCCESS;
}

int MPI_Cart_shift(MPI_Comm, int direction, int, int *src, int *dst) {
    int nb = g_periods[direction] ? 0 : MPI_PROC_NULL;
    *src = nb;
    *dst = nb;
    return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }

int MPI_Allgather(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf, int, MPI_Datatype, MPI_Comm) {
    std::vector<char> tmp;
    pack(sbuf, scount, stype, tmp);
    std::memcpy(rbuf, tmp.data(), tmp.size());
    return MPI_SUCCESS;
}

int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *out) {
    const TypeDesc &o = desc(old);
    TypeDesc d;
    for (int c = 0; c < count; ++c)
        for (auto &r : o.runs) d.runs.push_back({c * o.extent + r.first, r.second});
    d.extent = count * o.extent;
    *out = add_type(d);
    return MPI_SUCCESS;
}

int MPI_Type_vector(int count, int blocklen, int stride, MPI_Datatype old, MPI_Datatype *out) {
    const TypeDesc &o = desc(old);
    TypeDesc d;
    for (int c = 0; c < count; ++c)
        for (int b = 0; b < blocklen; ++b)
            for (auto &r : o.runs)
                d.runs.push_back({((long)c * stride + b) * o.extent + r.first, r.second});
    d.extent = ((long)(count - 1) * stride + blocklen) * o.extent;
    *out = add_type(d);
    return MPI_SUCCESS;
}

int MPI_Type_create_resized(MPI_Datatype old, long, long extent, MPI_Datatype *out) {
    TypeDesc d = desc(old);
    d.extent = extent;
    *out = add_type(d);
    return MPI_SUCCESS;
}

int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype *) { return MPI_SUCCESS; }

int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm, MPI_Request *req) {
    if (req) *req = 0;
    if (dest == MPI_PROC_NULL) return MPI_SUCCESS;
    std::vector<char> data;
    pack(buf, count, type, data);
    for (size_t i = 0; i < g_recvs.size(); ++i) {
        if (g_recvs[i].tag == tag) {
            unpack(data, g_recvs[i].buf, g_recvs[i].count, g_recvs[i].type);
            g_recvs.erase(g_recvs.begin() + (long)i);
            return MPI_SUCCESS;
        }
    }
    g_sends.push_back({tag, std::move(data)});
    return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm, MPI_Request *req) {
    if (req) *req = 0;
    if (source == MPI_PROC_NULL) return MPI_SUCCESS;
    for (size_t i = 0; i < g_sends.size(); ++i) {
        if (g_sends[i].tag == tag) {
            unpack(g_sends[i].data, buf, count, type);
            g_sends.erase(g_sends.begin() + (long)i);
            return MPI_SUCCESS;
        }
    }
    g_recvs.push_back({tag, buf, count, type});
    return MPI_SUCCESS;
}

int MPI_Waitall(int, MPI_Request *, MPI_Status *) {
    if (!g_recvs.empty() || !g_sends.empty()) {
        std::fprintf(stderr, "mpi shim: %zu receives and %zu sends unmatched at Waitall\n",
                     g_recvs.size(), g_sends.size());
        std::abort();
    }
    return MPI_SUCCESS;
}

}  // extern "C"
