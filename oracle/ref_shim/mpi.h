/*
 * Single-rank stand-in for the MPI calls made by the reference DD-alphaAMG
 * (Schwinger model) sources.  Test infrastructure only: it lets the
 * reference's own src/*.cpp compile and run as ONE rank, so that its
 * outputs can pin the CPU restatement in oracle/ddamg_oracle.c.
 *
 * Semantics with one rank:
 *   - every point-to-point partner is the rank itself, so MPI_Sendrecv is a
 *     pack (send datatype) + unpack (recv datatype) copy; this reproduces the
 *     periodic halo wrap of the reference's exchange_halo / exchange_halo_l;
 *   - collectives (Allreduce, Gatherv, Scatterv, Bcast, Gather) copy the
 *     local contribution through the declared datatypes;
 *   - derived datatypes support MPI_Type_vector and MPI_Type_create_resized,
 *     the only constructors the reference uses.
 * It is not a general MPI implementation.
 */
#ifndef DDAMG_REF_SHIM_MPI_H
#define DDAMG_REF_SHIM_MPI_H

#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <ctime>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Group;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_SUCCESS 0
#define MPI_IDENT 0
#define MPI_UNEQUAL 3
#define MPI_SUM 1

/* predefined datatypes: ids 1..5 */
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_DOUBLE_COMPLEX 3
#define MPI_LONG_LONG_INT 4
#define MPI_CHAR 5

namespace ddamg_shim {
struct Type {
    long count = 1;      /* number of blocks */
    long blocklen = 1;   /* base elements per block */
    long stride = 1;     /* base elements between block starts */
    long base = 1;       /* bytes per base element */
    long extent = 1;     /* bytes (used for displacement arithmetic) */
};
inline std::vector<Type>& types() {
    static std::vector<Type> t = [] {
        std::vector<Type> v(6);
        const long sz[6] = {1, (long)sizeof(int), (long)sizeof(double), 2 * (long)sizeof(double),
                            (long)sizeof(long long), 1};
        for (int i = 0; i < 6; i++) { v[i].base = sz[i]; v[i].extent = sz[i]; }
        return v;
    }();
    return t;
}
inline long type_bytes(MPI_Datatype d) { const Type& t = types()[d]; return t.count * t.blocklen * t.base; }
inline void pack(const char* src, int n, MPI_Datatype d, std::vector<char>& out) {
    const Type& t = types()[d];
    for (int k = 0; k < n; k++) {
        const char* s = src + (long)k * t.extent;
        for (long b = 0; b < t.count; b++)
            out.insert(out.end(), s + b * t.stride * t.base, s + b * t.stride * t.base + t.blocklen * t.base);
    }
}
inline void unpack(const std::vector<char>& in, char* dst, int n, MPI_Datatype d) {
    const Type& t = types()[d];
    size_t p = 0;
    for (int k = 0; k < n; k++) {
        char* s = dst + (long)k * t.extent;
        for (long b = 0; b < t.count; b++) {
            std::memcpy(s + b * t.stride * t.base, in.data() + p, t.blocklen * t.base);
            p += t.blocklen * t.base;
        }
    }
}
inline int next_comm() { static int c = 2; return c++; }
}  // namespace ddamg_shim

inline int MPI_Init(int*, char***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Abort(MPI_Comm, int code) { std::fprintf(stderr, "MPI_Abort(%d)\n", code); std::exit(code ? code : 1); }
inline double MPI_Wtime() {
    timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
inline int MPI_Comm_compare(MPI_Comm a, MPI_Comm b, int* r) { *r = (a == b) ? MPI_IDENT : MPI_UNEQUAL; return 0; }
inline int MPI_Cart_create(MPI_Comm, int, const int*, const int*, int, MPI_Comm* c) { *c = ddamg_shim::next_comm(); return 0; }
inline int MPI_Cart_coords(MPI_Comm, int, int n, int* coords) { for (int i = 0; i < n; i++) coords[i] = 0; return 0; }
inline int MPI_Cart_shift(MPI_Comm, int, int, int* a, int* b) { *a = 0; *b = 0; return 0; }
inline int MPI_Cart_rank(MPI_Comm, const int*, int* r) { *r = 0; return 0; }
inline int MPI_Comm_group(MPI_Comm, MPI_Group* g) { *g = 1; return 0; }
inline int MPI_Group_incl(MPI_Group, int, const int*, MPI_Group* g) { *g = 1; return 0; }
inline int MPI_Comm_create(MPI_Comm, MPI_Group, MPI_Comm* c) { *c = ddamg_shim::next_comm(); return 0; }
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }

inline int MPI_Type_vector(int count, int blocklen, int stride, MPI_Datatype old, MPI_Datatype* out) {
    auto& T = ddamg_shim::types();
    const ddamg_shim::Type& o = T[old];
    if (o.count != 1 || o.blocklen != 1) { std::fprintf(stderr, "shim: nested vector types unsupported\n"); std::exit(2); }
    ddamg_shim::Type t;
    t.count = count; t.blocklen = blocklen; t.stride = stride; t.base = o.base;
    t.extent = ((long)(count - 1) * stride + blocklen) * o.base;
    T.push_back(t);
    *out = (MPI_Datatype)(T.size() - 1);
    return 0;
}
inline int MPI_Type_create_resized(MPI_Datatype old, long, long extent, MPI_Datatype* out) {
    auto& T = ddamg_shim::types();
    ddamg_shim::Type t = T[old];
    t.extent = extent;
    T.push_back(t);
    *out = (MPI_Datatype)(T.size() - 1);
    return 0;
}
inline int MPI_Type_commit(MPI_Datatype*) { return 0; }

inline int MPI_Sendrecv(const void* sb, int sc, MPI_Datatype st, int, int, void* rb, int rc, MPI_Datatype rt, int, int,
                        MPI_Comm, MPI_Status*) {
    std::vector<char> buf;
    ddamg_shim::pack((const char*)sb, sc, st, buf);
    if ((long)buf.size() != ddamg_shim::type_bytes(rt) * rc) { std::fprintf(stderr, "shim: Sendrecv size mismatch\n"); std::exit(2); }
    ddamg_shim::unpack(buf, (char*)rb, rc, rt);
    return 0;
}
inline int MPI_Allreduce(const void* sb, void* rb, int n, MPI_Datatype d, MPI_Op, MPI_Comm) {
    std::memmove(rb, sb, ddamg_shim::type_bytes(d) * n);
    return 0;
}
inline int MPI_Gather(const void* sb, int sc, MPI_Datatype st, void* rb, int, MPI_Datatype, int, MPI_Comm) {
    std::memmove(rb, sb, ddamg_shim::type_bytes(st) * sc);
    return 0;
}
inline int MPI_Gatherv(const void* sb, int sc, MPI_Datatype st, void* rb, const int* counts, const int* displs,
                       MPI_Datatype rt, int, MPI_Comm) {
    std::vector<char> buf;
    ddamg_shim::pack((const char*)sb, sc, st, buf);
    ddamg_shim::unpack(buf, (char*)rb + (long)displs[0] * ddamg_shim::types()[rt].extent, counts[0], rt);
    return 0;
}
inline int MPI_Scatterv(const void* sb, const int* counts, const int* displs, MPI_Datatype st, void* rb, int rc,
                        MPI_Datatype rt, int, MPI_Comm) {
    std::vector<char> buf;
    ddamg_shim::pack((const char*)sb + (long)displs[0] * ddamg_shim::types()[st].extent, counts[0], st, buf);
    ddamg_shim::unpack(buf, (char*)rb, rc, rt);
    return 0;
}

#endif
