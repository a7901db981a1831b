// metis_helper.cpp -- a one-graph-at-a-time METIS_PartGraphKway server.
//
// Metis keeps global random state, so two calls running at once in one
// process change each other's results.  When many partitions run side by
// side (the batched and served modes) each concurrent coarsest-graph call
// goes to one of these helper processes instead, which gives every call its
// own address space and so the same result as a lone in-process call.
//
// Protocol on stdin/stdout, all little-endian, repeated until EOF:
//   request : int64 n, int64 m, int64 nparts, float ubvec,
//             int64 xadj[n+1], int64 adjncy[m], int64 vwgt[n], int64 adjwgt[m]
//   response: int64 status (METIS return code), int64 objval, int64 part[n]
#include <cstdint>
#include <cstdio>
#include <vector>
#include <unistd.h>

typedef int64_t metis_idx_t;
typedef float metis_real_t;
extern "C" int METIS_PartGraphKway(metis_idx_t*, metis_idx_t*, metis_idx_t*, metis_idx_t*, metis_idx_t*, metis_idx_t*,
                                   metis_idx_t*, metis_idx_t*, metis_real_t*, metis_real_t*, metis_idx_t*, metis_idx_t*,
                                   metis_idx_t*);

static bool read_all(void* p, size_t bytes) {
    char* c = (char*)p;
    while (bytes > 0) {
        ssize_t r = read(0, c, bytes);
        if (r <= 0) return false;
        c += r;
        bytes -= (size_t)r;
    }
    return true;
}

static bool write_all(const void* p, size_t bytes) {
    const char* c = (const char*)p;
    while (bytes > 0) {
        ssize_t r = write(1, c, bytes);
        if (r <= 0) return false;
        c += r;
        bytes -= (size_t)r;
    }
    return true;
}

int main() {
    while (true) {
        int64_t hdr[3];
        float ub;
        if (!read_all(hdr, sizeof(hdr)) || !read_all(&ub, sizeof(ub))) return 0;
        int64_t n = hdr[0], m = hdr[1], nparts = hdr[2];
        if (n < 0 || m < 0 || nparts < 1) return 1;
        std::vector<metis_idx_t> xadj(n + 1), adj(m), vw(n), ew(m), part(n > 0 ? n : 1, 0);
        if (!read_all(xadj.data(), sizeof(int64_t) * (n + 1)) || !read_all(adj.data(), sizeof(int64_t) * m) ||
            !read_all(vw.data(), sizeof(int64_t) * n) || !read_all(ew.data(), sizeof(int64_t) * m))
            return 1;
        metis_idx_t nn = n, ncon = 1, np = nparts, obj = 0;
        int64_t status = METIS_PartGraphKway(&nn, &ncon, xadj.data(), adj.data(), vw.data(), nullptr, ew.data(), &np,
                                             nullptr, &ub, nullptr, &obj, part.data());
        int64_t out[2] = {status, (int64_t)obj};
        if (!write_all(out, sizeof(out)) || !write_all(part.data(), sizeof(int64_t) * n)) return 1;
    }
}
