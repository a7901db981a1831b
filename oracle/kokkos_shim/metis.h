// metis.h -- TEST INFRASTRUCTURE ONLY.
//
// The reference calls METIS_PartGraphKway with `int` arrays and a `real_t`
// imbalance (reference src/initial_partition.hpp:65, :103-105).  The only
// Metis here is CUDA's bundled libmetis_static.a, built with 64-bit idx_t and
// 32-bit float real_t.  This header declares that library's C entry point and
// adds a C++ overload taking `int` arrays that widens them, calls the library
// and narrows the results back.
#pragma once
#include <cstdint>
#include <vector>

typedef int64_t idx_t;
typedef float real_t;

enum rstatus_et { METIS_OK = 1, METIS_ERROR_INPUT = -2, METIS_ERROR_MEMORY = -3, METIS_ERROR = -4 };

extern "C" int METIS_PartGraphKway(idx_t* nvtxs, idx_t* ncon, idx_t* xadj, idx_t* adjncy, idx_t* vwgt, idx_t* vsize,
                                   idx_t* adjwgt, idx_t* nparts, real_t* tpwgts, real_t* ubvec, idx_t* options,
                                   idx_t* edgecut, idx_t* part);

inline int METIS_PartGraphKway(int* nvtxs, int* ncon, int* xadj, int* adjncy, int* vwgt, int* vsize, int* adjwgt,
                               int* nparts, real_t* tpwgts, real_t* ubvec, int* options, int* edgecut, int* part) {
    const int64_t n = *nvtxs;
    const int64_t nc = *ncon;
    const int64_t m = xadj[n];
    std::vector<idx_t> x(xadj, xadj + n + 1), a(adjncy, adjncy + m);
    std::vector<idx_t> vw, vs, aw, p(n > 0 ? n : 1);
    if (vwgt) vw.assign(vwgt, vwgt + n * nc);
    if (vsize) vs.assign(vsize, vsize + n);
    if (adjwgt) aw.assign(adjwgt, adjwgt + m);
    idx_t nv = n, ncn = nc, np = *nparts, ec = 0;
    int rc = METIS_PartGraphKway(&nv, &ncn, x.data(), a.data(), vwgt ? vw.data() : nullptr, vsize ? vs.data() : nullptr,
                                 adjwgt ? aw.data() : nullptr, &np, tpwgts, ubvec, nullptr, &ec, p.data());
    (void)options;
    *edgecut = (int)ec;
    for (int64_t i = 0; i < n; i++) part[i] = (int)p[i];
    return rc;
}
