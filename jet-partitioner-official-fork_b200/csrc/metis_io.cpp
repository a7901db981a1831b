// metis_io.cpp -- METIS text graph reader (host code, multi-threaded).
//
// Reads the file format the reference's load_metis_graph accepts
// (app/io.hpp:99-217) with the same rules, in parallel over the host cores:
//   * leading lines starting with '%' are comments; the header line holds
//     n, m and optionally fmt and ncon; fmt must be 0 (no weights) or 1 (edge
//     weights) and ncon 0 (vertex weights are not supported, as in the
//     reference);
//   * in the body, any '%' starts a comment that runs through the end of its
//     line, and that line's newline then ends no row (the reference's
//     next_line skips it);
//   * every other newline ends a row while fewer than n rows have ended;
//     characters other than digits, '%' and newlines separate numbers;
//   * numbers are neighbour ids (1-based) or, with fmt 1, alternately id and
//     edge weight, the alternation running across lines;
//   * a missing final newline is supplied.
// The file must then hold exactly n rows and 2m nonzeros (else
// JET_ERR_INVALID).  One rule is stricter than the reference: numbers after
// the n-th row are an error here (the reference would write them past its
// row map).
//
// Parsing runs in two passes over chunks that start at line boundaries:
// pass 1 counts numbers and row ends per chunk, a prefix over the chunks
// gives each its first edge and row, pass 2 writes the arrays.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/jet_b200.h"

namespace jetb {
void set_last_error(const std::string& msg);
}

namespace {

struct Chunk {
    size_t begin = 0, end = 0;
    int64_t numbers = 0;  // numbers before the n-th row end (counted for the cap below)
    int64_t rows = 0;     // row-ending newlines
    int64_t tail_numbers = 0;  // numbers after this chunk's row ends once the global cap is reached (pass 2)
};

// Pass 1: numbers and row-ending newlines in [b, e).
void count_chunk(const char* s, Chunk& c) {
    const char* f = s + c.begin;
    const char* e = s + c.end;
    int64_t nums = 0, rows = 0;
    while (f < e) {
        char ch = *f;
        if (ch >= '0' && ch <= '9') {
            while (f < e && *f >= '0' && *f <= '9') f++;
            nums++;
        } else if (ch == '%') {
            while (f < e && *f != '\n') f++;
            f++;  // the comment's newline ends no row
        } else {
            if (ch == '\n') rows++;
            f++;
        }
    }
    c.numbers = nums;
    c.rows = rows;
}

template <class O, class E, class W>
struct Out {
    E* row;
    O* adj;
    W* val;
};

// Pass 2: writes ids, weights and row offsets of one chunk.
//   tok0     numbers before this chunk
//   row0     row ends before this chunk (global, uncapped)
//   n        rows the header promises; row ends beyond it are ignored
// Returns false when a number appears after the n-th row end.
template <class O, class E, class W>
bool parse_chunk(const char* s, const Chunk& c, int64_t tok0, int64_t row0, int64_t n, bool has_ew, Out<O, E, W> out) {
    const char* f = s + c.begin;
    const char* e = s + c.end;
    int64_t tok = tok0, rows = row0;
    while (f < e) {
        char ch = *f;
        if (ch >= '0' && ch <= '9') {
            int64_t v = 0;
            while (f < e && *f >= '0' && *f <= '9') v = v * 10 + (*f++ - '0');
            if (rows >= n) return false;
            if (has_ew) {
                if ((tok & 1) == 0) out.adj[tok >> 1] = (O)(v - 1);
                else out.val[tok >> 1] = (W)v;
            } else {
                out.adj[tok] = (O)(v - 1);
            }
            tok++;
        } else if (ch == '%') {
            while (f < e && *f != '\n') f++;
            f++;
        } else {
            if (ch == '\n') {
                rows++;
                if (rows <= n) out.row[rows] = (E)(has_ew ? (tok >> 1) : tok);
            }
            f++;
        }
    }
    return true;
}

template <class O, class E, class W>
int read_body(const char* s, size_t body, size_t sz, int64_t n, int64_t m, bool has_ew, int threads, int64_t* n_out,
              int64_t* nnz_out, void** row_out, void** adj_out, void** val_out) {
    // chunk boundaries at line starts
    int nt = std::max(1, threads);
    size_t len = sz - body;
    if (len < ((size_t)1 << 20)) nt = 1;
    std::vector<Chunk> ch(nt);
    size_t pos = body;
    for (int t = 0; t < nt; t++) {
        ch[t].begin = pos;
        size_t cut = (t == nt - 1) ? sz : std::max(pos, body + len * (t + 1) / nt);
        while (cut < sz && s[cut - 1] != '\n') cut++;
        ch[t].end = cut;
        pos = cut;
    }
    auto run = [&](auto fn) {
        std::vector<std::thread> th;
        for (int t = 1; t < nt; t++) th.emplace_back(fn, t);
        fn(0);
        for (auto& x : th) x.join();
    };
    run([&](int t) { count_chunk(s, ch[t]); });
    std::vector<int64_t> tok0(nt + 1, 0), row0(nt + 1, 0);
    for (int t = 0; t < nt; t++) {
        tok0[t + 1] = tok0[t] + ch[t].numbers;
        row0[t + 1] = row0[t] + ch[t].rows;
    }
    int64_t tokens = tok0[nt];
    int64_t nnz = has_ew ? tokens / 2 : tokens;
    if (row0[nt] < n || nnz != 2 * m || (has_ew && (tokens & 1))) {
        jetb::set_last_error("METIS file: read " + std::to_string(std::min<int64_t>(row0[nt], n)) + " lines and " +
                             std::to_string(nnz) + " nonzeros; header promises " + std::to_string(n) + " and " +
                             std::to_string(2 * m));
        return JET_ERR_INVALID;
    }
    E* row = (E*)std::malloc(sizeof(E) * (size_t)(n + 1));
    O* adj = (O*)std::malloc(sizeof(O) * (size_t)std::max<int64_t>(nnz, 1));
    W* val = (W*)std::malloc(sizeof(W) * (size_t)std::max<int64_t>(nnz, 1));
    if (!row || !adj || !val) {
        std::free(row); std::free(adj); std::free(val);
        jetb::set_last_error("METIS file: host allocation failed");
        return JET_ERR_OOM;
    }
    row[0] = 0;
    Out<O, E, W> out{row, adj, val};
    std::vector<char> ok(nt, 1);
    run([&](int t) { ok[t] = parse_chunk<O, E, W>(s, ch[t], tok0[t], row0[t], n, has_ew, out); });
    if (std::find(ok.begin(), ok.end(), 0) != ok.end()) {
        std::free(row); std::free(adj); std::free(val);
        jetb::set_last_error("METIS file: numbers after the last of the header's rows");
        return JET_ERR_INVALID;
    }
    if (!has_ew) std::fill(val, val + nnz, (W)1);
    *n_out = n;
    *nnz_out = nnz;
    *row_out = row;
    *adj_out = adj;
    *val_out = val;
    return JET_OK;
}

}  // namespace

extern "C" int jet_read_metis(const char* path, int tier, int threads, int64_t* n_out, int64_t* nnz_out, void** row_map,
                              void** entries, void** values, int* uniform_ew) {
    if (!path || !n_out || !nnz_out || !row_map || !entries || !values || !uniform_ew || tier < 0 || tier > 2) {
        jetb::set_last_error("jet_read_metis: bad argument");
        return JET_ERR_INVALID;
    }
    FILE* fp = std::fopen(path, "rb");
    if (!fp) {
        jetb::set_last_error(std::string("jet_read_metis: could not open ") + path);
        return JET_ERR_INVALID;
    }
    std::fseek(fp, 0, SEEK_END);
    long fsz = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    if (fsz <= 0) {
        std::fclose(fp);
        jetb::set_last_error("jet_read_metis: empty file");
        return JET_ERR_INVALID;
    }
    std::vector<char> buf((size_t)fsz + 1);
    size_t got = std::fread(buf.data(), 1, (size_t)fsz, fp);
    std::fclose(fp);
    if (got != (size_t)fsz) {
        jetb::set_last_error("jet_read_metis: short read");
        return JET_ERR_INVALID;
    }
    size_t sz = (size_t)fsz;
    if (buf[sz - 1] != '\n') buf[sz++] = '\n';
    const char* s = buf.data();
    // header: skip comment lines, then up to four numbers on one line
    size_t p = 0;
    while (p < sz && s[p] == '%') {
        while (p < sz && s[p] != '\n') p++;
        p++;
    }
    int64_t head[4] = {0, 0, 0, 0};
    int nh = 0;
    while (p < sz && s[p] != '\n') {
        if (s[p] >= '0' && s[p] <= '9') {
            int64_t v = 0;
            while (p < sz && s[p] >= '0' && s[p] <= '9') v = v * 10 + (s[p++] - '0');
            if (nh < 4) head[nh] = v;
            nh++;
        } else {
            p++;
        }
    }
    p++;  // past the header's newline
    if (nh < 2) {
        jetb::set_last_error("jet_read_metis: header needs n and m");
        return JET_ERR_INVALID;
    }
    int64_t n = head[0], m = head[1], fmt = head[2], ncon = head[3];
    if ((fmt != 0 && fmt != 1) || ncon != 0) {
        jetb::set_last_error("jet_read_metis: unsupported format flags " + std::to_string(fmt) + " / ncon " +
                             std::to_string(ncon) + " (vertex weights are not supported)");
        return JET_ERR_INVALID;
    }
    if (tier == 0 && (n > INT32_MAX || 2 * m > INT32_MAX)) {
        jetb::set_last_error("jet_read_metis: graph too large for 32-bit offsets");
        return JET_ERR_INVALID;
    }
    if (tier < 2 && n > INT32_MAX) {
        jetb::set_last_error("jet_read_metis: too many vertices for 32-bit ids");
        return JET_ERR_INVALID;
    }
    bool has_ew = fmt == 1;
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    *uniform_ew = has_ew ? 0 : 1;
    switch (tier) {
        case 0: return read_body<int32_t, int32_t, int32_t>(s, p, sz, n, m, has_ew, threads, n_out, nnz_out, row_map, entries, values);
        case 1: return read_body<int32_t, int64_t, int64_t>(s, p, sz, n, m, has_ew, threads, n_out, nnz_out, row_map, entries, values);
        default: return read_body<int64_t, int64_t, int64_t>(s, p, sz, n, m, has_ew, threads, n_out, nnz_out, row_map, entries, values);
    }
}

extern "C" void jet_free_host(void* p) { std::free(p); }
