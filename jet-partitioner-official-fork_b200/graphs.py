"""Graph containers, METIS-format I/O and seeded synthetic generators.

The generators build the workloads the partitioner is measured on:

* ``grid2d``  -- 4-neighbour 2D grid (256x256: 65,536 vertices, 130,560 edges)
* ``grid3d``  -- 7-point 3D grid (128^3: 2,097,152 vertices, 6,242,304 edges)
* ``rmat``    -- R-MAT power-law graph, symmetrised, de-duplicated, no loops
* ``rgg``     -- 2D random geometric graph in the unit square

All generators are seeded and run either on the CPU or on a CUDA device
(torch); the same seed gives different graphs on different devices because
the two random number generators differ.  Graphs are returned as ``CSRGraph``
with both edge directions stored (the layout the partitioner expects: a
symmetric CSR without self-loops), in one of three integer tiers mirroring the
reference's ``jet_defs.h``: ``"i32"`` (int32 everywhere), ``"big"`` (int32
ordinals, int64 offsets and weights) and ``"biggest"`` (all int64).

The METIS text reader/writer follows app/io.hpp:99-231 of the reference (format
flags 0 and 1 only; vertex weights are not read).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

TIERS = {
    "i32": (torch.int32, torch.int32, torch.int32),
    "big": (torch.int32, torch.int64, torch.int64),
    "biggest": (torch.int64, torch.int64, torch.int64),
}
TIER_ID = {"i32": 0, "big": 1, "biggest": 2}


@dataclass
class CSRGraph:
    """Symmetric CSR graph: ``row`` (n+1 offsets), ``adj`` (neighbour ids),
    ``val`` (edge weights), ``vw`` (vertex weights); ``uniform`` is True when
    every edge weight is 1 (the reference's ``uniform_ew``)."""

    n: int
    row: torch.Tensor
    adj: torch.Tensor
    val: torch.Tensor
    vw: torch.Tensor
    uniform: bool
    tier: str = "i32"

    @property
    def nnz(self) -> int:
        return int(self.adj.numel())

    @property
    def device(self):
        return self.row.device

    def to(self, device) -> "CSRGraph":
        return CSRGraph(self.n, self.row.to(device), self.adj.to(device), self.val.to(device),
                        self.vw.to(device), self.uniform, self.tier)

    def as_tier(self, tier: str) -> "CSRGraph":
        o, e, w = TIERS[tier]
        return CSRGraph(self.n, self.row.to(e), self.adj.to(o), self.val.to(w), self.vw.to(w),
                        self.uniform, tier)

    def numpy(self):
        """(row, adj, val, vw) as contiguous numpy arrays."""
        g = self.to("cpu")
        return (np.ascontiguousarray(g.row.numpy()), np.ascontiguousarray(g.adj.numpy()),
                np.ascontiguousarray(g.val.numpy()), np.ascontiguousarray(g.vw.numpy()))


def from_undirected(n: int, u: torch.Tensor, v: torch.Tensor, w: Optional[torch.Tensor] = None,
                    tier: str = "i32", vw: Optional[torch.Tensor] = None) -> CSRGraph:
    """Builds a symmetric CSR from undirected edges (u, v) (u != v, no
    duplicates).  Rows are sorted by neighbour id."""
    dev = u.device
    o, e, wt = TIERS[tier]
    u = u.to(torch.int64)
    v = v.to(torch.int64)
    uniform = w is None
    if w is None:
        w = torch.ones(u.numel(), dtype=torch.int64, device=dev)
    src = torch.cat([u, v])
    dst = torch.cat([v, u])
    ww = torch.cat([w.to(torch.int64), w.to(torch.int64)])
    key = src * n + dst
    order = torch.argsort(key)
    src = src[order]
    dst = dst[order]
    ww = ww[order]
    deg = torch.bincount(src, minlength=n)
    row = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    row[1:] = torch.cumsum(deg, 0)
    if vw is None:
        vw = torch.ones(n, dtype=torch.int64, device=dev)
    return CSRGraph(n, row.to(e), dst.to(o), ww.to(wt), vw.to(wt), uniform, tier)


def _gen(seed: int, device) -> torch.Generator:
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    return g


def _randint_cpu(lo: int, hi: int, count: int, seed: int, device) -> torch.Tensor:
    """Integers uniform in [lo, hi) drawn on the host from ``seed``, so that a
    graph is the same whichever device it is built on."""
    return torch.randint(lo, hi, (count,), generator=_gen(seed, "cpu")).to(device)


def grid2d(nx: int, ny: int, weighted: bool = False, seed: int = 1, tier: str = "i32", device="cpu") -> CSRGraph:
    idx = torch.arange(nx * ny, device=device).reshape(ny, nx)
    us = [idx[:, :-1].reshape(-1), idx[:-1, :].reshape(-1)]
    vs = [idx[:, 1:].reshape(-1), idx[1:, :].reshape(-1)]
    u = torch.cat(us)
    v = torch.cat(vs)
    w = None
    if weighted:
        w = _randint_cpu(1, 11, u.numel(), seed, device)
    return from_undirected(nx * ny, u, v, w, tier)


def grid3d(nx: int, ny: int, nz: int, weighted: bool = True, seed: int = 1, tier: str = "i32", device="cpu") -> CSRGraph:
    """7-point 3D grid; with ``weighted`` each undirected edge gets a weight
    uniform in [1, 10] drawn from ``seed`` (on the host: the same graph on
    every device)."""
    idx = torch.arange(nx * ny * nz, device=device).reshape(nz, ny, nx)
    u = torch.cat([idx[:, :, :-1].reshape(-1), idx[:, :-1, :].reshape(-1), idx[:-1, :, :].reshape(-1)])
    v = torch.cat([idx[:, :, 1:].reshape(-1), idx[:, 1:, :].reshape(-1), idx[1:, :, :].reshape(-1)])
    w = None
    if weighted:
        w = _randint_cpu(1, 11, u.numel(), seed, device)
    return from_undirected(nx * ny * nz, u, v, w, tier)


_M63 = 1 << 63


def _s64(c: int) -> int:
    """A 64-bit constant as the int64 with the same bits."""
    return c - (1 << 64) if c >= _M63 else c


_SM0, _SM1, _SM2 = _s64(0x9E3779B97F4A7C15), _s64(0xBF58476D1CE4E5B9), _s64(0x94D049BB133111EB)


def _srl(x: torch.Tensor, s: int) -> torch.Tensor:
    """Logical right shift of int64 bit patterns."""
    return (x >> s) & ((1 << (64 - s)) - 1)


def _mix64(x: torch.Tensor) -> torch.Tensor:
    """splitmix64 (S. Vigna) on int64 bit patterns: wrapping integer
    arithmetic, identical on every device."""
    x = x + _SM0
    x = (x ^ _srl(x, 30)) * _SM1
    x = (x ^ _srl(x, 27)) * _SM2
    return x ^ _srl(x, 31)


def _uniform(seed: int, idx: torch.Tensor) -> torch.Tensor:
    """Doubles in [0, 1) from the counter idx under seed (53 random bits)."""
    key = _mix64(torch.full_like(idx, _s64(seed & ((1 << 64) - 1)))) ^ idx
    return _srl(_mix64(key), 11).to(torch.float64) * (1.0 / (1 << 53))


def rmat(scale: int, edge_factor: int = 8, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 1, tier: str = "big", device="cpu", chunk: int = 1 << 25) -> CSRGraph:
    """R-MAT with 2^scale vertices and edge_factor * 2^scale sampled edges,
    symmetrised, de-duplicated, self-loops removed, unit weights.  Every
    random number is a counter-based hash of (seed, edge, bit), so the graph
    is the same on every device."""
    n = 1 << scale
    m = edge_factor * n
    probs = torch.tensor([a, b, c, 1.0 - a - b - c], device=device, dtype=torch.float64)
    cum = torch.cumsum(probs, 0)
    keys = []
    done = 0
    while done < m:
        cnt = min(chunk, m - done)
        eidx = (torch.arange(cnt, dtype=torch.int64, device=device) + done) * 64
        u = torch.zeros(cnt, dtype=torch.int64, device=device)
        v = torch.zeros(cnt, dtype=torch.int64, device=device)
        for bit in range(scale):
            r = _uniform(seed, eidx + bit)
            q = torch.searchsorted(cum, r, right=True).clamp_(max=3)
            u |= (q >> 1) << bit
            v |= (q & 1) << bit
        lo = torch.minimum(u, v)
        hi = torch.maximum(u, v)
        keep = lo != hi
        keys.append(lo[keep] * n + hi[keep])
        done += cnt
    key = torch.unique(torch.cat(keys))
    return from_undirected(n, key // n, key % n, None, tier)


def rgg(n: int, mean_degree: float = 10.0, seed: int = 1, weighted: bool = True, tier: str = "i32",
        device="cpu") -> CSRGraph:
    """Random geometric graph: n points uniform in the unit square, an edge
    between points closer than r = sqrt(mean_degree / (pi n)); weights uniform
    in [1, 10] when ``weighted``."""
    gen = _gen(seed, "cpu")
    pts = torch.rand(n, 2, generator=gen, dtype=torch.float64).to(device)
    r = math.sqrt(mean_degree / (math.pi * n))
    cells = max(1, int(1.0 / r))
    cx = (pts[:, 0] * cells).long().clamp_(max=cells - 1)
    cy = (pts[:, 1] * cells).long().clamp_(max=cells - 1)
    cell = cy * cells + cx
    order = torch.argsort(cell, stable=True)  # stable: the same edge order (and weights) on every device
    cell_sorted = cell[order]
    starts = torch.searchsorted(cell_sorted, torch.arange(cells * cells + 1, device=device))
    us, vs = [], []
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            ncx = cx + dx
            ncy = cy + dy
            ok = (ncx >= 0) & (ncx < cells) & (ncy >= 0) & (ncy < cells)
            src = torch.nonzero(ok).flatten()
            nc = (ncy[src] * cells + ncx[src])
            lo = starts[nc]
            cnt = starts[nc + 1] - lo
            tot = int(cnt.sum())
            if tot == 0:
                continue
            rep_src = torch.repeat_interleave(src, cnt)
            base = torch.repeat_interleave(lo - (torch.cumsum(cnt, 0) - cnt), cnt)
            pos = torch.arange(tot, device=device) + base
            dst = order[pos]
            keep = rep_src < dst
            rep_src = rep_src[keep]
            dst = dst[keep]
            d2 = ((pts[rep_src] - pts[dst]) ** 2).sum(1)
            close = d2 < r * r
            us.append(rep_src[close])
            vs.append(dst[close])
    u = torch.cat(us)
    v = torch.cat(vs)
    w = None
    if weighted:
        w = torch.randint(1, 11, (u.numel(),), generator=gen).to(device)
    return from_undirected(n, u, v, w, tier)


def random_graph(n: int, m: int, seed: int = 1, weighted: bool = True, tier: str = "i32") -> CSRGraph:
    """Erdos-Renyi-style multigraph sample reduced to a simple graph (tests)."""
    gen = _gen(seed, "cpu")
    u = torch.randint(0, n, (m,), generator=gen)
    v = torch.randint(0, n, (m,), generator=gen)
    lo = torch.minimum(u, v)
    hi = torch.maximum(u, v)
    keep = lo != hi
    key = torch.unique(lo[keep] * n + hi[keep])
    w = torch.randint(1, 11, (key.numel(),), generator=gen) if weighted else None
    return from_undirected(n, key // n, key % n, w, tier)


# ------------------------------------------------------------------ METIS I/O
def read_metis(path: str, tier: str = "i32", threads: int = 0) -> CSRGraph:
    """METIS text graph (app/io.hpp:99-217) read by the library's parallel
    reader (jet_read_metis): '%' comments, header 'n m [fmt [ncon]]', fmt 0
    (no weights) or 1 (edge weights), 1-based neighbour ids.  Vertex weights
    are set to 1 as the reference's driver does (app/driver.cpp:102-103);
    unweighted files give unit edge weights and uniform=True."""
    import ctypes
    from . import load, _check
    lib = load()
    n = ctypes.c_int64(0)
    nnz = ctypes.c_int64(0)
    row, adj, val = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    uni = ctypes.c_int(0)
    _check(lib.jet_read_metis(path.encode(), TIER_ID[tier], int(threads), ctypes.byref(n), ctypes.byref(nnz),
                              ctypes.byref(row), ctypes.byref(adj), ctypes.byref(val), ctypes.byref(uni)))
    o, e, w = TIERS[tier]
    try:
        def grab(ptr, count, dt):
            npdt = torch.empty(0, dtype=dt).numpy().dtype
            buf = (ctypes.c_char * (count * npdt.itemsize)).from_address(ptr.value) if count else b""
            return torch.from_numpy(np.frombuffer(buf, dtype=npdt, count=count).copy())
        nn, mm = int(n.value), int(nnz.value)
        row_t = grab(row, nn + 1, e)
        adj_t = grab(adj, mm, o)
        val_t = grab(val, mm, w)
    finally:
        for ptr in (row, adj, val):
            lib.jet_free_host(ptr)
    return CSRGraph(nn, row_t, adj_t, val_t, torch.ones(nn, dtype=w), bool(uni.value), tier)


def write_metis(g: CSRGraph, path: str) -> None:
    row, adj, val, _ = g.numpy()
    with open(path, "w") as f:
        f.write("%d %d%s\n" % (g.n, g.nnz // 2, "" if g.uniform else " 1"))
        for i in range(g.n):
            a = adj[row[i]:row[i + 1]] + 1
            if g.uniform:
                f.write(" ".join(map(str, a.tolist())) + "\n")
            else:
                w = val[row[i]:row[i + 1]]
                f.write(" ".join("%d %d" % (x, y) for x, y in zip(a.tolist(), w.tolist())) + "\n")


def write_part(part, path: str) -> None:
    """One part id per line (app/io.hpp:219-231)."""
    p = part.cpu().numpy() if isinstance(part, torch.Tensor) else np.asarray(part)
    with open(path, "w") as f:
        f.write("".join("%d\n" % x for x in p.tolist()))


def read_part(path: str, n: int) -> np.ndarray:
    """Partition file written by write_part (app/io.hpp:233-244)."""
    vals = np.loadtxt(path, dtype=np.int64, ndmin=1)
    return vals[:n].astype(np.int32)
