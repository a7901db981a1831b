"""ctypes wrapper around the CPU oracle (oracle/jet_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
benchmark's CPU-baseline leg.  Parity status: pinned to the reference's own
code built under oracle/_ref/ (oracle/ref.py, tests/test_ref_pin.py).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libjet_oracle.so")
_lib = None

TIER_DT = {0: (np.int32, np.int32, np.int32), 1: (np.int32, np.int64, np.int64), 2: (np.int64, np.int64, np.int64)}
TIER_ID = {"i32": 0, "big": 1, "biggest": 2}


class OrcConfig(ctypes.Structure):
    _fields_ = [("coarsening_alg", ctypes.c_int32), ("num_parts", ctypes.c_int32),
                ("max_imb_ratio", ctypes.c_double), ("refine_tolerance", ctypes.c_double),
                ("ultra_settings", ctypes.c_int32), ("verbose", ctypes.c_int32)]


class OrcStats(ctypes.Structure):
    _fields_ = [("cut", ctypes.c_int64), ("largest", ctypes.c_int64), ("smallest", ctypes.c_int64),
                ("imb", ctypes.c_double), ("levels", ctypes.c_int32), ("coarsest_n", ctypes.c_int32),
                ("t_coarsen", ctypes.c_double), ("t_init", ctypes.c_double), ("t_refine", ctypes.c_double),
                ("t_total", ctypes.c_double),
                ("level_cut", ctypes.c_int64 * 256), ("level_n", ctypes.c_int64 * 256),
                ("level_nnz", ctypes.c_int64 * 256), ("level_iters", ctypes.c_int32 * 256),
                ("level_lp_iters", ctypes.c_int32 * 256)]


def build() -> str:
    """Compiles the oracle with its Makefile (g++, CUDA's bundled Metis)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(_HERE, "jet_oracle.cpp")
        if not os.path.exists(_LIB_PATH) or (os.path.exists(src) and os.path.getmtime(src) > os.path.getmtime(_LIB_PATH)):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.orc_rng.restype = ctypes.c_uint64
        _lib.orc_rng.argtypes = [ctypes.c_uint64] * 3
        _lib.orc_pod_hash32.restype = ctypes.c_uint32
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


def _tier_of(row, adj):
    if adj.dtype == np.int64:
        return 2
    return 1 if row.dtype == np.int64 else 0


class G:
    """numpy view of a graph in one tier."""

    def __init__(self, row, adj, val, vw, uniform=False):
        self.row = np.ascontiguousarray(row)
        self.adj = np.ascontiguousarray(adj)
        self.val = np.ascontiguousarray(val)
        self.vw = np.ascontiguousarray(vw)
        self.n = len(self.row) - 1
        self.uniform = bool(uniform)
        self.tier = _tier_of(self.row, self.adj)
        od, ed, wd = TIER_DT[self.tier]
        assert self.adj.dtype == od and self.row.dtype == ed and self.val.dtype == wd and self.vw.dtype == wd

    @classmethod
    def from_csr(cls, g):
        row, adj, val, vw = g.numpy()
        return cls(row, adj, val, vw, g.uniform)


def partition(g: G, k: int, alg: int = 1, imb: float = 1.03, seed: int = 1, tol: float = 0.999,
              ultra: bool = False, verbose: bool = False):
    cfg = OrcConfig(alg, k, imb, tol, int(ultra), int(verbose))
    part = np.zeros(g.n, dtype=np.int32)
    cut = ctypes.c_int64(0)
    st = OrcStats()
    rc = lib().orc_partition(g.tier, ctypes.byref(cfg), ctypes.c_int64(g.n), _p(g.row), _p(g.adj), _p(g.val), _p(g.vw),
                             int(g.uniform), ctypes.c_uint64(seed), _p(part), ctypes.byref(cut), ctypes.byref(st))
    if rc != 0:
        raise RuntimeError("oracle partition failed with code %d" % rc)
    return part, int(cut.value), st


def coarsen(g: G, alg: int, level: int = 1, seed: int = 1, uniform=None):
    od = TIER_DT[g.tier][0]
    m = np.zeros(g.n, dtype=od)
    hn = np.zeros(g.n, dtype=od)
    nc = ctypes.c_int64(0)
    u = g.uniform if uniform is None else uniform
    rc = lib().orc_coarsen(g.tier, alg, level, ctypes.c_uint64(seed), ctypes.c_int64(g.n), _p(g.row), _p(g.adj),
                           _p(g.val), _p(g.vw), int(u), _p(m), _p(hn), ctypes.byref(nc))
    assert rc == 0
    return m, int(nc.value), hn


def contract(g: G, cmap, nc: int):
    od, ed, wd = TIER_DT[g.tier]
    cmap = np.ascontiguousarray(cmap, dtype=od)
    crow = np.zeros(nc + 1, dtype=ed)
    cadj = np.zeros(max(1, len(g.adj)), dtype=od)
    cval = np.zeros(max(1, len(g.adj)), dtype=wd)
    cvw = np.zeros(max(1, nc), dtype=wd)
    cnnz = ctypes.c_int64(0)
    rc = lib().orc_contract(g.tier, ctypes.c_int64(g.n), _p(g.row), _p(g.adj), _p(g.val), _p(g.vw), _p(cmap),
                            ctypes.c_int64(nc), _p(crow), _p(cadj), _p(cval), _p(cvw), ctypes.byref(cnnz))
    assert rc == 0
    m = int(cnnz.value)
    return G(crow, cadj[:m].copy(), cval[:m].copy(), cvw[:nc].copy(), False)


def conn_build(g: G, part, k: int):
    od, ed, wd = TIER_DT[g.tier]
    part = np.ascontiguousarray(part, dtype=np.int32)
    off = np.zeros(g.n + 1, dtype=ed)
    ent = np.zeros(max(1, len(g.adj)), dtype=np.int32)
    val = np.zeros(max(1, len(g.adj)), dtype=wd)
    size = np.zeros(g.n, dtype=np.int32)
    rc = lib().orc_conn_build(g.tier, ctypes.c_int64(g.n), _p(g.row), _p(g.adj), _p(g.val), _p(part), k, _p(off),
                              _p(ent), _p(val), _p(size))
    assert rc == 0
    c = int(off[-1])
    return off, ent[:c].copy(), val[:c].copy(), size


def refine_iters(g: G, part, k: int, imb: float, filter_ratio: float, iters: int):
    """Runs `iters` refinement iterations (LP / weak / strong, as jet_refine's
    loop body would choose them).  Returns a dict with the final state."""
    od, ed, wd = TIER_DT[g.tier]
    part = np.array(part, dtype=np.int32, copy=True)
    sizes = np.zeros(k, dtype=wd)
    cut = ctypes.c_int64(0)
    off = np.zeros(g.n + 1, dtype=ed)
    ent = np.zeros(max(1, len(g.adj)), dtype=np.int32)
    cval = np.zeros(max(1, len(g.adj)), dtype=wd)
    size = np.zeros(g.n, dtype=np.int32)
    dc = np.zeros(g.n, dtype=np.int32)
    moves = np.zeros(max(1, iters), dtype=np.int64)
    kinds = np.zeros(max(1, iters), dtype=np.int32)
    rc = lib().orc_refine_iters(g.tier, ctypes.c_int64(g.n), _p(g.row), _p(g.adj), _p(g.val), _p(g.vw), _p(part), k,
                                ctypes.c_double(imb), ctypes.c_double(filter_ratio), iters, _p(sizes),
                                ctypes.byref(cut), _p(off), _p(ent), _p(cval), _p(size), _p(dc), _p(moves), _p(kinds))
    if rc != 0:
        raise RuntimeError("oracle refine_iters failed with code %d" % rc)
    c = int(off[-1])
    return dict(part=part, sizes=sizes, cut=int(cut.value), off=off, ent=ent[:c].copy(), val=cval[:c].copy(),
                size=size, dest_cache=dc, moves=moves[:iters], kinds=kinds[:iters])


def refine_level(g: G, part, k: int, imb: float = 1.03, tol: float = 0.999):
    part = np.array(part, dtype=np.int32, copy=True)
    cut = ctypes.c_int64(0)
    it = ctypes.c_int32(0)
    rc = lib().orc_refine_level(g.tier, ctypes.c_int64(g.n), _p(g.row), _p(g.adj), _p(g.val), _p(g.vw), _p(part), k,
                                ctypes.c_double(imb), ctypes.c_double(tol), int(g.uniform), ctypes.byref(cut),
                                ctypes.byref(it))
    assert rc == 0
    return part, int(cut.value), int(it.value)


def pstat(g: G, part, k: int):
    """[cut, max part cut, comm size, largest, smallest, total] (app/part_eval.cpp)."""
    out = np.zeros(6, dtype=np.int64)
    part = np.ascontiguousarray(part, dtype=np.int32)
    rc = lib().orc_pstat(g.tier, ctypes.c_int64(g.n), _p(g.row), _p(g.adj), _p(g.val), _p(g.vw), _p(part), k, _p(out))
    assert rc == 0
    return out


def metis(g: G, k: int, imb: float = 1.03):
    part = np.zeros(g.n, dtype=np.int32)
    rc = lib().orc_metis(g.tier, ctypes.c_int64(g.n), _p(g.row), _p(g.adj), _p(g.val), _p(g.vw), k,
                         ctypes.c_double(imb), _p(part))
    if rc != 0:
        raise RuntimeError("metis failed")
    return part


def gain_bucket(gain: int, vwgt: int, wide: bool = False) -> int:
    if wide:
        return lib().orc_gain_bucket64(ctypes.c_int64(gain), ctypes.c_int64(vwgt))
    return lib().orc_gain_bucket32(ctypes.c_int32(gain), ctypes.c_int32(vwgt))


def rng(seed: int, stream: int, idx: int) -> int:
    return int(lib().orc_rng(seed, stream, idx))


def uncoarsen(levels, maps, coarsest_part, k: int, imb: float = 1.03, tol: float = 0.999, ultra: bool = False):
    """Refines a fixed hierarchy (levels[0] finest, maps[l] sends level l-1 to
    level l, maps[0] unused) from a coarsest partition.  Returns (part, cut)."""
    tier = levels[0].tier
    nl = len(levels)
    ns = np.array([lv.n for lv in levels], dtype=np.int64)
    arr = lambda xs: (ctypes.c_void_p * nl)(*[ctypes.c_void_p(x.ctypes.data) if x is not None else None for x in xs])
    od = TIER_DT[tier][0]
    mp = [None] + [np.ascontiguousarray(m, dtype=od) for m in maps[1:]]
    cp = np.ascontiguousarray(coarsest_part, dtype=np.int32)
    cfg = OrcConfig(1, k, imb, tol, int(ultra), 0)
    part = np.zeros(levels[0].n, dtype=np.int32)
    cut = ctypes.c_int64(0)
    rc = lib().orc_uncoarsen(tier, nl, _p(ns), arr([lv.row for lv in levels]), arr([lv.adj for lv in levels]),
                             arr([lv.val for lv in levels]), arr([lv.vw for lv in levels]), arr(mp), _p(cp),
                             ctypes.byref(cfg), int(levels[0].uniform), _p(part), ctypes.byref(cut))
    if rc != 0:
        raise RuntimeError("oracle uncoarsen failed with code %d" % rc)
    return part, int(cut.value)
