"""ctypes wrapper around the Jet reference's own CPU code (oracle/ref_harness.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/ to pin the CPU oracle and the GPU
path to the reference, and by the benchmark's reference arm (the timed CPU
baseline).  The libraries are built by oracle/ref.mk from the unmodified
reference sources and the Kokkos stand-in in oracle/kokkos_shim/:

    libjet_ref_serial.so  Kokkos::Serial (the reference's single-thread run)
    libjet_ref_host.so    OpenMP on every host core (the reference's jet_host)

Every function takes the same arguments as its namesake in oracle.py and
returns the same shapes, so tests can compare the two directly.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from oracle import TIER_DT, G, _p  # noqa: F401  (G is re-exported for callers)

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {"serial": os.path.join(_HERE, "_ref", "libjet_ref_serial.so"),
         "host": os.path.join(_HERE, "_ref", "libjet_ref_host.so")}
_REF_SRC = "/root/reference"
_loaded = {}


class ReferenceCrash(RuntimeError):
    """The reference raised SIGFPE: its rebalance_weak divides by zero when no
    part is undersized (src/jet_refiner.hpp:618)."""


def _rc(rc: int, what: str):
    if rc == 8:
        raise ReferenceCrash("the reference's %s raised SIGFPE (division by zero in rebalance_weak, "
                             "src/jet_refiner.hpp:618)" % what)
    if rc != 0:
        raise RuntimeError("reference %s failed with code %d" % (what, rc))


def available(space: str = "serial") -> bool:
    """True when the library is built, or can be built because the reference
    sources are present on this machine."""
    return os.path.exists(_LIBS[space]) or os.path.isdir(_REF_SRC)


def build() -> None:
    """Builds oracle/_ref/ with oracle/ref.mk (needs the reference sources)."""
    subprocess.run(["make", "-s", "-f", "ref.mk", "REF=" + _REF_SRC], cwd=_HERE, check=True)


def lib(space: str = "serial"):
    if space not in _loaded:
        path = _LIBS[space]
        if not os.path.exists(path):
            if not os.path.isdir(_REF_SRC):
                raise RuntimeError("%s is not built and the reference sources are absent" % path)
            build()
        lib_ = ctypes.CDLL(path)
        lib_.ref_pod_hash32.restype = ctypes.c_uint32
        _loaded[space] = lib_
    return _loaded[space]


def concurrency(space: str = "host") -> int:
    return int(lib(space).ref_concurrency())


def partition(g: G, k: int, alg: int = 1, imb: float = 1.03, seed: int = 1, tol: float = 0.999,
              ultra: bool = False, space: str = "serial"):
    """Full partition through the reference's partitioner::partition.
    Returns (part, cut, imbalance, seconds of the partition call)."""
    part = np.zeros(g.n, dtype=np.int32)
    cut = ctypes.c_int64(0)
    imb_out = ctypes.c_double(0)
    secs = ctypes.c_double(0)
    rc = lib(space).ref_partition(g.tier, alg, k, ctypes.c_double(imb), ctypes.c_double(tol), int(ultra),
                                  ctypes.c_int64(g.n), _p(g.row), _p(g.adj), _p(g.val), _p(g.vw), int(g.uniform),
                                  ctypes.c_uint64(seed), _p(part), ctypes.byref(cut), ctypes.byref(imb_out),
                                  ctypes.byref(secs), 1)
    _rc(rc, "partition")
    return part, int(cut.value), float(imb_out.value), float(secs.value)


def coarsen(g: G, alg: int, seed: int = 1, uniform=None, space: str = "serial"):
    od = TIER_DT[g.tier][0]
    m = np.zeros(g.n, dtype=od)
    nc = ctypes.c_int64(0)
    u = g.uniform if uniform is None else uniform
    rc = lib(space).ref_coarsen(g.tier, alg, ctypes.c_uint64(seed), ctypes.c_int64(g.n), _p(g.row), _p(g.adj),
                                _p(g.val), _p(g.vw), int(u), _p(m), ctypes.byref(nc))
    assert rc == 0
    return m, int(nc.value)


def contract(g: G, cmap, nc: int, space: str = "serial"):
    """Coarse graph for a given map; rows in the reference's hash-slot order."""
    od, ed, wd = TIER_DT[g.tier]
    cmap = np.ascontiguousarray(cmap, dtype=od)
    crow = np.zeros(nc + 1, dtype=ed)
    cadj = np.zeros(max(1, len(g.adj)), dtype=od)
    cval = np.zeros(max(1, len(g.adj)), dtype=wd)
    cvw = np.zeros(max(1, nc), dtype=wd)
    cnnz = ctypes.c_int64(0)
    rc = lib(space).ref_contract(g.tier, ctypes.c_int64(g.n), _p(g.row), _p(g.adj), _p(g.val), _p(g.vw), _p(cmap),
                                 ctypes.c_int64(nc), _p(crow), _p(cadj), _p(cval), _p(cvw), ctypes.byref(cnnz))
    assert rc == 0
    m = int(cnnz.value)
    return G(crow, cadj[:m].copy(), cval[:m].copy(), cvw[:nc].copy(), False)


def conn_build(g: G, part, k: int, space: str = "serial"):
    od, ed, wd = TIER_DT[g.tier]
    part = np.ascontiguousarray(part, dtype=np.int32)
    off = np.zeros(g.n + 1, dtype=ed)
    ent = np.zeros(max(1, len(g.adj)), dtype=np.int32)
    val = np.zeros(max(1, len(g.adj)), dtype=wd)
    size = np.zeros(g.n, dtype=np.int32)
    rc = lib(space).ref_conn_build(g.tier, ctypes.c_int64(g.n), _p(g.row), _p(g.adj), _p(g.val), _p(part), k,
                                   _p(off), _p(ent), _p(val), _p(size))
    assert rc == 0
    c = int(off[-1])
    return off, ent[:c].copy(), val[:c].copy(), size


def refine_iters(g: G, part, k: int, imb: float, filter_ratio: float, iters: int, space: str = "serial"):
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
    rc = lib(space).ref_refine_iters(g.tier, ctypes.c_int64(g.n), _p(g.row), _p(g.adj), _p(g.val), _p(g.vw),
                                     _p(part), k, ctypes.c_double(imb), ctypes.c_double(filter_ratio), iters,
                                     _p(sizes), ctypes.byref(cut), _p(off), _p(ent), _p(cval), _p(size), _p(dc),
                                     _p(moves), _p(kinds))
    _rc(rc, "refinement iterations")
    c = int(off[-1])
    return dict(part=part, sizes=sizes, cut=int(cut.value), off=off, ent=ent[:c].copy(), val=cval[:c].copy(),
                size=size, dest_cache=dc, moves=moves[:iters], kinds=kinds[:iters])


def refine_level(g: G, part, k: int, imb: float = 1.03, tol: float = 0.999, ultra: bool = False,
                 space: str = "serial"):
    part = np.array(part, dtype=np.int32, copy=True)
    cut = ctypes.c_int64(0)
    it = ctypes.c_int32(0)
    rc = lib(space).ref_refine_level(g.tier, ctypes.c_int64(g.n), _p(g.row), _p(g.adj), _p(g.val), _p(g.vw),
                                     _p(part), k, ctypes.c_double(imb), ctypes.c_double(tol), int(ultra),
                                     int(g.uniform), ctypes.byref(cut), ctypes.byref(it))
    _rc(rc, "jet_refine")
    return part, int(cut.value)


def uncoarsen(levels, maps, coarsest_part, k: int, imb: float = 1.03, tol: float = 0.999, ultra: bool = False,
              space: str = "serial"):
    """Refines a fixed hierarchy (levels[0] finest, maps[l] sends level l-1 to
    level l, maps[0] unused) from a coarsest partition.  Returns (part, cut)."""
    tier = levels[0].tier
    nl = len(levels)
    ns = np.array([lv.n for lv in levels], dtype=np.int64)
    arr = lambda xs: (ctypes.c_void_p * nl)(*[ctypes.c_void_p(x.ctypes.data) if x is not None else None for x in xs])
    od = TIER_DT[tier][0]
    mp = [None] + [np.ascontiguousarray(m, dtype=od) for m in maps[1:]]
    cp = np.ascontiguousarray(coarsest_part, dtype=np.int32)
    part = np.zeros(levels[0].n, dtype=np.int32)
    cut = ctypes.c_int64(0)
    rc = lib(space).ref_uncoarsen(tier, nl, _p(ns), arr([lv.row for lv in levels]), arr([lv.adj for lv in levels]),
                                  arr([lv.val for lv in levels]), arr([lv.vw for lv in levels]), arr(mp), _p(cp), k,
                                  ctypes.c_double(imb), ctypes.c_double(tol), int(ultra), int(levels[0].uniform),
                                  _p(part), ctypes.byref(cut))
    _rc(rc, "uncoarsen")
    return part, int(cut.value)


def pstat(g: G, part, k: int, space: str = "serial"):
    """[cut, max part cut, comm size, largest, smallest, total] (app/part_eval.cpp)."""
    out = np.zeros(6, dtype=np.int64)
    part = np.ascontiguousarray(part, dtype=np.int32)
    rc = lib(space).ref_pstat(g.tier, ctypes.c_int64(g.n), _p(g.row), _p(g.adj), _p(g.val), _p(g.vw), _p(part), k,
                              _p(out))
    assert rc == 0
    return out


def gain_bucket(gain: int, vwgt: int, wide: bool = False) -> int:
    if wide:
        return lib().ref_gain_bucket64(ctypes.c_int64(gain), ctypes.c_int64(vwgt))
    return lib().ref_gain_bucket32(ctypes.c_int32(gain), ctypes.c_int32(vwgt))


def load_metis(path: str, cap_rows: int, cap_nnz: int):
    """The reference's own METIS reader (app/io.hpp:99-217), std tier.
    Returns (row, adj, val, uniform) or None when it rejects the file."""
    n = ctypes.c_int64(0)
    nnz = ctypes.c_int64(0)
    row = np.zeros(cap_rows + 1, dtype=np.int32)
    adj = np.zeros(max(cap_nnz, 1), dtype=np.int32)
    val = np.zeros(max(cap_nnz, 1), dtype=np.int32)
    uni = ctypes.c_int(0)
    rc = lib().ref_load_metis(path.encode(), ctypes.byref(n), ctypes.byref(nnz), _p(row), ctypes.c_int64(cap_rows + 1),
                              _p(adj), _p(val), ctypes.c_int64(cap_nnz), ctypes.byref(uni))
    if rc == 1:
        return None
    assert rc == 0, "capacity too small"
    nn, mm = int(n.value), int(nnz.value)
    return row[:nn + 1].copy(), adj[:mm].copy(), val[:mm].copy(), bool(uni.value)


def pod_hash32(x: int) -> int:
    return int(lib().ref_pod_hash32(ctypes.c_int32(x)))
