"""B200 Jet multilevel k-way graph partitioner -- Python host mirror.

This module binds the C ABI of ``libjetb200.so`` (declared in
``include/jet_b200.h``) with ctypes and mirrors the reference's public
surface (header/jet.h, header/jet_config.h, header/experiment_data.hpp):

* ``config_t``       -- the reference's config struct, same fields/defaults
* ``partition*``     -- the nine entry points of header/jet.h:46-107
* ``experiment_data``-- per-phase timings and per-level refinement records
* component entry points (``coarsen_map``, ``contract``, ``conn_build``,
  ``refine_iters``, ``refine_level``, ``pstat``, ``project``) over device
  tensors, used by the parity tests.

PyTorch is used only to hold device memory and pass streams.  The CUDA
library is required: every call raises ``JetError`` when it cannot be loaded
or no CUDA device is present -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
import numpy as np
from typing import List, Optional

import torch

from . import graphs  # noqa: F401  (re-exported)
from .graphs import CSRGraph, TIERS, TIER_ID

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libjetb200.so")

JET_OK = 0
JET_ERR_INVALID = 1
JET_ERR_CUDA = 2
JET_ERR_METIS = 3
JET_ERR_OOM = 4
JET_ERR_OVERFLOW = 5
JET_ERR_TIMEOUT = 6
JET_ERR_NOT_BUILT = 7
JET_MEM_HOST = 0
JET_MEM_DEVICE = 1

ERROR_NAMES = {0: "JET_OK", 1: "JET_ERR_INVALID", 2: "JET_ERR_CUDA", 3: "JET_ERR_METIS", 4: "JET_ERR_OOM",
               5: "JET_ERR_OVERFLOW", 6: "JET_ERR_TIMEOUT", 7: "JET_ERR_NOT_BUILT"}

MEASUREMENT_NAMES = [  # header/experiment_data.hpp:77-98
    "coarsen-map", "coarsen-build", "coarsen-count", "coarsen-prefix-sum", "coarsen-bucket", "coarsen-dedupe",
    "coarsen-radix-sort", "coarsen-radix-dedupe", "coarsen-write-graph", "coarsen-permute", "coarsen-map-construct",
    "heavy", "initial-transfer-to-device", "hashmap-allocate", "hashmap-insert", "initial-partition", "coarsen",
    "refine", "free-graph", "total"]

EXPORTED_SYMBOLS = [
    "jet_partition_i32", "jet_partition_big", "jet_partition_biggest", "jet_coarsen_map", "jet_contract",
    "jet_conn_build", "jet_refine_iters", "jet_refine_level", "jet_pstat", "jet_project", "jet_version",
    "jet_last_error", "jet_device_ok", "jet_prof_enable", "jet_prof_read", "jet_launch_count", "jet_pstat_noalloc",
    "jet_set_refine_drivers", "jet_partition_batch", "jet_server_create", "jet_server_submit", "jet_server_wait",
    "jet_server_footprint", "jet_server_stats_get", "jet_server_destroy", "jet_refine_hierarchy",
    "jet_device_alloc", "jet_device_free", "jet_copy", "jet_read_metis", "jet_free_host",
    "jet_test_inject_metis_failures", "jet_test_grid_barrier", "jet_test_table_overflow", "jet_prof_phases", "jet_metis_call_stats",
]


def metis_call_stats() -> dict:
    """Where this process's coarsest-graph Metis calls ran (jet_metis_call_stats)."""
    out = (ctypes.c_int64 * 6)()
    _check(load().jet_metis_call_stats(out))
    return dict(helper_calls=out[0], helper_failures=out[1], inprocess_calls=out[2], helpers=out[3],
                helpers_unavailable=bool(out[4]), helper_metis_errors=out[5])

PHASES = ["lp_select", "afterburn", "afterburn_hub", "reb_prep", "reb_select", "bucket_scan", "cand_sort", "evict",
          "strong_tail", "apply", "update_sub", "update_add", "rebuild", "cut", "control", "copy", "cookie",
          "strong_first", "redraw", "weight_scan"]


def prof_phases(on: bool):
    """Phase clocks of the persistent level loops: prof_phases(True) starts,
    prof_phases(False) returns {driver: {phase: (cycles, count)}}."""
    out = (ctypes.c_uint64 * (6 * 24))()
    _check(load().jet_prof_phases(int(on), out))
    if on:
        return None
    res = {}
    for d, nm in enumerate(["cta", "cluster", "coop"]):
        res[nm] = {p: (int(out[48 * d + i]), int(out[48 * d + 24 + i])) for i, p in enumerate(PHASES)
                   if out[48 * d + 24 + i]}
    return res

# level-loop drivers (jet_set_refine_drivers)
DRIVER_CTA, DRIVER_COOP, DRIVER_GRAPH, DRIVER_CLUSTER, DRIVER_CTA_SMEM, DRIVER_REB_QUEUE, DRIVER_ALL = 1, 2, 4, 8, 16, 32, 63


class JetError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("%s: %s" % (ERROR_NAMES.get(code, str(code)), msg))
        self.code = code


# ------------------------------------------------------------------ C structs
class jet_config_c(ctypes.Structure):
    _fields_ = [("coarsening_alg", ctypes.c_int32), ("num_iter", ctypes.c_int32), ("max_imb_ratio", ctypes.c_double),
                ("num_parts", ctypes.c_int32), ("refine_tolerance", ctypes.c_double), ("dump_coarse", ctypes.c_int32),
                ("verbose", ctypes.c_int32), ("ultra_settings", ctypes.c_int32)]


class jet_level_stats_c(ctypes.Structure):
    _fields_ = [("edge_cut", ctypes.c_int64), ("imb", ctypes.c_double), ("num_edges", ctypes.c_uint64),
                ("num_vertices", ctypes.c_uint64), ("total_ref_time", ctypes.c_double),
                ("iterations_time", ctypes.c_double), ("total_iterations", ctypes.c_int32),
                ("lp_iterations", ctypes.c_int32)]


class jet_stats_c(ctypes.Structure):
    _fields_ = [("measurements", ctypes.c_double * 20), ("num_levels", ctypes.c_int32),
                ("levels", jet_level_stats_c * 256), ("edge_cut", ctypes.c_int64), ("max_part_cut", ctypes.c_int64),
                ("objective", ctypes.c_int64), ("imb_ratio", ctypes.c_double), ("largest_part", ctypes.c_int64),
                ("smallest_part", ctypes.c_int64), ("coarsest_vertices", ctypes.c_int64),
                ("refine_iterations", ctypes.c_int64)]


_lib = None


def library_path() -> str:
    return LIB_PATH


def load(build_if_missing: bool = False):
    """Loads libjetb200.so; raises JetError when it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if build_if_missing:
            from . import build as _b  # noqa
            _b.build()
        else:
            raise JetError(JET_ERR_NOT_BUILT, "%s is missing; run jet-partitioner-official-fork_b200/build.py" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    lib.jet_version.restype = ctypes.c_char_p
    lib.jet_last_error.restype = ctypes.c_char_p
    lib.jet_launch_count.restype = ctypes.c_int64
    lib.jet_set_refine_drivers.restype = ctypes.c_int
    lib.jet_set_refine_drivers.argtypes = [ctypes.c_int]
    _lib = lib
    return lib


def _check(rc: int):
    if rc != JET_OK:
        raise JetError(rc, load().jet_last_error().decode())


def _require_cuda():
    if not torch.cuda.is_available():
        raise JetError(JET_ERR_NOT_BUILT, "no CUDA device: the B200 partitioner has no CPU path")
    _check(load().jet_device_ok())


def _ptr(t: Optional[torch.Tensor]):
    return ctypes.c_void_p(t.data_ptr() if t is not None else 0)


def _stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


# ------------------------------------------------------------------ reference mirror
@dataclass
class config_t:
    """header/jet_config.h:43-52."""

    coarsening_alg: int = 0
    num_iter: int = 1
    max_imb_ratio: float = 1.03
    num_parts: int = 2
    refine_tolerance: float = 0.999
    dump_coarse: bool = False
    verbose: bool = False
    ultra_settings: bool = False

    def to_c(self) -> jet_config_c:
        return jet_config_c(int(self.coarsening_alg), int(self.num_iter), float(self.max_imb_ratio),
                            int(self.num_parts), float(self.refine_tolerance), int(self.dump_coarse),
                            int(self.verbose), int(self.ultra_settings))


@dataclass
class CoarseLevel:
    edge_cut: int
    imb: float
    numEdges: int
    numVertices: int
    totalRefTime: float
    iterationsTime: float
    totalIterations: int
    lpIterations: int


@dataclass
class experiment_data:
    """header/experiment_data.hpp:74-243 (fields, log and reports)."""

    measurements: List[float] = field(default_factory=lambda: [0.0] * 20)
    coarseLevels: List[CoarseLevel] = field(default_factory=list)
    fine_ec: int = 0
    max_part_cut: int = 0
    obj: int = 0
    imb_ratio: float = 0.0
    largest_part: int = 0
    smallest_part: int = 0
    coarsest_vertices: int = 0
    refine_iterations: int = 0

    def fill(self, st: jet_stats_c):
        self.measurements = [st.measurements[i] for i in range(20)]
        self.coarseLevels = [CoarseLevel(lv.edge_cut, lv.imb, lv.num_edges, lv.num_vertices, lv.total_ref_time,
                                         lv.iterations_time, lv.total_iterations, lv.lp_iterations)
                             for lv in st.levels[:min(st.num_levels, 256)]]
        self.fine_ec = st.edge_cut
        self.max_part_cut = st.max_part_cut
        self.obj = st.objective
        self.imb_ratio = st.imb_ratio
        self.largest_part = st.largest_part
        self.smallest_part = st.smallest_part
        self.coarsest_vertices = st.coarsest_vertices
        self.refine_iterations = st.refine_iterations

    def getMeasurement(self, name: str) -> float:
        return self.measurements[MEASUREMENT_NAMES.index(name)]

    def log(self, filename: str, first: bool, last: bool):
        with open(filename, "a") as f:
            if first:
                f.write("[")
            f.write("{")
            f.write('"edge-cut":%d,"max-part-cut":%d,"objective":%d,"imbalance-ratio":%f,'
                    % (self.fine_ec, self.max_part_cut, self.obj, self.imb_ratio))
            for nm, v in zip(MEASUREMENT_NAMES, self.measurements):
                f.write('"%s-duration-seconds":%f,' % (nm, v))
            f.write('"number-coarse-levels":%d,' % len(self.coarseLevels))
            f.write('"finest-refinement-duration-seconds":%f' % (self.coarseLevels[-1].totalRefTime if self.coarseLevels else 0.0))
            f.write("}")
            f.write("]" if last else ",")

    def refinementReport(self) -> str:
        lines = ["%-6s%-16s%-10s%-13s%-16s%-22s%-17s%-14s%-23s" % (
            "Level", "Edge Cut", "Imbalance", "Vertices", "Edges", "Total Refinement Time", "Total Iterations",
            "LP Iterations", "Average Iteration Time")]
        n = len(self.coarseLevels)
        for i, cl in enumerate(self.coarseLevels):
            avg = cl.iterationsTime / cl.totalIterations if cl.totalIterations else 0.0
            lines.append("%-6d%-16d%-10.6f%-13d%-16d%-22.6f%-17d%-14d%-23.6f" % (
                n - 1 - i, cl.edge_cut, cl.imb, cl.numVertices, cl.numEdges, cl.totalRefTime, cl.totalIterations,
                cl.lpIterations, avg))
        return "\n".join(lines)

    def verboseReport(self) -> str:
        m = dict(zip(MEASUREMENT_NAMES, self.measurements))
        return ("Final cut: %d; Max part cut: %d; imb: %f; largest: %d; smallest: %d\n"
                "Coarsening time: %.5g\nInitial partitioning time: %.5g\nUncoarsening time: %.5g\n"
                "Total Partitioning Time: %.5g\nComm size: %d" % (
                    self.fine_ec, self.max_part_cut, self.imb_ratio, self.largest_part, self.smallest_part,
                    m["coarsen"], m["initial-partition"], m["refine"], m["total"], self.obj))


_PARTITION_FN = {"i32": "jet_partition_i32", "big": "jet_partition_big", "biggest": "jet_partition_biggest"}


def _partition(tier: str, config: config_t, g: CSRGraph, vweights: Optional[torch.Tensor], uniform_ew: bool,
               seed: int, host_out: bool, stream=None):
    _require_cuda()
    lib = load()
    o, e, w = TIERS[tier]
    vw = g.vw if vweights is None else vweights
    on_dev = g.row.is_cuda
    row = g.row.to(e).contiguous()
    adj = g.adj.to(o).contiguous()
    val = g.val.to(w).contiguous()
    vw = vw.to(w).contiguous()
    if on_dev:
        part = torch.empty(g.n, dtype=torch.int32, device=row.device)
        mem = JET_MEM_DEVICE
    else:
        part = torch.empty(g.n, dtype=torch.int32)
        mem = JET_MEM_HOST
    cut_c = (ctypes.c_int32 if tier == "i32" else ctypes.c_int64)(0)
    st = jet_stats_c()
    cfg = config.to_c()
    sp = _stream_ptr(stream) if on_dev else ctypes.c_void_p(0)
    n_c = ctypes.c_int64(g.n) if tier == "biggest" else ctypes.c_int32(g.n)
    fn = getattr(lib, _PARTITION_FN[tier])
    rc = fn(ctypes.byref(cfg), n_c, _ptr(row), _ptr(adj), _ptr(val), _ptr(vw), int(bool(uniform_ew)), mem,
            ctypes.c_uint64(seed), sp, _ptr(part), ctypes.byref(cut_c), ctypes.byref(st))
    _check(rc)
    exp = experiment_data()
    exp.fill(st)
    if host_out:
        part = part.cpu()
    return part, int(cut_c.value), exp


# header/jet.h:46-107.  Each returns (part, edge_cut, experiment).  The *_host
# and *_serial variants take and return host tensors (the reference runs those
# on host execution spaces; here all compute is on the GPU).
def partition(config, g, vweights=None, uniform_ew=None, seed=1, stream=None):
    return _partition("i32", config, g, vweights, g.uniform if uniform_ew is None else uniform_ew, seed, False, stream)


def partition_host(config, g, vweights=None, uniform_ew=None, seed=1):
    return _partition("i32", config, g.to("cpu"), vweights, g.uniform if uniform_ew is None else uniform_ew, seed, True)


partition_serial = partition_host


def partition_big(config, g, vweights=None, uniform_ew=None, seed=1, stream=None):
    return _partition("big", config, g, vweights, g.uniform if uniform_ew is None else uniform_ew, seed, False, stream)


def partition_host_big(config, g, vweights=None, uniform_ew=None, seed=1):
    return _partition("big", config, g.to("cpu"), vweights, g.uniform if uniform_ew is None else uniform_ew, seed, True)


partition_serial_big = partition_host_big


def partition_biggest(config, g, vweights=None, uniform_ew=None, seed=1, stream=None):
    return _partition("biggest", config, g, vweights, g.uniform if uniform_ew is None else uniform_ew, seed, False, stream)


def partition_host_biggest(config, g, vweights=None, uniform_ew=None, seed=1):
    return _partition("biggest", config, g.to("cpu"), vweights, g.uniform if uniform_ew is None else uniform_ew, seed, True)


partition_serial_biggest = partition_host_biggest


# ------------------------------------------------------------------ batched and served
class jet_graph_desc(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("row_map", ctypes.c_void_p), ("entries", ctypes.c_void_p),
                ("values", ctypes.c_void_p), ("vweights", ctypes.c_void_p), ("uniform_ew", ctypes.c_int32),
                ("config", jet_config_c), ("seed", ctypes.c_uint64), ("part_out", ctypes.c_void_p),
                ("edge_cut", ctypes.c_int64), ("status", ctypes.c_int32), ("latency_ms", ctypes.c_double),
                ("error", ctypes.c_char * 112)]


class jet_server_stats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("refused", ctypes.c_int64), ("peak_footprint_bytes", ctypes.c_int64),
                ("peak_concurrent", ctypes.c_int32)]


def _desc(tier: str, config: config_t, g: CSRGraph, seed: int, keep: list) -> jet_graph_desc:
    """Fills a request for one graph; tensors it points at are appended to
    `keep` (they must outlive the call or the request)."""
    o, e, w = TIERS[tier]
    row = g.row.to(e).contiguous()
    adj = g.adj.to(o).contiguous()
    val = g.val.to(w).contiguous()
    vw = g.vw.to(w).contiguous()
    part = torch.empty(g.n, dtype=torch.int32, device=row.device)
    keep.append((row, adj, val, vw, part))
    d = jet_graph_desc()
    d.n = g.n
    d.row_map, d.entries, d.values, d.vweights = row.data_ptr(), adj.data_ptr(), val.data_ptr(), vw.data_ptr()
    d.uniform_ew = int(bool(g.uniform))
    d.config = config.to_c()
    d.seed = seed
    d.part_out = part.data_ptr()
    return d


def partition_batch(configs, graphs, seeds=None, workers: int = 8, tier: str = "i32"):
    """Partitions many graphs of one tier in one call (jet_partition_batch).
    `configs` is one config_t or one per graph.  All graphs on the GPU or
    all on the host.  Returns [(part, edge_cut, latency_ms)], each result
    equal to the single-graph call with the same config and seed."""
    _require_cuda()
    lib = load()
    graphs = list(graphs)
    if not graphs:
        return []
    if isinstance(configs, config_t):
        configs = [configs] * len(graphs)
    seeds = list(seeds) if seeds is not None else [1] * len(graphs)
    on_dev = graphs[0].row.is_cuda
    if any(g.row.is_cuda != on_dev for g in graphs):
        raise JetError(JET_ERR_INVALID, "graphs must all be on the GPU or all on the host")
    keep = []
    arr = (jet_graph_desc * len(graphs))()
    for i, (c, g, sd) in enumerate(zip(configs, graphs, seeds)):
        arr[i] = _desc(tier, c, g, sd, keep)
    if on_dev:
        torch.cuda.synchronize()
    rc = lib.jet_partition_batch(TIER_ID[tier], ctypes.c_int64(len(graphs)), arr,
                                 JET_MEM_DEVICE if on_dev else JET_MEM_HOST, int(workers))
    if rc != JET_OK:
        bad = [i for i in range(len(graphs)) if arr[i].status != JET_OK]
        raise JetError(rc, "batched partition failed for graphs %s: %s" % (bad[:8], arr[bad[0]].error.decode() if bad else ""))
    return [(keep[i][4], int(arr[i].edge_cut), float(arr[i].latency_ms)) for i in range(len(graphs))]


class Server:
    """Request loop (jet_server_*): submit() queues a partition request and
    returns a ticket; requests are admitted oldest first while a worker is
    free and their estimated device footprints fit the byte budget, and run
    concurrently.  wait() returns (part, edge_cut, latency_ms)."""

    def __init__(self, tier: str = "i32", workers: int = 8, mem_budget_bytes: int = 120 << 30, device_memory: bool = True):
        _require_cuda()
        self._lib = load()
        self._lib.jet_server_create.restype = ctypes.c_void_p
        self._lib.jet_server_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int64]
        self._lib.jet_server_submit.restype = ctypes.c_int64
        self._lib.jet_server_submit.argtypes = [ctypes.c_void_p, ctypes.POINTER(jet_graph_desc)]
        self._lib.jet_server_wait.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(jet_graph_desc),
                                              ctypes.c_double]
        self._lib.jet_server_stats_get.argtypes = [ctypes.c_void_p, ctypes.POINTER(jet_server_stats)]
        self._lib.jet_server_destroy.argtypes = [ctypes.c_void_p]
        self.tier = tier
        self.device_memory = device_memory
        self._h = self._lib.jet_server_create(TIER_ID[tier], JET_MEM_DEVICE if device_memory else JET_MEM_HOST,
                                              int(workers), ctypes.c_int64(int(mem_budget_bytes)))
        if not self._h:
            raise JetError(JET_ERR_INVALID, "server creation failed")
        self._keep = {}

    def submit(self, config: config_t, g: CSRGraph, seed: int = 1) -> int:
        if self.device_memory and not g.row.is_cuda:
            raise JetError(JET_ERR_INVALID, "this server takes graphs in GPU memory")
        keep = []
        d = _desc(self.tier, config, g, seed, keep)
        if self.device_memory:
            torch.cuda.current_stream().synchronize()
        t = int(self._lib.jet_server_submit(self._h, ctypes.byref(d)))
        if t < 0:
            raise JetError(-t, "request refused")
        self._keep[t] = keep
        return t

    def wait(self, ticket: int, timeout_ms: float = -1.0):
        out = jet_graph_desc()
        rc = self._lib.jet_server_wait(self._h, ctypes.c_int64(ticket), ctypes.byref(out), ctypes.c_double(timeout_ms))
        if rc == JET_ERR_TIMEOUT:
            raise TimeoutError(ticket)
        _check(rc)
        keep = self._keep.pop(ticket)
        if out.status != JET_OK:
            raise JetError(out.status, "request %d failed: %s" % (ticket, out.error.decode()))
        return keep[0][4], int(out.edge_cut), float(out.latency_ms)

    def stats(self) -> dict:
        st = jet_server_stats()
        _check(self._lib.jet_server_stats_get(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in jet_server_stats._fields_}

    def close(self):
        if self._h:
            self._lib.jet_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def refine_hierarchy(config: config_t, tier: str = "i32", graphs_path: Optional[str] = None,
                     part_path: Optional[str] = None, capacity: Optional[int] = None):
    """Refines a dumped hierarchy (jet_refine_hierarchy, the import_coarse
    app of the reference): returns (part, edge_cut, experiment)."""
    _require_cuda()
    lib = load()
    if capacity is None:
        with open(graphs_path or "coarse_graphs.out", "rb") as f:
            f.read(4)
            capacity = int(np.frombuffer(f.read(8 if tier == "biggest" else 4), dtype=np.int64 if tier == "biggest" else np.int32)[0])
    part = np.empty(max(capacity, 1), dtype=np.int32)
    n = ctypes.c_int64(0)
    cut = ctypes.c_int64(0)
    st = jet_stats_c()
    cfg = config.to_c()
    gp = graphs_path.encode() if graphs_path else None
    pp = part_path.encode() if part_path else None
    _check(lib.jet_refine_hierarchy(TIER_ID[tier], ctypes.byref(cfg), ctypes.c_char_p(gp), ctypes.c_char_p(pp),
                                    part.ctypes.data_as(ctypes.c_void_p), ctypes.c_int64(capacity), ctypes.byref(n),
                                    ctypes.byref(cut), ctypes.byref(st), _stream_ptr()))
    exp = experiment_data()
    exp.fill(st)
    return torch.from_numpy(part[:n.value].copy()), int(cut.value), exp


def assign_lpt(costs, world_size: int):
    """Owner rank of each item: longest-processing-time first onto the least
    loaded rank (ties to the lower rank).  Used to shard independent graphs
    over GPUs with no collective on the data path."""
    import heapq
    world_size = max(1, int(world_size))
    owner = [0] * len(costs)
    heap = [(0, r) for r in range(world_size)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + costs[i], r))
    return owner


def server_footprint(tier: str, n: int, nnz: int, k: int) -> int:
    """Estimated device bytes one request holds while it runs."""
    lib = load()
    lib.jet_server_footprint.restype = ctypes.c_int64
    return int(lib.jet_server_footprint(TIER_ID[tier], ctypes.c_int64(n), ctypes.c_int64(nnz), ctypes.c_int32(k)))


# ------------------------------------------------------------------ components
def _dev_graph(g: CSRGraph) -> CSRGraph:
    if not g.row.is_cuda:
        g = g.to("cuda")
    o, e, w = TIERS[g.tier]
    return CSRGraph(g.n, g.row.to(e).contiguous(), g.adj.to(o).contiguous(), g.val.to(w).contiguous(),
                    g.vw.to(w).contiguous(), g.uniform, g.tier)


def coarsen_map(g: CSRGraph, alg: int, level: int = 1, seed: int = 1, uniform: Optional[bool] = None):
    """One coarsening map; returns (map, nc, initial proposals)."""
    _require_cuda()
    g = _dev_graph(g)
    o = TIERS[g.tier][0]
    m = torch.empty(max(g.n, 1), dtype=o, device=g.row.device)
    hn = torch.empty(max(g.n, 1), dtype=o, device=g.row.device)
    nc = ctypes.c_int64(0)
    u = g.uniform if uniform is None else uniform
    _check(load().jet_coarsen_map(TIER_ID[g.tier], alg, level, ctypes.c_uint64(seed), ctypes.c_int64(g.n),
                                  ctypes.c_int64(g.nnz), _ptr(g.row), _ptr(g.adj), _ptr(g.val), _ptr(g.vw), int(u),
                                  _ptr(m), _ptr(hn), ctypes.byref(nc), _stream_ptr()))
    return m[:g.n], int(nc.value), hn[:g.n]


def contract(g: CSRGraph, cmap: torch.Tensor, nc: int) -> CSRGraph:
    _require_cuda()
    g = _dev_graph(g)
    o, e, w = TIERS[g.tier]
    dev = g.row.device
    crow = torch.empty(nc + 1, dtype=e, device=dev)
    cadj = torch.empty(max(g.nnz, 1), dtype=o, device=dev)
    cval = torch.empty(max(g.nnz, 1), dtype=w, device=dev)
    cvw = torch.empty(max(nc, 1), dtype=w, device=dev)
    cnnz = ctypes.c_int64(0)
    cmap = cmap.to(dev).to(o).contiguous()
    _check(load().jet_contract(TIER_ID[g.tier], ctypes.c_int64(g.n), ctypes.c_int64(g.nnz), _ptr(g.row), _ptr(g.adj),
                               _ptr(g.val), _ptr(g.vw), _ptr(cmap), ctypes.c_int64(nc), _ptr(crow), _ptr(cadj),
                               _ptr(cval), _ptr(cvw), ctypes.byref(cnnz), _stream_ptr()))
    m = int(cnnz.value)
    return CSRGraph(nc, crow, cadj[:m], cval[:m], cvw[:nc], False, g.tier)


def conn_build(g: CSRGraph, part: torch.Tensor, k: int):
    """Connectivity tables: (offsets, entries, values, sizes)."""
    _require_cuda()
    g = _dev_graph(g)
    o, e, w = TIERS[g.tier]
    dev = g.row.device
    off = torch.empty(g.n + 1, dtype=e, device=dev)
    ent = torch.empty(max(g.nnz, 1), dtype=torch.int32, device=dev)
    val = torch.empty(max(g.nnz, 1), dtype=w, device=dev)
    size = torch.empty(max(g.n, 1), dtype=torch.int32, device=dev)
    part = part.to(dev).to(torch.int32).contiguous()
    _check(load().jet_conn_build(TIER_ID[g.tier], ctypes.c_int64(g.n), ctypes.c_int64(g.nnz), _ptr(g.row), _ptr(g.adj),
                                 _ptr(g.val), _ptr(part), int(k), _ptr(off), _ptr(ent), _ptr(val), _ptr(size),
                                 _stream_ptr()))
    c = int(off[-1].item())
    return off, ent[:c], val[:c], size[:g.n]


def refine_iters(g: CSRGraph, part: torch.Tensor, k: int, imb: float, filter_ratio: float, iters: int):
    _require_cuda()
    g = _dev_graph(g)
    o, e, w = TIERS[g.tier]
    dev = g.row.device
    part = part.to(dev).to(torch.int32).clone()
    sizes = torch.empty(k, dtype=w, device=dev)
    cut = ctypes.c_int64(0)
    off = torch.empty(g.n + 1, dtype=e, device=dev)
    ent = torch.empty(max(g.nnz, 1), dtype=torch.int32, device=dev)
    val = torch.empty(max(g.nnz, 1), dtype=w, device=dev)
    size = torch.empty(max(g.n, 1), dtype=torch.int32, device=dev)
    dc = torch.empty(max(g.n, 1), dtype=torch.int32, device=dev)
    moves = (ctypes.c_int64 * max(iters, 1))()
    kinds = (ctypes.c_int32 * max(iters, 1))()
    _check(load().jet_refine_iters(TIER_ID[g.tier], ctypes.c_int64(g.n), ctypes.c_int64(g.nnz), _ptr(g.row),
                                   _ptr(g.adj), _ptr(g.val), _ptr(g.vw), _ptr(part), int(k), ctypes.c_double(imb),
                                   ctypes.c_double(filter_ratio), int(iters), _ptr(sizes), ctypes.byref(cut), _ptr(off),
                                   _ptr(ent), _ptr(val), _ptr(size), _ptr(dc), moves, kinds, _stream_ptr()))
    c = int(off[-1].item())
    return dict(part=part, sizes=sizes, cut=int(cut.value), off=off, ent=ent[:c], val=val[:c], size=size[:g.n],
                dest_cache=dc[:g.n], moves=list(moves)[:iters], kinds=list(kinds)[:iters])


def refine_level(g: CSRGraph, part: torch.Tensor, k: int, imb: float = 1.03, tol: float = 0.999):
    _require_cuda()
    g = _dev_graph(g)
    part = part.to(g.row.device).to(torch.int32).clone()
    cut = ctypes.c_int64(0)
    it = ctypes.c_int32(0)
    _check(load().jet_refine_level(TIER_ID[g.tier], ctypes.c_int64(g.n), ctypes.c_int64(g.nnz), _ptr(g.row),
                                   _ptr(g.adj), _ptr(g.val), _ptr(g.vw), _ptr(part), int(k), ctypes.c_double(imb),
                                   ctypes.c_double(tol), int(g.uniform), ctypes.byref(cut), ctypes.byref(it),
                                   _stream_ptr()))
    return part, int(cut.value), int(it.value)


def pstat(g: CSRGraph, part: torch.Tensor, k: int):
    """[cut, max part cut, comm size, largest, smallest, total] as pstat reports them."""
    _require_cuda()
    g = _dev_graph(g)
    part = part.to(g.row.device).to(torch.int32).contiguous()
    out = (ctypes.c_int64 * 6)()
    _check(load().jet_pstat(TIER_ID[g.tier], ctypes.c_int64(g.n), ctypes.c_int64(g.nnz), _ptr(g.row), _ptr(g.adj),
                            _ptr(g.val), _ptr(g.vw), _ptr(part), int(k), out, _stream_ptr()))
    return list(out)


def pstat_noalloc(g: CSRGraph, part: torch.Tensor, k: int):
    """pstat without any device allocation by the library (jet_pstat_noalloc):
    for callers that record into a stream capture or forbid allocation after
    start-up.  Same six numbers as ``pstat``; k <= 16384.  The graph and part
    must already be on the device."""
    _require_cuda()
    if not (g.row.is_cuda and part.is_cuda):
        raise JetError(JET_ERR_INVALID, "pstat_noalloc takes device tensors")
    out = (ctypes.c_int64 * 6)()
    _check(load().jet_pstat_noalloc(TIER_ID[g.tier], ctypes.c_int64(g.n), ctypes.c_int64(g.nnz), _ptr(g.row),
                                    _ptr(g.adj), _ptr(g.val), _ptr(g.vw), _ptr(part), int(k), out, _stream_ptr()))
    return list(out)


def project(cmap: torch.Tensor, coarse_part: torch.Tensor, tier: str = "i32") -> torch.Tensor:
    _require_cuda()
    o = TIERS[tier][0]
    cmap = cmap.to(o).contiguous()
    coarse_part = coarse_part.to(torch.int32).contiguous()
    fine = torch.empty(cmap.numel(), dtype=torch.int32, device=cmap.device)
    _check(load().jet_project(TIER_ID[tier], ctypes.c_int64(cmap.numel()), _ptr(cmap), _ptr(coarse_part), _ptr(fine),
                              _stream_ptr()))
    return fine


def launch_count() -> int:
    """Kernels launched by the library so far in this process."""
    return int(load().jet_launch_count())


def set_refine_drivers(mask: int) -> int:
    """Allowed level-loop drivers (DRIVER_* bits); returns the previous mask.
    Every driver yields the same partition, only the speed differs."""
    return int(load().jet_set_refine_drivers(int(mask)))


def prof_enable(on: bool = True):
    _check(load().jet_prof_enable(int(on)))


PROF_CLASSES = ["conn_build", "lp_select", "afterburn", "update", "contract", "coarsen_map", "conn_build_finest",
                "reb_select", "reb_sort", "reb_evict", "apply", "update_large", "cut_after"]


def prof_read():
    """Per kernel class: summed event time (ms), algorithmic bytes, launches."""
    nk = len(PROF_CLASSES)
    ms = (ctypes.c_double * nk)()
    by = (ctypes.c_double * nk)()
    ln = (ctypes.c_int64 * nk)()
    _check(load().jet_prof_read(ms, by, ln))
    names = PROF_CLASSES
    return {nm: dict(ms=ms[i], bytes=by[i], launches=ln[i]) for i, nm in enumerate(names)}
