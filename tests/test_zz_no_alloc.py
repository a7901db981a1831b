"""jet_pstat_noalloc: partition statistics for callers that cannot let the
library allocate device memory (services that reserve the GPU's memory up
front and forbid later allocation).  Its scratch is a fixed device array
shared by all calls, so this checks, through the C ABI, that two calls in a
row each return exactly what jet_pstat and the CPU oracle return -- the
second call must not see leftovers of the first -- and that a warm call
leaves the device's free memory unchanged.  This file is collected last so a
run that stops at the first failure has run everything else already."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TIER = {"i32": 0, "big": 1, "biggest": 2}


def noalloc(jet, g, part, k):
    out = (ctypes.c_int64 * 6)(*([-7] * 6))
    rc = jet.load().jet_pstat_noalloc(TIER[g.tier], ctypes.c_int64(g.n), ctypes.c_int64(g.nnz),
                                      ctypes.c_void_p(g.row.data_ptr()), ctypes.c_void_p(g.adj.data_ptr()),
                                      ctypes.c_void_p(g.val.data_ptr()), ctypes.c_void_p(g.vw.data_ptr()),
                                      ctypes.c_void_p(part.data_ptr()), int(k), out,
                                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc, list(out)


def reference_pstat(jet, g, part, k):
    out = (ctypes.c_int64 * 6)()
    rc = jet.load().jet_pstat(TIER[g.tier], ctypes.c_int64(g.n), ctypes.c_int64(g.nnz),
                              ctypes.c_void_p(g.row.data_ptr()), ctypes.c_void_p(g.adj.data_ptr()),
                              ctypes.c_void_p(g.val.data_ptr()), ctypes.c_void_p(g.vw.data_ptr()),
                              ctypes.c_void_p(part.data_ptr()), int(k), out,
                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    return list(out)


def graphs_for(graphs):
    yield graphs.grid2d(60, 50, weighted=True, seed=2).as_tier("i32"), 8
    yield graphs.rmat(12, 8, seed=3, tier="big"), 700
    yield graphs.rgg(4000, 10.0, seed=5).as_tier("biggest"), 64


def test_noalloc_matches_pstat_twice(jet, graphs, orc):
    for g, k in graphs_for(graphs):
        gd = g.to("cuda")
        rng = np.random.default_rng(k)
        part_h = rng.integers(0, k, g.n).astype(np.int32)
        part = torch.from_numpy(part_h).cuda()
        want = reference_pstat(jet, gd, part, k)
        assert want == orc.pstat(orc.G.from_csr(g), part_h, k).tolist()
        for _ in range(2):
            rc, got = noalloc(jet, gd, part, k)
            assert rc == 0
            assert got == want, (g.tier, k, got, want)


def test_noalloc_warm_call_allocates_nothing(jet, graphs):
    g = graphs.rgg(20000, 10.0, seed=7).to("cuda")
    part = torch.from_numpy(np.random.default_rng(1).integers(0, 32, g.n).astype(np.int32)).cuda()
    rc, first = noalloc(jet, g, part, 32)  # loads the module and looks up the array on this device
    assert rc == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        rc, got = noalloc(jet, g, part, 32)
        assert rc == 0 and got == first
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_out_of_range(jet, graphs):
    g = graphs.grid2d(20, 20).to("cuda")
    part = torch.zeros(g.n, dtype=torch.int32, device="cuda")
    rc, _ = noalloc(jet, g, part, 16385)  # more parts than the scratch array serves
    assert rc == 1
    bad = part.clone()
    bad[5] = 9
    rc, _ = noalloc(jet, g, bad, 4)  # a part id outside [0, k)
    assert rc == 1
    assert b"outside" in jet.load().jet_last_error()
    part[::2] = 1
    rc, got = noalloc(jet, g, part, 2)  # the shared scratch holds no leftovers of the failed call
    assert rc == 0 and got == reference_pstat(jet, g, part, 2)
    out = (ctypes.c_int64 * 6)()
    rc = jet.load().jet_pstat_noalloc(0, ctypes.c_int64(g.n), ctypes.c_int64(g.nnz), ctypes.c_void_p(g.row.data_ptr()),
                                      None, None, ctypes.c_void_p(g.vw.data_ptr()), ctypes.c_void_p(part.data_ptr()),
                                      2, out, None)
    assert rc == 1  # entries / values missing while nnz > 0
