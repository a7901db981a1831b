"""Failure handling, driven without faulting, trapping or hanging a GPU:

  * a Metis failure injected on the host surfaces as JET_ERR_METIS from the
    partition call (the reference exits the process there,
    src/initial_partition.hpp:106-109), for a single call and for a request
    in the server's mix, and the library keeps working afterwards;
  * the cooperative level driver's grid barrier, with one block that never
    arrives and a short poll limit, gives up, flags the timeout and returns:
    the call reports JET_ERR_TIMEOUT and the context stays usable;
  * the connectivity-table insert detects a full table (more distinct parts
    than slots) through its probe bound and reports JET_ERR_OVERFLOW.
Host-side failures (corrupt CSR, oversize admission, wait timeouts) are
tested in test_gpu_parity.py and test_batch.py."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_injected_metis_failure_returns_error(jet, graphs, orc):
    lib = jet.load()
    g = graphs.grid2d(40, 30, weighted=True, seed=1).to("cuda")
    cfg = jet.config_t(coarsening_alg=1, num_parts=8)
    assert lib.jet_test_inject_metis_failures(1) == 0
    with pytest.raises(jet.JetError) as e:
        jet.partition(cfg, g, seed=1)
    assert e.value.code == 3  # JET_ERR_METIS
    assert "Metis" in str(e.value)
    # the injection is used up; the library still partitions, bit-exact
    part, cut, _ = jet.partition(cfg, g, seed=1)
    want, wcut, _ = orc.partition(orc.G.from_csr(g.to("cpu")), 8, alg=1, seed=1)
    assert cut == wcut and np.array_equal(part.cpu().numpy(), want)


def test_injected_metis_failure_in_server_mix(jet, graphs):
    lib = jet.load()
    gs = [graphs.grid2d(30 + i, 20, weighted=True, seed=i).to("cuda") for i in range(4)]
    cfg = jet.config_t(coarsening_alg=1, num_parts=4)
    alone = [jet.partition(cfg, g, seed=1)[1] for g in gs]
    srv = jet.Server("i32", workers=2, mem_budget_bytes=1 << 30)
    try:
        lib.jet_test_inject_metis_failures(1)
        tickets = [srv.submit(cfg, g, seed=1) for g in gs]
        failed, ok = 0, 0
        for t, want in zip(tickets, alone):
            try:
                _, cut, _ = srv.wait(t)
                assert cut == want
                ok += 1
            except jet.JetError as e:
                assert e.code == 3
                failed += 1
        assert failed == 1 and ok == 3
    finally:
        lib.jet_test_inject_metis_failures(0)
        srv.close()


def test_grid_barrier_timeout_returns_error(jet, graphs):
    lib = jet.load()
    passed = ctypes.c_int(0)
    # everyone arrives: every barrier completes
    assert lib.jet_test_grid_barrier(16, -1, 20, 50, ctypes.byref(passed)) == 0
    assert passed.value == 16 * 50
    # block 3 never arrives: the others' waits run out after 2^12 polls
    rc = lib.jet_test_grid_barrier(16, 3, 12, 5, ctypes.byref(passed))
    assert rc == 6  # JET_ERR_TIMEOUT
    assert passed.value == 0
    assert b"gave up" in lib.jet_last_error()
    # the context is still usable
    g = graphs.grid2d(20, 20, weighted=True, seed=2).to("cuda")
    part, cut, _ = jet.partition(jet.config_t(coarsening_alg=1, num_parts=4), g, seed=1)
    assert cut > 0 and int(part.max()) == 3


@pytest.mark.parametrize("cap,k,nparts,want", [(8, 64, 8, 0), (16, 64, 9, 0), (4, 64, 9, 5), (64, 64, 64, 0),
                                               (31, 256, 40, 5)])
def test_table_overflow_detected(jet, cap, k, nparts, want):
    claimed = ctypes.c_int(0)
    rc = jet.load().jet_test_table_overflow(cap, k, nparts, ctypes.byref(claimed))
    assert rc == want  # 5 = JET_ERR_OVERFLOW
    assert claimed.value == min(cap, nparts)
    torch.cuda.synchronize()
