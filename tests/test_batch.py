"""Batched and served partitioning: every result equals the single-graph
call with the same config and seed (bit for bit), alone or in a mix, and
admission respects the memory budget."""
import time

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def host(t):
    return t.detach().cpu().numpy()


def mixed_graphs(graphs, tier):
    gs = [graphs.grid2d(60 + 13 * i, 40 + 7 * i, weighted=True, seed=i) for i in range(4)]
    gs += [graphs.rgg(2000 + 1500 * i, 8.0 + i, seed=10 + i) for i in range(4)]
    gs += [graphs.rmat(10 + (i % 2), 8, seed=20 + i, tier=tier) for i in range(3)]
    gs += [graphs.grid3d(20, 18, 16, weighted=True, seed=30)]
    return [g.as_tier(tier) for g in gs]


def single(jet, tier, cfg, g, seed):
    fn = {"i32": jet.partition, "big": jet.partition_big, "biggest": jet.partition_biggest}[tier]
    part, cut, _ = fn(cfg, g, seed=seed)
    return host(part), cut


@pytest.mark.parametrize("tier", ["i32", "big"])
@pytest.mark.parametrize("where", ["device", "host"])
def test_batch_equals_single(jet, graphs, tier, where):
    gs = mixed_graphs(graphs, tier)
    ks = [8, 16, 32, 64]
    cfgs = [jet.config_t(coarsening_alg=(i % 3), num_parts=ks[i % 4], max_imb_ratio=1.03 if i % 3 else 1.10)
            for i in range(len(gs))]
    seeds = [100 + i for i in range(len(gs))]
    dev = [g.to("cuda") for g in gs]
    want = [single(jet, tier, c, g, s) for c, g, s in zip(cfgs, dev, seeds)]
    inp = dev if where == "device" else [g.to("cpu") for g in gs]
    got = jet.partition_batch(cfgs, inp, seeds, workers=6, tier=tier)
    for (wp, wc), (gp, gc, lat) in zip(want, got):
        assert gc == wc
        assert np.array_equal(host(gp), wp)
        assert lat > 0


def test_server_mix_equals_alone(jet, graphs):
    """Requests arrive while others run; each result equals the graph
    partitioned alone."""
    gs = [g.to("cuda") for g in mixed_graphs(graphs, "i32")]
    cfgs = [jet.config_t(coarsening_alg=1, num_parts=[16, 32, 64][i % 3]) for i in range(len(gs))]
    want = [single(jet, "i32", c, g, 7 + i) for i, (c, g) in enumerate(zip(cfgs, gs))]
    srv = jet.Server("i32", workers=4, mem_budget_bytes=8 << 30)
    try:
        tickets = []
        for i, (c, g) in enumerate(zip(cfgs, gs)):
            tickets.append(srv.submit(c, g, seed=7 + i))
            if i % 3 == 2:
                time.sleep(0.01)  # later requests arrive while earlier ones are on the GPU
        got = [srv.wait(t) for t in tickets]
        st = srv.stats()
    finally:
        srv.close()
    for (wp, wc), (gp, gc, lat) in zip(want, got):
        assert gc == wc
        assert np.array_equal(host(gp), wp)
    assert st["completed"] == len(gs) and st["failed"] == 0
    assert st["peak_concurrent"] >= 2


def test_server_budget_and_refusal(jet, graphs):
    gs = [graphs.grid2d(120, 100, weighted=True, seed=i).to("cuda") for i in range(6)]
    fp = jet.server_footprint("i32", gs[0].n, gs[0].nnz, 16)
    budget = int(fp * 2.5)  # at most two of these at once
    srv = jet.Server("i32", workers=6, mem_budget_bytes=budget)
    try:
        cfg = jet.config_t(coarsening_alg=1, num_parts=16)
        ts = [srv.submit(cfg, g, seed=3) for g in gs]
        res = [srv.wait(t) for t in ts]
        big = graphs.grid2d(600, 600).to("cuda")
        with pytest.raises(jet.JetError):
            srv.submit(cfg, big, seed=1)  # its footprint alone exceeds the budget
        st = srv.stats()
    finally:
        srv.close()
    assert st["peak_footprint_bytes"] <= budget
    assert st["peak_concurrent"] <= 2
    assert st["refused"] == 1
    want = single(jet, "i32", jet.config_t(coarsening_alg=1, num_parts=16), gs[0], 3)
    assert res[0][1] == want[1] and np.array_equal(host(res[0][0]), want[0])


def test_server_wait_timeout_then_result(jet, graphs):
    g = graphs.grid2d(200, 200, weighted=True, seed=1).to("cuda")
    srv = jet.Server("i32", workers=1, mem_budget_bytes=8 << 30)
    try:
        t = srv.submit(jet.config_t(coarsening_alg=1, num_parts=8), g, seed=2)
        try:
            srv.wait(t, timeout_ms=0.0)
        except TimeoutError:
            pass
        part, cut, lat = srv.wait(t)
    finally:
        srv.close()
    assert cut == single(jet, "i32", jet.config_t(coarsening_alg=1, num_parts=8), g, 2)[1]
