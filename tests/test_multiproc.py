"""The multi-GPU bench path on CPU: two gloo ranks shard the batched config
by longest-processing-time first (disjoint, complete, balanced) and reduce
their timed-region lengths to the max over ranks, as bench.py does."""
import importlib.util
import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT, load_pkg


def _bench():
    spec = importlib.util.spec_from_file_location("jet_bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        jet = load_pkg()
        bench = _bench()
        specs = bench.batched_specs(512)
        owner = jet.assign_lpt([n for n, _ in specs], world)
        mine = [i for i in range(len(specs)) if owner[i] == rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        t_max = bench.max_over_ranks(1.5 + rank, world, dist, torch.device("cpu"))
        load = sum(specs[i][0] for i in mine)
        loads = [None] * world
        dist.all_gather_object(loads, load)
        if rank == 0:
            out.put((gathered, t_max, loads))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_and_max_timing():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, t_max, loads = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    allitems = sorted(gathered[0] + gathered[1])
    assert allitems == list(range(512))              # complete
    assert not set(gathered[0]) & set(gathered[1])   # disjoint
    assert t_max == 2.5                              # max over ranks
    assert max(loads) <= 1.01 * min(loads) + 2e5     # LPT balance within one item


def test_assign_lpt_single_rank():
    jet = load_pkg()
    assert jet.assign_lpt([5, 3, 9], 1) == [0, 0, 0]
    assert jet.assign_lpt([5, 3, 9, 1], 2) == [1, 1, 0, 1]  # 9 | 5 + 3 + 1
