"""Hierarchy dump (config.dump_coarse) and import (jet_refine_hierarchy):
the files follow the reference's binary layout, their levels are the
oracle's contractions of each other, and refining the imported hierarchy
gives back the partition of the run that wrote it."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TYPES = {"i32": (np.int32, np.int32, np.int32), "big": (np.int32, np.int64, np.int64),
         "biggest": (np.int64, np.int64, np.int64)}


def read_hierarchy(path, tier):
    o, e, w = TYPES[tier]
    buf = open(path, "rb").read()
    pos = 0

    def take(dtype, count):
        nonlocal pos
        a = np.frombuffer(buf, dtype=dtype, count=count, offset=pos)
        pos += a.nbytes
        return a

    size = int(take(np.int32, 1)[0])
    levels, prev_n = [], 0
    for lv in range(size):
        n = int(take(o, 1)[0])
        m = int(take(e, 1)[0])
        row, adj, val, vw = take(e, n + 1), take(o, m), take(w, m), take(w, n)
        mp = take(o, prev_n) if lv > 0 else None
        levels.append((n, m, row, adj, val, vw, mp))
        prev_n = n
    assert pos == len(buf)
    return levels


@pytest.mark.parametrize("tier,kind", [("i32", "grid2d"), ("big", "rgg"), ("biggest", "grid2d")])
def test_dump_then_import(jet, graphs, orc, tier, kind, tmp_path, monkeypatch):
    g = (graphs.grid2d(120, 100, weighted=True, seed=4) if kind == "grid2d" else graphs.rgg(9000, 9.0, seed=6)).as_tier(tier)
    fn = {"i32": jet.partition, "big": jet.partition_big, "biggest": jet.partition_biggest}[tier]
    cfg = jet.config_t(coarsening_alg=1, num_parts=16, max_imb_ratio=1.03)
    want_part, want_cut, _ = fn(cfg, g.to("cuda"), seed=5)
    monkeypatch.chdir(tmp_path)
    dcfg = jet.config_t(coarsening_alg=1, num_parts=16, max_imb_ratio=1.03, dump_coarse=True)
    part, cut, _ = fn(dcfg, g.to("cuda"), seed=5)
    assert cut == want_cut and torch.equal(part, want_part)  # dumping changes nothing
    assert os.path.exists("coarse_graphs.out") and os.path.exists("coarse_part.out")
    levels = read_hierarchy("coarse_graphs.out", tier)
    n0, m0, row, adj, val, vw, _ = levels[0]
    assert n0 == g.n and np.array_equal(row, g.row.numpy()) and np.array_equal(adj, g.adj.numpy())
    assert np.array_equal(val, g.val.numpy()) and np.array_equal(vw, g.vw.numpy())
    for fine, coarse in zip(levels, levels[1:]):
        n, m, crow, cadj, cval, cvw, mp = coarse
        assert len(mp) == fine[0] and mp.min() >= 0 and mp.max() == n - 1
        og = orc.G(fine[2], fine[3], fine[4], fine[5])
        c = orc.contract(og, mp.astype(np.int64 if TYPES[tier][0] == np.int64 else np.int32), n)
        assert np.array_equal(c.row, crow) and np.array_equal(c.adj, cadj)
        assert np.array_equal(c.val, cval) and np.array_equal(c.vw, cvw)
    cp = np.fromfile("coarse_part.out", dtype=np.int32)
    assert len(cp) == levels[-1][0] and cp.min() >= 0 and cp.max() < 16
    got_part, got_cut, exp = jet.refine_hierarchy(cfg, tier)
    assert got_cut == want_cut
    assert np.array_equal(got_part.numpy(), want_part.cpu().numpy())
    assert len(exp.coarseLevels) == len(levels)


def test_import_rejects_malformed(jet, tmp_path):
    p = tmp_path / "bad.out"
    p.write_bytes(np.array([3, 10, 5], dtype=np.int32).tobytes())  # claims 3 levels, truncated
    q = tmp_path / "part.out"
    q.write_bytes(np.zeros(10, dtype=np.int32).tobytes())
    with pytest.raises(jet.JetError):
        jet.refine_hierarchy(jet.config_t(num_parts=4), "i32", str(p), str(q), capacity=10)
