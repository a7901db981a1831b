"""Model check of the rebalance eviction queue, on the CPU.

The CUDA rebalance tail decides evictions without sorting every candidate
(csrc/refine.cuh, d_reb_classify / d_reb_ordered).  A candidate's score is
its bucket's offset inside its part's bucket range plus the weight of the
bucket's candidates before it in vertex order ("within"); it leaves while
the score is below its part's excess (get_evictions,
src/jet_refiner.hpp:392-409).  With positive weights a bucket whose offset
reaches the excess keeps every candidate and (weak) a bucket that ends below
it loses every one, so only the straddling buckets (strong: also every
evicted bucket, whose scores feed the destination draws) need the order.

This test restates both procedures in numpy on random bucket assignments and
checks that they evict the same vertices with the same scores and part
adjustments.  It checks the argument the kernels rest on; the kernels
themselves are compared with the oracle in tests/test_gpu_parity.py.
"""
import numpy as np
import pytest

MAX_BUCKETS = 50


def _random_state(rng, strong):
    k = int(rng.integers(2, 12))
    sections = int(rng.integers(1, 4))
    width = MAX_BUCKETS * sections
    tmb = MAX_BUCKETS * k * sections
    n = int(rng.integers(1, 400))
    part = rng.integers(0, k, n)
    w = rng.integers(1, 12, n)
    # candidates: a random subset, bucket type skewed towards a few values
    cand = rng.random(n) < 0.7
    gt = np.minimum(rng.geometric(0.25, n) - 1, MAX_BUCKETS - 1)
    sec = np.arange(n) % sections
    off = 1 if strong else 0
    gid = np.where(cand, (MAX_BUCKETS * part + gt) * sections + sec + off, -1)
    buckets = np.zeros(tmb + 1 + width, dtype=np.int64)
    np.add.at(buckets, gid[cand], w[cand])
    boff = np.concatenate([[0], np.cumsum(buckets[:tmb + 1])])[:tmb + 1]
    sizes = np.bincount(part, weights=w, minlength=k).astype(np.int64)
    size_max = int(max(1, np.median(sizes) * rng.uniform(0.6, 1.1)))
    return dict(k=k, width=width, tmb=tmb, n=n, part=part, w=w, gid=gid, buckets=buckets, boff=boff, sizes=sizes,
                size_max=size_max)


def _full_sort(st, strong):
    """sort_candidates + d_evict_sorted: every candidate in (bucket, vertex) order."""
    order = sorted((int(b), i) for i, b in enumerate(st["gid"]) if b >= 0)
    taken, score, adjust = set(), {}, {}
    seen = {}
    for b, i in order:
        within = seen.get(b, 0)
        seen[b] = within + int(st["w"][i])
        p = int(st["part"][i])
        base = int(st["boff"][b]) - int(st["boff"][p * st["width"]])
        limit = int(st["sizes"][p]) - st["size_max"]
        s = within + base
        if s < limit:
            taken.add(i)
            if strong:
                score[i] = within
                if s + int(st["w"][i]) >= limit:
                    adjust[p] = s + int(st["w"][i])
    return taken, score, adjust


def _queue(st, strong):
    """d_reb_classify + d_reb_ordered."""
    taken, queued = set(), []
    for i, b in enumerate(st["gid"]):
        if b < 0:
            continue
        p = int(st["part"][i])
        base = int(st["boff"][b]) - int(st["boff"][p * st["width"]])
        limit = int(st["sizes"][p]) - st["size_max"]
        if base >= limit:
            continue
        if not strong and base + int(st["buckets"][b]) < limit:
            taken.add(i)
        else:
            queued.append(i)
    score, adjust = {}, {}
    keys = sorted((int(st["gid"][i]), i) for i in queued)
    run_b, run = None, 0
    for b, i in keys:
        if b != run_b:
            run_b, run = b, 0
        within = run
        run += int(st["w"][i])
        p = int(st["part"][i])
        s = within + int(st["boff"][b]) - int(st["boff"][p * st["width"]])
        limit = int(st["sizes"][p]) - st["size_max"]
        if s < limit:
            taken.add(i)
            if strong:
                score[i] = within
                if s + int(st["w"][i]) >= limit:
                    adjust[p] = s + int(st["w"][i])
    return taken, score, adjust, len(queued)


@pytest.mark.parametrize("strong", [False, True], ids=["weak", "strong"])
def test_queue_evicts_what_the_full_sort_evicts(strong):
    rng = np.random.default_rng(7 + strong)
    queued_total = cand_total = 0
    for _ in range(400):
        st = _random_state(rng, strong)
        want = _full_sort(st, strong)
        got = _queue(st, strong)
        assert got[0] == want[0]
        assert got[1] == want[1]
        assert got[2] == want[2]
        queued_total += got[3]
        cand_total += int((st["gid"] >= 0).sum())
    # the queue is a part of the candidates, not all of them
    assert queued_total < cand_total
