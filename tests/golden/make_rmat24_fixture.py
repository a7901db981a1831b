"""Writes tests/golden/rmat24_k256_oracle.json: the CPU oracle's partition of
the power-law config -- R-MAT 2^24 (edge factor 8, a = 0.57, b = c = 0.19,
symmetrised, de-duplicated, unit weights, seed 1, generated on the host),
int64 offsets and weights, 2-hop matching, k = 256, imbalance 1.10,
coarsening seed 1 -- as its cut and a SHA-256 of the part array, with
SHA-256 digests of the graph's arrays so that a GPU run can check that it
partitioned the same graph.  The oracle takes about 12 minutes on one host
thread, too long for the benchmark; the fixture lets the GPU test compare
at full size without it.

    python tests/golden/make_rmat24_fixture.py
"""
import hashlib
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def digest(a):
    return hashlib.sha256(a.tobytes()).hexdigest()


def main():
    from conftest import load_pkg
    import oracle
    jet = load_pkg()
    t = time.time()
    g = jet.graphs.rmat(24, 8, seed=1, tier="big", device="cpu")
    og = oracle.G.from_csr(g)
    gen_s = time.time() - t
    t = time.time()
    part, cut, st = oracle.partition(og, 256, alg=0, imb=1.10, seed=1)
    out = {"graph": "R-MAT 2^24, edge factor 8, a=0.57 b=c=0.19, symmetrised, de-duplicated, unit weights, seed 1, "
                    "generated on the host (jet.graphs.rmat(24, 8, seed=1, tier='big', device='cpu'))",
           "config": {"k": 256, "coarsening_alg": 0, "max_imb_ratio": 1.10, "seed": 1, "tier": "big"},
           "n": int(og.n), "nnz": int(og.row[-1]),
           "row_sha256": digest(og.row), "adj_sha256": digest(og.adj),
           "cut": int(cut), "part_sha256": digest(part), "imbalance": float(st.imb), "levels": int(st.levels),
           "oracle_seconds": time.time() - t, "generation_seconds": gen_s}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rmat24_k256_oracle.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
