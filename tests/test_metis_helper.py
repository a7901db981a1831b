"""The Metis helper process (used for concurrent coarsest-graph calls in the
batched and served modes) returns exactly what an in-process call returns."""
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import PKG_DIR

HELPER = os.path.join(PKG_DIR, "jet_metis_helper")


def call_helper(proc, row, adj, vw, ew, k, ub):
    n, m = len(row) - 1, len(adj)
    msg = struct.pack("<qqqf", n, m, k, ub)
    for a in (row, adj, vw, ew):
        msg += np.asarray(a, dtype=np.int64).tobytes()
    proc.stdin.write(msg)
    proc.stdin.flush()
    status, obj = struct.unpack("<qq", proc.stdout.read(16))
    part = np.frombuffer(proc.stdout.read(8 * n), dtype=np.int64)
    return status, obj, part


@pytest.mark.skipif(not os.path.exists(HELPER), reason="library not built")
def test_helper_matches_in_process_metis(jet, graphs, orc):
    proc = subprocess.Popen([HELPER], stdin=subprocess.PIPE, stdout=subprocess.PIPE)
    try:
        for seed, k in [(1, 8), (2, 16), (3, 64)]:
            g = graphs.rgg(1500 + 300 * seed, 9.0, seed=seed)
            og = orc.G.from_csr(g)
            want = orc.metis(og, k, 1.03)
            status, obj, got = call_helper(proc, og.row, og.adj, og.vw, og.val, k, 1.03)
            assert status == 1  # METIS_OK
            assert np.array_equal(got.astype(np.int32), want)
    finally:
        proc.stdin.close()
        proc.wait(timeout=10)
    assert proc.returncode == 0
