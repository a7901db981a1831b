"""The library's METIS text reader (jet_read_metis) against the Python writer
and against the reference's own reader (app/io.hpp:99-217, built under
oracle/_ref) on generated and hand-written files.  Host-only: no GPU."""
import os

import numpy as np
import pytest

CASES = {
    # leading comments, blank line for an isolated vertex, no final newline
    "comments_isolated": "% a comment\n% another\n4 2\n2 3\n1\n1\n\n",
    "no_final_newline": "3 2\n2\n1 3\n2",
    "weighted": "3 2 1\n2 5\n1 5 3 7\n2 7\n",
    "tabs_and_spaces": "3 2\n\t2   \n1\t3\n 2\n",
    # a comment inside the body ends no row: its line joins the next one
    "inline_comment": "3 2\n2 % trailing note\n\n1 3\n2\n",
    "extra_trailing_newlines": "2 1\n2\n1\n\n\n\n",
}
BAD = {
    "vertex_weights": "2 1 10\n1 2\n1 1\n",
    "ncon": "2 1 0 2\n2\n1\n",
    "too_few_nonzeros": "3 2\n2\n1\n2\n",
    "too_few_rows": "3 1\n2\n1\n",
}


def write(tmp_path, name, text):
    p = tmp_path / (name + ".graph")
    p.write_bytes(text.encode())
    return str(p)


@pytest.mark.parametrize("name", sorted(CASES))
def test_reader_matches_reference_reader(tmp_path, graphs, ref, name):
    path = write(tmp_path, name, CASES[name])
    want = ref.load_metis(path, 64, 256)
    assert want is not None
    g = graphs.read_metis(path)
    assert np.array_equal(g.row.numpy(), want[0])
    assert np.array_equal(g.adj.numpy(), want[1])
    assert np.array_equal(g.val.numpy(), want[2])
    assert g.uniform == want[3]


@pytest.mark.parametrize("name", sorted(BAD))
def test_reader_rejects_what_the_reference_rejects(tmp_path, graphs, ref, jet, name):
    path = write(tmp_path, name, BAD[name])
    assert ref.load_metis(path, 64, 256) is None
    with pytest.raises(jet.JetError) as e:
        graphs.read_metis(path)
    assert e.value.code == 1


@pytest.mark.parametrize("kind", ["grid_unit", "grid3d_weighted", "rgg", "rmat"])
@pytest.mark.parametrize("threads", [1, 7])
def test_round_trip(tmp_path, graphs, ref, kind, threads):
    g = {"grid_unit": lambda: graphs.grid2d(70, 40),
         "grid3d_weighted": lambda: graphs.grid3d(60, 40, 25, weighted=True, seed=2),
         "rgg": lambda: graphs.rgg(30000, 10.0, seed=4),
         "rmat": lambda: graphs.rmat(14, 8, seed=2, tier="i32")}[kind]()
    path = str(tmp_path / "g.graph")
    graphs.write_metis(g, path)
    assert os.path.getsize(path) > (1 << 20) or kind == "grid_unit"  # big enough for several chunks
    for tier in ("i32", "big", "biggest"):
        h = graphs.read_metis(path, tier=tier, threads=threads)
        assert h.n == g.n and h.uniform == g.uniform
        assert np.array_equal(h.row.numpy(), g.row.numpy())
        assert np.array_equal(h.adj.numpy(), g.adj.numpy())
        assert np.array_equal(h.val.numpy(), g.val.numpy())
        assert np.array_equal(h.vw.numpy(), np.ones(g.n))
    want = ref.load_metis(path, g.n, g.nnz)
    assert np.array_equal(want[1], g.adj.numpy()) and np.array_equal(want[2], g.val.numpy())
