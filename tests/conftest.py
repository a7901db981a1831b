import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "jet-partitioner-official-fork_b200")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def load_pkg():
    """Imports the package directory (its name is not a Python identifier)."""
    if "jet_b200" in sys.modules:
        return sys.modules["jet_b200"]
    spec = importlib.util.spec_from_file_location("jet_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["jet_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def jet():
    return load_pkg()


@pytest.fixture(scope="session")
def graphs(jet):
    return jet.graphs


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle


def sorted_rows(row, adj, val):
    """CSR with each row sorted by neighbour id (for order-free comparison)."""
    row = np.asarray(row, dtype=np.int64)
    adj = np.asarray(adj)
    val = np.asarray(val)
    n = len(row) - 1
    rid = np.repeat(np.arange(n), np.diff(row))
    order = np.lexsort((adj, rid))
    return adj[order], val[order]


def table_multisets(off, ent, val, size):
    """Per-vertex sorted list of (part, weight) for valid slots."""
    off = np.asarray(off, dtype=np.int64)
    out = []
    for i in range(len(off) - 1):
        s = off[i]
        e = ent[s:s + size[i]]
        v = val[s:s + size[i]]
        keep = e >= 0
        out.append(sorted(zip(e[keep].tolist(), v[keep].tolist())))
    return out


@pytest.fixture(scope="session")
def ref():
    """The reference's own CPU code (oracle/_ref); tests using it skip when it
    is neither built nor buildable here."""
    import ref as ref_mod
    if not ref_mod.available():
        pytest.skip("reference build unavailable")
    ref_mod.lib()
    return ref_mod
