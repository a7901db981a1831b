"""The C-ABI library loads and exports every function declared in
include/jet_b200.h (no compute call: runs without a GPU)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "jet_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(jet_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for want in ("jet_partition_i32", "jet_partition_big", "jet_partition_biggest", "jet_contract", "jet_conn_build"):
        assert want in names


def test_library_exports_every_declared_symbol(jet):
    lib = jet.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert b"sm_100a" in lib.jet_version()


def test_python_mirror_lists_exports(jet):
    assert sorted(jet.EXPORTED_SYMBOLS) == sorted(n for n in declared_functions() if n in jet.EXPORTED_SYMBOLS)
    for name in declared_functions():
        assert name in jet.EXPORTED_SYMBOLS, name


def test_config_mirror_defaults(jet):
    c = jet.config_t()
    # header/jet_config.h:43-52
    assert (c.coarsening_alg, c.num_iter, c.max_imb_ratio, c.num_parts, c.refine_tolerance) == (0, 1, 1.03, 2, 0.999)
    assert not c.dump_coarse and not c.verbose and not c.ultra_settings
    cc = c.to_c()
    assert ctypes.sizeof(cc) == 48


def test_no_cuda_raises(jet, graphs):
    import torch
    if torch.cuda.is_available():
        return
    import pytest
    with pytest.raises(jet.JetError):
        jet.partition(jet.config_t(num_parts=2), graphs.grid2d(4, 4))
