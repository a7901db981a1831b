"""include/jet.h, the C++ drop-in for the reference's jet.h, compiles against
the library (CPU) and partitions through it (GPU)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build_driver(tmp_path, jet):
    jet.load()
    exe = str(tmp_path / "driver_test")
    libdir = os.path.dirname(jet.library_path())
    cmd = ["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "cpp", "driver_test.cpp"), "-L" + libdir, "-ljetb200",
           "-L" + os.path.join(CUDA, "lib64"), "-lcudart", "-Wl,-rpath," + libdir, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_header_compiles_and_links(tmp_path, jet):
    assert os.path.exists(build_driver(tmp_path, jet))


@pytest.mark.gpu
def test_header_partitions(tmp_path, jet):
    exe = build_driver(tmp_path, jet)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = {ln.split()[0]: ln.split()[1:] for ln in r.stdout.splitlines()}
    host_cut, maxp, levels = map(int, lines["host"])
    assert host_cut > 0 and maxp == 15 and levels >= 2
    dev_cut, n = map(int, lines["device"])
    assert n == 96 * 80 and dev_cut == host_cut  # same seed, same graph, deterministic path
    assert lines["error"] == ["1"]
