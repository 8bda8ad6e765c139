"""C++ host side: the header-only KernelBVHController shim (include/gi/gi_controller.hpp)
and the pose-sweep harness tests/cpp/run_suite.cpp built on it."""
import csv
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gpu-cubql-intersector-standalone_b200")
BUILD = os.path.join(ROOT, "tests", "cpp", "_build")
SRC = os.path.join(ROOT, "tests", "cpp", "run_suite.cpp")
CUDA_INC = "/usr/local/cuda/include"


def _compile(extra, out=None):
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(ROOT, "oracle")] + extra + [SRC]
    if out is None:
        cmd.append("-fsyntax-only")
    else:
        cmd += ["-L" + PKG, "-lgi", "-L" + os.path.join(ROOT, "oracle"), "-loracle", "-Wl,-rpath," + PKG,
                "-Wl,-rpath," + os.path.join(ROOT, "oracle"), "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def build_suite(gi, oc):
    os.makedirs(BUILD, exist_ok=True)
    return _compile(["-I" + CUDA_INC], os.path.join(BUILD, "run_suite"))


def test_shim_compiles_without_cuda_headers():
    """The shim needs no CUDA toolkit: it falls back to its own POD vector types."""
    _compile([])


def test_suite_links_against_the_c_abi(gi, oc):
    """Every entry point the shim uses resolves in libgi.so."""
    exe = build_suite(gi, oc)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_run_suite_pose_sweep(gi, oc, tmp_path):
    """runSuite-shaped sweep: controller and one-shot paths equal the exact oracle
    (pair sets and segments) on every seeded pose."""
    exe = build_suite(gi, oc)
    out = tmp_path / "suite.csv"
    r = subprocess.run([exe, "6", "7", "30", "0.25", str(out), "1"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    rows = list(csv.DictReader(open(out)))
    assert len(rows) == 6
    for row in rows:
        assert row["truth"] == row["controller"] == row["standalone"]
        assert row["fp"] == row["fn"] == row["fp_standalone"] == row["fn_standalone"] == "0"
        assert row["segments"] == "1"
    assert sum(int(row["truth"]) for row in rows) > 0
