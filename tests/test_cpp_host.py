"""C++ host side: the header-only KernelBVHController shim (include/gi/gi_controller.hpp),
the pose-sweep harness gi::TestSuite (include/gi/gi_suite.hpp) with its pose
sequence gi_sweep_poses, and the harness driver tests/cpp/run_suite.cpp."""
import csv
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gpu-cubql-intersector-standalone_b200")
BUILD = os.path.join(ROOT, "tests", "cpp", "_build")
CUDA_INC = "/usr/local/cuda/include"

# the reference's CSV headers (src/CPU/TestSuite.cpp:329-331, 367-371, 409-413)
SUMMARY_HEADER = ("step,intersections,candidates,total_possible_pairs,candidate_yield,surface_overlap_omega,"
                  "hybrid_ms,hybrid_standalone_ms,cgal_classic_ms,cgal_parallel_ms,"
                  "hybrid_match,standalone_match,cgal_parallel_match")
STANDARD_HEADER = ("step,gpu_total_ms,cross_check_engine_ms,dual_tree_step_ms,parallel_dfs_descent_ms,"
                   "preallocate_ms,assembly_phase_ms,aabb_candidate_exec_ms,gpu_float_predicates_ms,"
                   "gpu_double_predicates_ms,thrust_compaction_d2h_ms,cpu_narrow_phase_ms,"
                   "loop_workspace_cleanup_ms,explicit_cleanup_sync_ms,"
                   "confirmed_green_pairs,confirmed_yellow_pairs,confirmed_orange_pairs")
STANDALONE_HEADER = ("step,gpu_total_ms,raw_alloc_copy_ms,thrust_init_overhead_ms,build_refit_mesh_a_ms,"
                     "build_refit_mesh_b_ms,cross_check_engine_ms,dual_tree_step_ms,parallel_dfs_descent_ms,"
                     "preallocate_ms,assembly_phase_ms,aabb_candidate_exec_ms,gpu_float_predicates_ms,"
                     "gpu_double_predicates_ms,thrust_compaction_d2h_ms,cpu_narrow_phase_ms,"
                     "loop_workspace_cleanup_ms,explicit_cleanup_sync_ms,"
                     "confirmed_green_pairs,confirmed_yellow_pairs,confirmed_orange_pairs")


def _compile(src, extra, out=None, oracle=False):
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(ROOT, "oracle")] + extra + [os.path.join(ROOT, "tests", "cpp", src)]
    if out is None:
        cmd.append("-fsyntax-only")
    else:
        cmd += ["-L" + PKG, "-lgi", "-Wl,-rpath," + PKG, "-o", out]
        if oracle:
            cmd += ["-L" + os.path.join(ROOT, "oracle"), "-loracle", "-Wl,-rpath," + os.path.join(ROOT, "oracle")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def build_suite(gi, oc):
    os.makedirs(BUILD, exist_ok=True)
    return _compile("run_suite.cpp", ["-I" + CUDA_INC], os.path.join(BUILD, "run_suite"), oracle=True)


def test_shim_compiles_without_cuda_headers():
    """The shim and the harness need no CUDA toolkit: they fall back to their own POD vector types."""
    _compile("run_suite.cpp", [])
    _compile("suite_csv.cpp", [])


def test_suite_links_against_the_c_abi(gi, oc):
    """Every entry point the shim and the harness use resolves in libgi.so."""
    exe = build_suite(gi, oc)
    assert os.path.exists(exe)


def test_sweep_poses_match_the_reference_draws(gi):
    """gi_sweep_poses gives, bit for bit, the poses a GCC build of the reference's
    sweep draws (tests/golden/sweep_poses.json, tests/golden/make_sweep_golden.py)."""
    cases = json.load(open(os.path.join(ROOT, "tests", "golden", "sweep_poses.json")))
    for c in cases:
        rot, tr = gi.sweep_poses(c["seed"], c["steps"], c["max_rot_deg"], c["max_trans"], c["base_rot_b"],
                                 c["base_trans_b"])
        want_r = np.array([[float.fromhex(x) for x in row] for row in c["rot_b"]])
        want_t = np.array([[float.fromhex(x) for x in row] for row in c["trans_b"]])
        assert np.array_equal(rot, want_r) and np.array_equal(tr, want_t)
    # bounds and the invalid-argument path
    rot, tr = gi.sweep_poses(5, 1000, 2.0, 0.01)
    assert np.abs(rot).max() <= 2.0 and np.abs(tr).max() <= 0.01
    from gpuintersector import GIError

    with pytest.raises(GIError):
        gi.sweep_poses(5, 3, -1.0, 0.1)


def test_suite_csv_files_and_names(gi, tmp_path):
    """The harness writes the reference's three CSV files with its headers (this
    library's columns follow the reference's) at 10 significant digits."""
    os.makedirs(BUILD, exist_ok=True)
    exe = _compile("suite_csv.cpp", ["-I" + CUDA_INC], os.path.join(BUILD, "suite_csv"))
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    names = dict(line.split(" -> ") for line in r.stdout.splitlines())
    assert names["benchmark_results.csv"] == "benchmark_results_x.csv"
    assert names["out.d/run"] == "out.d/run_x.csv" and names["a/b.c/d.csv"] == "a/b.c/d_x.csv"
    # runIntersectionPipeline's predicate mode: the reference's modes 0-4 select the
    # FP32 cascade, 5 the plain FP64 form, anything else is an invalid argument
    assert [names["mode %d" % m] for m in range(0, 6)] == ["0", "0", "0", "0", "0", "1"]
    assert names["mode -1"] == "error 1" and names["mode 6"] == "error 1"
    summary = open(tmp_path / "sweep.csv").read().splitlines()
    assert summary[0] == SUMMARY_HEADER
    assert summary[1] == "0,768,12345,409010176,3.018262313e-05,0.0123456789,0.3333333333,12.5,333.3333333,0,1,1,0"
    std = open(tmp_path / "sweep_standard_breakdown.csv").read().splitlines()
    assert std[0].startswith(STANDARD_HEADER + ",")
    row = dict(zip(std[0].split(","), std[1].split(",")))
    assert row["gpu_total_ms"] == "0.25" and row["aabb_candidate_exec_ms"] == "0.125"
    assert row["gpu_double_predicates_ms"] == "0.0625" and row["confirmed_yellow_pairs"] == "45"
    assert row["candidates"] == "12345" and row["confirmed_orange_pairs"] == "0"
    sa = open(tmp_path / "sweep_standalone_breakdown.csv").read().splitlines()
    assert sa[0].startswith(STANDALONE_HEADER + ",") and len(sa) == 3


@pytest.mark.gpu
def test_run_suite_pose_sweep(gi, oc, tmp_path):
    """runSuite sweep on 2 x 20 k-triangle UV spheres: the controller path, the
    one-shot path and the multi-threaded oracle equal the single-thread oracle
    on every seeded pose (pair sets), the controller's segments equal the
    oracle's, and the three CSV files carry the reference's columns."""
    exe = build_suite(gi, oc)
    out = tmp_path / "suite.csv"
    r = subprocess.run([exe, "6", "1337", "15", "0.5", str(out), "1"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr
    assert "6 / 6 steps matched" in r.stdout and "segments identical on 6 / 6 steps" in r.stdout
    assert "Steps with Full Consensus: 6 / 6" in r.stdout
    rows = list(csv.DictReader(open(out)))
    assert open(out).readline().strip() == SUMMARY_HEADER
    assert len(rows) == 6
    rot, _ = gi.sweep_poses(1337, 6, 15.0, 0.5)
    for row in rows:
        assert row["hybrid_match"] == row["standalone_match"] == row["cgal_parallel_match"] == "1"
        assert 0.0 <= float(row["surface_overlap_omega"]) < 1.0
        assert int(row["candidates"]) >= int(row["intersections"])
        assert int(row["total_possible_pairs"]) == 20224 * 20224
    assert sum(int(row["intersections"]) for row in rows) > 0
    for suffix, header in (("_standard_breakdown", STANDARD_HEADER), ("_standalone_breakdown", STANDALONE_HEADER)):
        b = list(csv.DictReader(open(tmp_path / ("suite%s.csv" % suffix))))
        assert len(b) == 6 and open(tmp_path / ("suite%s.csv" % suffix)).readline().startswith(header)
        for row, s in zip(b, rows):
            assert row["pairs"] == s["intersections"] and float(row["gpu_total_ms"]) > 0
