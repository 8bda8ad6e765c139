"""Run history, CSV export and run diffs (host code in libgi.so, called without a
device), pinned to the reference's own IntersectionHistory
(src/CPU/IntersectionHistory.h): byte-exact digests of the CSVs it wrote
(tests/golden/history.json, made by tests/golden/make_history_golden.py) and,
where the reference program is built (oracle/_ref/history_ref), live comparisons
on seeded runs."""
import csv
import hashlib
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

sys.path.insert(0, GOLDEN)
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "history_ref")


@pytest.fixture(scope="module")
def golden():
    return json.load(open(os.path.join(GOLDEN, "history.json")))


@pytest.fixture(scope="module")
def runs(oc):
    import make_history_golden as mhg

    return {name: (vA, tA, vB, tB, pairs) for name, vA, tA, vB, tB, pairs in mhg.runs()}


def _digest(path):
    data = open(path, "rb").read()
    return dict(sha256=hashlib.sha256(data).hexdigest(), bytes=len(data), rows=data.count(b"\n") - 1)


def _history(runs, names):
    from gpuintersector.history import IntersectionHistory, PosedMesh

    h = IntersectionHistory()
    for n in names:
        vA, tA, vB, tB, pairs = runs[n]
        h.record_posed(n, 1.0, pairs, PosedMesh(vA, tA), PosedMesh(vB, tB))
    return h


@pytest.mark.parametrize("name", ["run1", "run2", "xrun"])
def test_export_matches_reference_bytes(runs, golden, tmp_path, name):
    h = _history(runs, [name])
    out = tmp_path / (name + ".csv")
    for nthreads in (1, 0):
        assert h.export_run_csv(0, out, nthreads=nthreads) == runs[name][4].shape[0]
        assert _digest(out) == golden["export_" + name]
    if name == "xrun":
        assert open(out).read() == golden["xrun_csv"]


@pytest.mark.parametrize("filt", ["all", "only1", "only2", "both"])
def test_diff_matches_reference_bytes(runs, golden, tmp_path, filt):
    h = _history(runs, ["run1", "run2"])
    out = tmp_path / "diff.csv"
    n1, n2, nb = h.export_diff_csv(0, 1, filt, out)
    assert (n1, n2, nb) == (154, 40, 614)
    assert _digest(out) == golden["diff_" + filt]


def test_filter_aliases_and_unknown(runs, tmp_path):
    h = _history(runs, ["run1", "run2"])
    a, b = tmp_path / "a.csv", tmp_path / "b.csv"
    for alias, canon in (("1", "only1"), ("Exclusive1", "only1"), ("2", "only2"), ("EXCLUSIVE2", "only2"),
                         ("BOTH", "both")):
        h.export_diff_csv(0, 1, alias, a)
        h.export_diff_csv(0, 1, canon, b)
        assert open(a, "rb").read() == open(b, "rb").read()
    h.export_diff_csv(0, 1, "nothing", a)  # an unknown filter writes the header only, as the reference
    assert open(a).read().count("\n") == 1


def test_ring_of_five_and_overview(runs):
    from gpuintersector.history import IntersectionHistory, PosedMesh

    vA, tA, vB, tB, pairs = runs["run1"]
    A, B = PosedMesh(vA, tA), PosedMesh(vB, tB)
    h = IntersectionHistory()
    assert "No history entries" in h.overview()
    ids = [h.record_posed("m%d" % k, 0.5 * k, pairs[: k + 1], A, B) for k in range(7)]
    assert ids == list(range(7))
    assert [e.id for e in h.entries] == [2, 3, 4, 5, 6]
    with pytest.raises(KeyError):
        h.entry(1)
    ov = h.overview().splitlines()
    assert ov[0].startswith("Entry ID") and len(ov) == 6
    assert ov[1].split()[:2] == ["2", "m2"] and ov[1].split()[-1] == "3"


def test_records_view_and_pose(gi, runs):
    from gpuintersector.history import IntersectionHistory

    vA, tA, vB, tB, pairs = runs["run1"]
    pose = gi.pose_from_euler_deg((10.0, 20.0, 30.0), (0.1, 0.0, 0.0), (0.3, 0.0, -0.2))
    h = IntersectionHistory()
    h.record_run("gpu", 0.25, pairs, (vA, tA), None, (vB, tB), pose)
    r = h.entry(0).records()
    wB = gi.pose_apply(pose, vB)
    assert np.array_equal(r["vB_idx"], tB[pairs[:, 1]])
    assert np.array_equal(r["b_v"], wB[tB[pairs[:, 1]]])
    assert np.array_equal(r["a_v"], vA[tA[pairs[:, 0]]])


def test_csv_parses_back_exactly(runs, tmp_path):
    h = _history(runs, ["xrun"])
    out = tmp_path / "x.csv"
    h.export_run_csv(0, out)
    vA, tA, vB, tB, pairs = runs["xrun"]
    rows = list(csv.reader(open(out)))[1:]
    for row, (a, b) in zip(rows, pairs):
        coords = np.array([float(x) for x in row[8:]])
        want = np.concatenate([vA[tA[a]].reshape(-1), vB[tB[b]].reshape(-1)])
        assert np.array_equal(coords.view(np.uint64), want.view(np.uint64))  # -0.0 kept


def test_invalid_inputs_rejected(runs, tmp_path):
    from gpuintersector import GIError
    from gpuintersector.history import PosedMesh, write_records_csv

    vA, tA, vB, tB, pairs = runs["xrun"]
    A, B = PosedMesh(vA, tA), PosedMesh(vB, tB)
    out = tmp_path / "bad.csv"
    for bad in ([[6, 0]], [[0, -1]], [[-2, 0]]):
        with pytest.raises(GIError):
            write_records_csv(out, A, B, np.array(bad))
        assert not out.exists()  # nothing written
    Abad = PosedMesh(vA[:5], tA)  # triangle 1 reaches vertex 5
    with pytest.raises(GIError):
        write_records_csv(out, Abad, B, np.array([[1, 0]]))
    with pytest.raises(GIError):
        write_records_csv(tmp_path / "no" / "dir.csv", A, B, pairs)


def test_pairs_diff_properties():
    from gpuintersector.history import pairs_diff

    rng = np.random.default_rng(3)
    for n1, n2 in ((0, 0), (0, 17), (23, 0), (1000, 700), (5000, 5000)):
        p1 = rng.integers(-3, 60, (n1, 2)).astype(np.int32)  # small range: many repeats and overlaps
        p2 = rng.integers(-3, 60, (n2, 2)).astype(np.int32)
        o1, o2, b = pairs_diff(p1, p2)
        s1, s2 = set(map(tuple, p1.tolist())), set(map(tuple, p2.tolist()))
        assert o1.tolist() == [list(x) for x in sorted(s1 - s2)]
        assert o2.tolist() == [list(x) for x in sorted(s2 - s1)]
        assert b.tolist() == [list(x) for x in sorted(s1 & s2)]


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference history program not built here")
def test_live_reference_on_seeded_runs(oc, tmp_path):
    import make_history_golden as mhg
    from gpuintersector.history import IntersectionHistory, PosedMesh

    rng = np.random.default_rng(11)
    for trial in range(4):
        nv, nt = 50, 80
        scale = 10.0 ** rng.integers(-12, 12)
        vA = rng.standard_normal((nv, 3)) * scale
        vB = rng.standard_normal((nv, 3)) * scale
        tA = rng.integers(0, nv, (nt, 3)).astype(np.uint32)
        tB = rng.integers(0, nv, (nt, 3)).astype(np.uint32)
        p1 = rng.integers(0, nt, (rng.integers(0, 200), 2)).astype(np.int32)
        p2 = np.concatenate([p1[::2], rng.integers(0, nt, (30, 2)).astype(np.int32)])
        h = IntersectionHistory()
        h.record_posed("a", 0, p1, PosedMesh(vA, tA), PosedMesh(vB, tB))
        h.record_posed("b", 0, p2, PosedMesh(vA, tA), PosedMesh(vB, tB))
        bins = []
        for k, p in enumerate((p1, p2)):
            bins.append(str(tmp_path / ("r%d.bin" % k)))
            mhg.write_records(bins[-1], vA, tA, vB, tB, p)
        ref, mine = tmp_path / "ref.csv", tmp_path / "mine.csv"
        subprocess.run([REF_BIN, "export", bins[0], str(ref)], check=True, capture_output=True)
        h.export_run_csv(0, mine)
        assert open(ref, "rb").read() == open(mine, "rb").read()
        for filt in ("all", "only2"):
            subprocess.run([REF_BIN, "diff", bins[0], bins[1], filt, str(ref)], check=True, capture_output=True)
            h.export_diff_csv(0, 1, filt, mine)
            assert open(ref, "rb").read() == open(mine, "rb").read()


@pytest.mark.gpu
def test_gpu_run_against_oracle_run_diff_is_empty(ctx, gi, oc, tmp_path):
    """The history use the reference makes of it: record the GPU run and the CPU
    run of the same scene and diff them; nothing is only in one of them."""
    import time

    from gpuintersector import meshgen as mg
    from gpuintersector.history import IntersectionHistory, PosedMesh

    from conftest import gi_pose, oracle_pose

    cfg = mg.config2()
    A = ctx.upload(cfg["vA"], cfg["tA"])
    B = ctx.upload(cfg["vB"], cfg["tB"])
    t0 = time.perf_counter()
    r = ctx.intersect(A, B, gi_pose(gi, cfg["poseA"]), gi_pose(gi, cfg["poseB"]), want_segments=False)
    ms_gpu = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    ref = oc.intersect_meshes(cfg["vA"], cfg["tA"], oracle_pose(oc, cfg["poseA"]), cfg["vB"], cfg["tB"],
                              oracle_pose(oc, cfg["poseB"]), want_segments=False)
    ms_cpu = (time.perf_counter() - t0) * 1e3
    PA = PosedMesh(cfg["vA"], cfg["tA"], gi_pose(gi, cfg["poseA"]))
    PB = PosedMesh(cfg["vB"], cfg["tB"], gi_pose(gi, cfg["poseB"]))
    h = IntersectionHistory()
    g = h.record_posed("gpu", ms_gpu, r.pairs, PA, PB)
    c = h.record_posed("oracle", ms_cpu, ref["pairs"], PA, PB)
    n1, n2, nb = h.export_diff_csv(g, c, "all", tmp_path / "d.csv")
    assert n1 == 0 and n2 == 0 and nb == len(ref["pairs"]) > 0
    assert h.export_run_csv(g, tmp_path / "g.csv") == len(r.pairs)
    A.release()
    B.release()
