"""Generates tests/golden/history.json: byte-exact digests of the CSVs that the
reference's own IntersectionHistory (src/CPU/IntersectionHistory.h, built by
oracle/history_ref.mk into oracle/_ref/history_ref) writes for fixed runs.

Runs:
  run1  the sorted pair set of config1.npz (UV spheres 128x80, B posed);
  run2  run1 without every fifth pair, plus 40 other pairs and 5 repeats, shuffled;
  xrun  8 pairs over a 12-vertex mesh whose coordinates exercise the 17-digit
        format (signed zero, subnormal, largest double, 1e-5, 1e16, thirds).
Posed coordinates are the oracle's transform of the inputs (FP64, no FMA).
For each CSV the digest, size and row count are stored; the xrun export is
also stored verbatim.

Run from the repository root after `make -f oracle/history_ref.mk`:
    python tests/golden/make_history_golden.py
"""
import hashlib
import json
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as oc  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "history_ref")


def runs():
    """(name, posed vA, tA, posed vB, tB, pairs) of every fixture run."""
    g = np.load(os.path.join(HERE, "config1.npz"))
    vB = oc.transform(oc.pose_raw(g["poseB_R"], g["poseB_C"], g["poseB_T"]), g["vB"])
    run1 = g["pairs"].astype(np.int32)
    rng = np.random.default_rng(7)
    keep = run1[np.arange(run1.shape[0]) % 5 != 0]
    extra = np.stack([rng.integers(0, g["tA"].shape[0], 40), rng.integers(0, g["tB"].shape[0], 40)], 1)
    run2 = np.concatenate([keep, extra.astype(np.int32), keep[:5]])
    run2 = run2[rng.permutation(run2.shape[0])]
    xv = np.array([[0.0, -0.0, 1.0], [5e-324, -2.2250738585072014e-308, 1.7976931348623157e308],
                   [1e-5, -1e-5, 0.1], [1e16, 123456789012345678.0, -1.0 / 3.0], [2.0 / 3.0, 1e-300, -1e300],
                   [0.5, 0.25, 3.0], [100.0, 1e15, 1e17], [-7.0, 9.999999999999999e-5, 1e-4],
                   [np.pi, np.e, -np.sqrt(2.0)], [1.0000000000000002, 0.9999999999999999, 4503599627370497.0],
                   [65536.0, -65536.5, 1e-320], [2.0 ** 100, 2.0 ** -100, -(2.0 ** 53)]])
    xt = np.array([[0, 1, 2], [3, 4, 5], [6, 7, 8], [9, 10, 11], [0, 5, 10], [11, 2, 7]], np.uint32)
    xpairs = np.array([[0, 1], [1, 0], [2, 3], [3, 2], [4, 5], [5, 4], [0, 0], [5, 5]], np.int32)
    return [("run1", g["vA"], g["tA"], vB, g["tB"], run1), ("run2", g["vA"], g["tA"], vB, g["tB"], run2),
            ("xrun", xv, xt, xv[::-1].copy(), xt, xpairs)]


def write_records(path, vA, tA, vB, tB, pairs):
    with open(path, "wb") as f:
        f.write(struct.pack("<Q", pairs.shape[0]))
        for a, b in pairs:
            ia, ib = tA[a], tB[b]
            f.write(np.concatenate([[a, b], ia, ib]).astype("<i4").tobytes())
            f.write(np.concatenate([vA[ia].reshape(-1), vB[ib].reshape(-1)]).astype("<f8").tobytes())


def digest(path):
    data = open(path, "rb").read()
    return dict(sha256=hashlib.sha256(data).hexdigest(), bytes=len(data), rows=data.count(b"\n") - 1)


def main():
    if not os.path.exists(REF_BIN):
        sys.exit("build the reference program first: make -f oracle/history_ref.mk")
    out = {}
    with tempfile.TemporaryDirectory() as td:
        bins = {}
        for name, vA, tA, vB, tB, pairs in runs():
            bins[name] = os.path.join(td, name + ".bin")
            write_records(bins[name], vA, tA, vB, tB, pairs)
            csv = os.path.join(td, name + ".csv")
            subprocess.run([REF_BIN, "export", bins[name], csv], check=True, capture_output=True)
            out["export_" + name] = digest(csv)
            if name == "xrun":
                out["xrun_csv"] = open(csv).read()
        for filt in ("all", "only1", "only2", "both"):
            csv = os.path.join(td, "diff_%s.csv" % filt)
            subprocess.run([REF_BIN, "diff", bins["run1"], bins["run2"], filt, csv], check=True, capture_output=True)
            out["diff_" + filt] = digest(csv)
    with open(os.path.join(HERE, "history.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
