"""Run history and run diffs for chasing parity failures.

Mirrors the reference's IntersectionHistory (src/CPU/IntersectionHistory.h:
43-232): the last runs are kept in a ring of five (recordRun, :62-80); the
overview lists them (printOverview, :82-104); a run is exported to CSV with,
per intersecting pair, the face ids, the six vertex indices and the eighteen
posed coordinates at 17 significant digits (exportRunToCsv, :114-160); two
runs are diffed by their (faceA, faceB) sets into a CSV whose first column is
ONLY_IN_<id1>, ONLY_IN_<id2> or IN_BOTH, filtered by all / only1 / only2 / both
(exportDiff, :162-232).

A run is kept as its pair list plus the posed meshes: the vertices go through
gi_pose_apply once at record time, so the coordinates are bit-identical to
what the library intersected.  Formatting and the diff run in libgi.so
(gi_records_write_csv, gi_pairs_diff) on host threads.
"""
import ctypes
import datetime

import numpy as np

from . import _abi

HEADER = ("FaceA,FaceB,VA0_Idx,VA1_Idx,VA2_Idx,VB0_Idx,VB1_Idx,VB2_Idx,"
          "A_V0_X,A_V0_Y,A_V0_Z,A_V1_X,A_V1_Y,A_V1_Z,A_V2_X,A_V2_Y,A_V2_Z,"
          "B_V0_X,B_V0_Y,B_V0_Z,B_V1_X,B_V1_Y,B_V1_Z,B_V2_X,B_V2_Y,B_V2_Z")

_FILTERS = {"all": (1, 1, 1), "only1": (1, 0, 0), "1": (1, 0, 0), "exclusive1": (1, 0, 0),
            "only2": (0, 1, 0), "2": (0, 1, 0), "exclusive2": (0, 1, 0), "both": (0, 0, 1)}


def _i32p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _check(rc, what):
    if rc:
        from . import GIError

        raise GIError(rc, what)


class PosedMesh:
    """Posed vertices (float64, n x 3) and triangles (uint32, m x 3) of one run."""

    def __init__(self, verts, tris, pose=None):
        from . import pose_apply

        v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 3)
        self.verts = pose_apply(pose, v) if pose is not None else v.copy()
        self.tris = np.array(tris, dtype=np.uint32, copy=True).reshape(-1, 3)

    def c(self):
        return _abi.RecordMesh(self.verts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self.verts.shape[0],
                               self.tris.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), self.tris.shape[0])


def write_records_csv(path, A, B, pairs, category=None, header=True, append=False, nthreads=0):
    """Rows of `pairs` (n x 2 faceA, faceB) over posed meshes A and B, in order."""
    p = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
    ca, cb = A.c(), B.c()
    rc = _abi.load().gi_records_write_csv(str(path).encode(), int(append), int(header),
                                          category.encode() if category else None, ctypes.byref(ca),
                                          ctypes.byref(cb), _i32p(p), p.shape[0], nthreads)
    _check(rc, "gi_records_write_csv")
    return p.shape[0]


def pairs_diff(p1, p2):
    """(only in p1, only in p2, in both), each sorted by (faceA, faceB), duplicates merged."""
    a = np.ascontiguousarray(p1, dtype=np.int32).reshape(-1, 2)
    b = np.ascontiguousarray(p2, dtype=np.int32).reshape(-1, 2)
    o1 = np.empty((max(a.shape[0], 1), 2), np.int32)
    o2 = np.empty((max(b.shape[0], 1), 2), np.int32)
    bo = np.empty((max(min(a.shape[0], b.shape[0]), 1), 2), np.int32)
    n1, n2, nb = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    rc = _abi.load().gi_pairs_diff(_i32p(a), a.shape[0], _i32p(b), b.shape[0], _i32p(o1), ctypes.byref(n1),
                                   _i32p(o2), ctypes.byref(n2), _i32p(bo), ctypes.byref(nb))
    _check(rc, "gi_pairs_diff")
    return o1[:n1.value].copy(), o2[:n2.value].copy(), bo[:nb.value].copy()


class HistoryEntry:
    def __init__(self, id_, method, elapsed_ms, pairs, A, B):
        self.id = id_
        self.method = method
        self.timestamp = datetime.datetime.now().strftime("%Y-%m-%d %H:%M:%S")
        self.elapsed_ms = float(elapsed_ms)
        self.pairs = np.array(pairs, dtype=np.int32, copy=True).reshape(-1, 2)
        self.A, self.B = A, B

    @property
    def count(self):
        return self.pairs.shape[0]

    def records(self):
        """Structured view of the run: face ids, vertex indices, posed coordinates."""
        ta = self.A.tris[self.pairs[:, 0]]
        tb = self.B.tris[self.pairs[:, 1]]
        return dict(faceA=self.pairs[:, 0], faceB=self.pairs[:, 1], vA_idx=ta, vB_idx=tb,
                    a_v=self.A.verts[ta], b_v=self.B.verts[tb])


class IntersectionHistory:
    """The last MAX_HISTORY runs (oldest dropped first)."""

    MAX_HISTORY = 5

    def __init__(self):
        self.entries = []
        self.next_id = 0

    def record_run(self, method, elapsed_ms, pairs, mesh_a, pose_a, mesh_b, pose_b):
        """mesh_*: (verts, tris) host arrays; pose_*: a gi pose or None (identity).
        The posed vertices are computed now and kept with the entry."""
        return self.record_posed(method, elapsed_ms, pairs, PosedMesh(*mesh_a, pose_a), PosedMesh(*mesh_b, pose_b))

    def record_posed(self, method, elapsed_ms, pairs, A, B):
        """As record_run over PosedMesh objects (runs of the same pose share them)."""
        e = HistoryEntry(self.next_id, method, elapsed_ms, pairs, A, B)
        self.next_id += 1
        if len(self.entries) >= self.MAX_HISTORY:
            self.entries.pop(0)
        self.entries.append(e)
        return e.id

    def entry(self, id_):
        for e in self.entries:
            if e.id == id_:
                return e
        raise KeyError("entry %d is not among the last %d runs" % (id_, self.MAX_HISTORY))

    def overview(self):
        lines = ["%-8s%-18s%-24s%-16s%-16s" % ("Entry ID", "Method", "Timestamp", "Time (ms)", "Intersections")]
        if not self.entries:
            lines.append("  [No history entries recorded yet]")
        for e in self.entries:
            lines.append("%-8d%-18s%-24s%-16.2f%-16d" % (e.id, e.method, e.timestamp, e.elapsed_ms, e.count))
        return "\n".join(lines)

    def export_run_csv(self, id_, path, nthreads=0):
        e = self.entry(id_)
        return write_records_csv(path, e.A, e.B, e.pairs, nthreads=nthreads)

    def diff(self, id1, id2):
        """(only in id1, only in id2, in both) as sorted (n, 2) pair arrays."""
        return pairs_diff(self.entry(id1).pairs, self.entry(id2).pairs)

    def export_diff_csv(self, id1, id2, filt, path, nthreads=0):
        """filt: all, only1 (1, exclusive1), only2 (2, exclusive2) or both; rows
        of pairs in both runs carry the first run's coordinates.  Returns the
        counts (only1, only2, both) of the whole diff."""
        e1, e2 = self.entry(id1), self.entry(id2)
        w1, w2, wb = _FILTERS.get(filt.lower(), (0, 0, 0))
        only1, only2, both = pairs_diff(e1.pairs, e2.pairs)
        parts = [("ONLY_IN_%d" % id1, only1, e1)] * w1 + [("ONLY_IN_%d" % id2, only2, e2)] * w2 + \
                [("IN_BOTH", both, e1)] * wb
        write_records_csv(path, e1.A, e1.B, np.empty((0, 2), np.int32), category="X", header=True)
        for cat, pairs, src in parts:
            write_records_csv(path, src.A, src.B, pairs, category=cat, header=False, append=True, nthreads=nthreads)
        return only1.shape[0], only2.shape[0], both.shape[0]
