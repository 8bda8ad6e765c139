"""Python host mirror of the reference's GPUIntersector interface over libgi.so.

The compute path is the CUDA library behind the C ABI (include/gi/gi.h); this
module only marshals arrays and handles.  It mirrors, with the same names and
argument meaning (reference project paths):

  KernelBVHController          src/GPUIntersector/KernelBVHController.h:36-95
    construct / setTransformBoth / runIntersectionPipeline / clearGPU /
    reconstructGPU / getCenterA / getCenterB / isGPUAllocated
  run_grid_forest_intersection_pipeline
                               src/GPUIntersector/StandaloneBVHPipeline.h:27-43
  compute_exact_intersection_curves
                               src/CPU/MeshIntersectionCurves.h:24-29

If libgi.so is missing or no CUDA device is present the calls raise; nothing
falls back to a CPU implementation.
"""
import ctypes
import os

import numpy as np

from . import _abi
from ._abi import GI_NOALLOC_MAX_PAIRS, GI_PREC_FP32_CASCADE, GI_PREC_FP64

__all__ = ["GIError", "Context", "Mesh", "Result", "BatchResult", "pose_identity", "pose_from_euler_deg", "pose_raw",
           "KernelBVHController", "run_grid_forest_intersection_pipeline", "compute_exact_intersection_curves",
           "GI_PREC_FP32_CASCADE", "GI_PREC_FP64", "lib"]


class GIError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__("gi status %d (%s)%s" % (status, _status_name(status), (": " + msg) if msg else ""))


def _status_name(s):
    try:
        return lib().gi_status_string(s).decode()
    except Exception:
        return "?"


def lib():
    return _abi.load()


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _up(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


# ---------------------------------------------------------------- poses
def pose_identity():
    p = _abi.Pose()
    lib().gi_pose_identity(ctypes.byref(p))
    return p


def pose_from_euler_deg(rot_deg, center=(0.0, 0.0, 0.0), trans=(0.0, 0.0, 0.0)):
    """R = Rz*Ry*Rx from degrees about `center`, then `trans` (RotationTools.h:28-70)."""
    p = _abi.Pose()
    r = np.ascontiguousarray(rot_deg, dtype=np.float64)
    c = np.ascontiguousarray(center, dtype=np.float64)
    t = np.ascontiguousarray(trans, dtype=np.float64)
    rc = lib().gi_pose_from_euler_deg(_dp(r), _dp(c), _dp(t), ctypes.byref(p))
    if rc:
        raise GIError(rc)
    return p


def pose_raw(R, center=(0.0, 0.0, 0.0), trans=(0.0, 0.0, 0.0)):
    """General pose world = R (v - center) + center + trans (R row-major 3x3)."""
    p = _abi.Pose()
    R = np.asarray(R, dtype=np.float64).reshape(9)
    for i in range(9):
        p.R[i] = float(R[i])
    for i in range(3):
        p.center[i] = float(center[i])
        p.trans[i] = float(trans[i])
    p.identity = 0
    return p


def pose_apply(pose, verts):
    v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 3)
    out = np.empty_like(v)
    rc = lib().gi_pose_apply(ctypes.byref(pose), _dp(v), v.shape[0], _dp(out))
    if rc:
        raise GIError(rc)
    return out


def sweep_poses(seed, steps, max_rot_deg=15.0, max_trans=0.5, base_rot_b=(0.0, 0.0, 0.0),
                base_trans_b=(0.0, 0.0, 0.0)):
    """B's Euler angles (degrees) and translations, (steps, 3) each, of the
    seeded pose sweep (gi_sweep_poses: the reference's TestSuite draws)."""
    rot = np.empty((steps, 3))
    tr = np.empty((steps, 3))
    br = np.ascontiguousarray(base_rot_b, dtype=np.float64)
    bt = np.ascontiguousarray(base_trans_b, dtype=np.float64)
    rc = lib().gi_sweep_poses(int(seed), int(steps), float(max_rot_deg), float(max_trans), _dp(br), _dp(bt),
                              _dp(rot), _dp(tr))
    if rc:
        raise GIError(rc, "gi_sweep_poses")
    return rot, tr


# ---------------------------------------------------------------- handles
class Context:
    """Owns one CUDA stream and the scratch buffers of the intersector."""

    def __init__(self, device=0, hbm_budget_bytes=0, flags=0):
        self._lib = lib()
        o = _abi.Options(device, flags, hbm_budget_bytes)
        h = ctypes.c_void_p()
        rc = self._lib.gi_create(ctypes.byref(o), ctypes.byref(h))
        if rc:
            raise GIError(rc, "gi_create")
        self.handle = h

    def check(self, rc, what=""):
        if rc:
            msg = self._lib.gi_last_error(self.handle).decode(errors="replace")
            raise GIError(rc, "%s %s" % (what, msg))

    def close(self):
        if self.handle:
            self._lib.gi_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # meshes
    def upload(self, verts, tris):
        return Mesh(self, verts, tris)

    def upload_device(self, d_verts_ptr, nv, d_tris_ptr, nt):
        """Mesh from device pointers (e.g. torch tensor .data_ptr()) on the context's device."""
        return Mesh(self, None, None, device_ptrs=(d_verts_ptr, nv, d_tris_ptr, nt))

    # intersection
    @staticmethod
    def _opts(want_segments=True, precision=GI_PREC_FP32_CASCADE, sort_output=True):
        o = _abi.IntersectOpts()
        lib().gi_intersect_opts_default(ctypes.byref(o))
        o.want_segments = 1 if want_segments else 0
        o.precision_mode = int(precision)
        o.sort_output = 1 if sort_output else 0
        return o

    def intersect(self, A, B, pose_a=None, pose_b=None, want_segments=True, precision=GI_PREC_FP32_CASCADE,
                  sort_output=True):
        o = self._opts(want_segments, precision, sort_output)
        r = ctypes.c_void_p()
        rc = self._lib.gi_intersect(self.handle, A.handle, ctypes.byref(pose_a) if pose_a is not None else None,
                                    B.handle, ctypes.byref(pose_b) if pose_b is not None else None,
                                    ctypes.byref(o), ctypes.byref(r))
        self.check(rc, "gi_intersect")
        return Result(r)

    def intersect_batch(self, jobs, want_segments=True, precision=GI_PREC_FP32_CASCADE, sort_output=True):
        """jobs: list of (A, pose_a, B, pose_b); returns a list of Result."""
        n = len(jobs)
        arr = (_abi.PairJob * n)()
        ident = pose_identity()
        for i, (A, pa, B, pb) in enumerate(jobs):
            arr[i].A = A.handle
            arr[i].B = B.handle
            arr[i].pose_a = pa if pa is not None else ident
            arr[i].pose_b = pb if pb is not None else ident
        outs = (ctypes.c_void_p * n)()
        o = self._opts(want_segments, precision, sort_output)
        rc = self._lib.gi_intersect_batch(self.handle, arr, n, ctypes.byref(o), outs)
        self.check(rc, "gi_intersect_batch")
        return [Result(ctypes.c_void_p(outs[i])) for i in range(n)]

    def intersect_batch_flat(self, jobs, want_segments=True, precision=GI_PREC_FP32_CASCADE, sort_output=True):
        """The batch call of intersect_batch with its results as whole-batch
        arrays instead of one Result per job (a batch of thousands of jobs
        does not pay per-job Python objects):

          pairs (N, 2) int32, job (N,) uint32: the job of each pair,
          offsets (njobs + 1,): job j owns pairs[offsets[j]:offsets[j + 1]],
          segments (M, 6) float64, seg_pair (M,) int64: index into pairs,
          stats: the launch-wide statistics of the call.

        pairs and segments are views of the library's pinned result block
        (all jobs' results lie in it back to back; copies are made otherwise)."""
        n = len(jobs)
        arr = (_abi.PairJob * n)()
        ident = pose_identity()
        for i, (A, pa, B, pb) in enumerate(jobs):
            arr[i].A = A.handle
            arr[i].B = B.handle
            arr[i].pose_a = pa if pa is not None else ident
            arr[i].pose_b = pb if pb is not None else ident
        outs = (ctypes.c_void_p * n)()
        o = self._opts(want_segments, precision, sort_output)
        rc = self._lib.gi_intersect_batch(self.handle, arr, n, ctypes.byref(o), outs)
        self.check(rc, "gi_intersect_batch")
        return BatchResult([_ResultOwner(ctypes.c_void_p(outs[i])) for i in range(n)])

    def intersect_oneshot(self, vA, tA, vB, tB, pose_a=None, pose_b=None, want_segments=True,
                          precision=GI_PREC_FP32_CASCADE, sort_output=True):
        vA = np.ascontiguousarray(vA, dtype=np.float64).reshape(-1, 3)
        vB = np.ascontiguousarray(vB, dtype=np.float64).reshape(-1, 3)
        tA = np.ascontiguousarray(tA, dtype=np.uint32).reshape(-1, 3)
        tB = np.ascontiguousarray(tB, dtype=np.uint32).reshape(-1, 3)
        o = self._opts(want_segments, precision, sort_output)
        r = ctypes.c_void_p()
        rc = self._lib.gi_intersect_oneshot(self.handle, _dp(vA), vA.shape[0], _up(tA), tA.shape[0],
                                            ctypes.byref(pose_a) if pose_a is not None else None,
                                            _dp(vB), vB.shape[0], _up(tB), tB.shape[0],
                                            ctypes.byref(pose_b) if pose_b is not None else None,
                                            ctypes.byref(o), ctypes.byref(r))
        self.check(rc, "gi_intersect_oneshot")
        return Result(r)

    def wait_stream(self, stream_ptr):
        """Orders the library's streams after the work queued so far on a CUDA
        stream (its cudaStream_t as an int, e.g. torch.cuda.current_stream().cuda_stream):
        call it before passing device inputs produced on that stream."""
        self.check(self._lib.gi_wait_stream(self.handle, ctypes.c_void_p(int(stream_ptr) or None)), "gi_wait_stream")

    def classify_pairs(self, A, B, pose_a, pose_b, d_pairs_ptr, npairs, d_out_ptr, precision=GI_PREC_FP32_CASCADE):
        """Exact test of npairs candidate pairs (device pointers: int32 pairs, uint8 out)."""
        rc = self._lib.gi_classify_pairs(self.handle, A.handle, ctypes.byref(pose_a) if pose_a is not None else None,
                                         B.handle, ctypes.byref(pose_b) if pose_b is not None else None,
                                         ctypes.c_void_p(d_pairs_ptr), npairs, int(precision),
                                         ctypes.c_void_p(d_out_ptr))
        self.check(rc, "gi_classify_pairs")

    def classify_pairs_noalloc(self, A, B, pose_a, pose_b, d_pairs_ptr, npairs, d_out_ptr,
                               precision=GI_PREC_FP32_CASCADE):
        """classify_pairs with the library's fixed per-device scratch (no allocation, at most
        GI_NOALLOC_MAX_PAIRS pairs; concurrent calls on one device race)."""
        rc = self._lib.gi_classify_pairs_noalloc(self.handle, A.handle,
                                                 ctypes.byref(pose_a) if pose_a is not None else None,
                                                 B.handle, ctypes.byref(pose_b) if pose_b is not None else None,
                                                 ctypes.c_void_p(d_pairs_ptr), npairs, int(precision),
                                                 ctypes.c_void_p(d_out_ptr))
        self.check(rc, "gi_classify_pairs_noalloc")

    def predicate_signs(self, kind, pts, drop=None):
        """The device's orientation predicates, stage by stage, on host arrays:
        pts (n, 12) for GI_PRED_ORIENT3D (a, b, c, d) or (n, 9) for GI_PRED_ORIENT2D
        (a, b, c) with drop (n,) axes.  Returns int8 (n, 8): FP32 filter (line,
        plane form), FP64 semi-static filter (line, plane form), the exact
        stage's FP64 filter, the exact integer sign, the exact stage's answer, and
        the integer branch (0 int128, 1 multi-limb)."""
        per = 12 if kind == _abi.GI_PRED_ORIENT3D else 9
        p = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, per)
        n = p.shape[0]
        out = np.zeros((n, 8), dtype=np.int8)
        d = None
        if kind == _abi.GI_PRED_ORIENT2D:
            d = np.ascontiguousarray(drop, dtype=np.int32).reshape(-1)
            if d.shape[0] != n:
                raise ValueError("one drop axis per query")
        rc = self._lib.gi_predicate_signs(self.handle, int(kind), p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                          d.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)) if d is not None else None,
                                          n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int8)))
        self.check(rc, "gi_predicate_signs")
        return out

    def load_scene(self, path_a, path_b, scale_to_unit=True):
        """Both OFF files loaded, the scene normalised on the device and both meshes
        built: (A, B, scene dict with the centres and scale, report A, report B)."""
        ha, hb = ctypes.c_void_p(), ctypes.c_void_p()
        sc = _abi.Scene()
        ra, rb = _abi.OffReport(), _abi.OffReport()
        self.check(self._lib.gi_scene_load(self.handle, os.fsencode(path_a), os.fsencode(path_b),
                                           1 if scale_to_unit else 0, ctypes.byref(ha), ctypes.byref(hb),
                                           ctypes.byref(sc), ctypes.byref(ra), ctypes.byref(rb)), "gi_scene_load")
        return Mesh._wrap(self, ha), Mesh._wrap(self, hb), sc.as_dict(), ra.as_dict(), rb.as_dict()

    def server(self, max_inflight=256, want_segments=True, precision=GI_PREC_FP32_CASCADE):
        return Server(self, max_inflight, want_segments, precision)


def load_off(path, nthreads=0):
    """OFF file as the reference loads it (fan-triangulated, degenerate and
    duplicate triangles dropped): (verts (nv,3) float64, tris (nt,3) uint32,
    face_row (nt,) uint32, report dict).  Host only; needs no device."""
    L = lib()
    h = ctypes.c_void_p()
    rep = _abi.OffReport()
    rc = L.gi_off_load(os.fsencode(path), nthreads, ctypes.byref(h), ctypes.byref(rep))
    if rc:
        raise GIError(rc, "gi_off_load(%s)" % path)
    try:
        v = ctypes.POINTER(ctypes.c_double)()
        t = ctypes.POINTER(ctypes.c_uint32)()
        fr = ctypes.POINTER(ctypes.c_uint32)()
        nv, nt = ctypes.c_uint32(), ctypes.c_uint32()
        L.gi_off_arrays(h, ctypes.byref(v), ctypes.byref(nv), ctypes.byref(t), ctypes.byref(nt), ctypes.byref(fr))
        verts = (np.ctypeslib.as_array(v, shape=(nv.value, 3)).copy() if nv.value else np.zeros((0, 3)))
        tris = (np.ctypeslib.as_array(t, shape=(nt.value, 3)).copy() if nt.value else np.zeros((0, 3), np.uint32))
        rows = (np.ctypeslib.as_array(fr, shape=(nt.value,)).copy() if nt.value else np.zeros(0, np.uint32))
    finally:
        L.gi_off_free(h)
    return verts, tris, rows, rep.as_dict()


def curves(segments, seg_pair, npairs, drop_coplanar_interior=True):
    """Intersection curves from a result's segments (gi_curves_build): returns
    (vertices (k, 3) float64, list of (vertex index array, closed flag))."""
    L = lib()
    seg = np.ascontiguousarray(segments, dtype=np.float64).reshape(-1, 6)
    sp = np.ascontiguousarray(seg_pair, dtype=np.int32).reshape(-1)
    h = ctypes.c_void_p()
    rc = L.gi_curves_build(seg.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                           sp.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), seg.shape[0], int(npairs),
                           1 if drop_coplanar_interior else 0, ctypes.byref(h))
    if rc:
        raise GIError(rc, "gi_curves_build")
    try:
        vp = ctypes.POINTER(ctypes.c_double)()
        nv = ctypes.c_uint64()
        L.gi_curves_vertices(h, ctypes.byref(vp), ctypes.byref(nv))
        verts = np.ctypeslib.as_array(vp, shape=(nv.value, 3)).copy() if nv.value else np.zeros((0, 3))
        off = ctypes.POINTER(ctypes.c_uint64)()
        idx = ctypes.POINTER(ctypes.c_uint32)()
        cl = ctypes.POINTER(ctypes.c_uint8)()
        nc = ctypes.c_uint64()
        L.gi_curves_polylines(h, ctypes.byref(off), ctypes.byref(idx), ctypes.byref(cl), ctypes.byref(nc))
        out = []
        if nc.value:
            o = np.ctypeslib.as_array(off, shape=(nc.value + 1,)).copy()
            ii = np.ctypeslib.as_array(idx, shape=(int(o[-1]),)).copy() if o[-1] else np.zeros(0, np.uint32)
            cc = np.ctypeslib.as_array(cl, shape=(nc.value,)).copy()
            out = [(ii[o[k]:o[k + 1]], bool(cc[k])) for k in range(nc.value)]
    finally:
        L.gi_curves_free(h)
    return verts, out


class Mesh:
    def __init__(self, ctx, verts, tris, device_ptrs=None):
        self.ctx = ctx
        h = ctypes.c_void_p()
        if device_ptrs is not None:
            dv, nv, dt, nt = device_ptrs
            rc = ctx._lib.gi_mesh_upload_device(ctx.handle, ctypes.c_void_p(dv), nv, ctypes.c_void_p(dt), nt,
                                                ctypes.byref(h))
        else:
            v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 3)
            t = np.ascontiguousarray(tris, dtype=np.uint32).reshape(-1, 3)
            rc = ctx._lib.gi_mesh_upload(ctx.handle, _dp(v), v.shape[0], _up(t), t.shape[0], ctypes.byref(h))
        ctx.check(rc, "gi_mesh_upload")
        self.handle = h

    @classmethod
    def _wrap(cls, ctx, handle):
        m = cls.__new__(cls)
        m.ctx = ctx
        m.handle = handle
        return m

    def info(self):
        nv, nt = ctypes.c_uint32(), ctypes.c_uint32()
        nodes, nbytes = ctypes.c_uint64(), ctypes.c_uint64()
        self.ctx._lib.gi_mesh_info(self.handle, ctypes.byref(nv), ctypes.byref(nt), ctypes.byref(nodes),
                                   ctypes.byref(nbytes))
        ms = ctypes.c_double()
        self.ctx._lib.gi_mesh_build_ms(self.handle, ctypes.byref(ms))
        return dict(nv=nv.value, nt=nt.value, nodes=nodes.value, bytes=nbytes.value, build_ms=ms.value)

    def download(self):
        """The vertices as stored on the device (after any normalisation), (nv, 3) float64."""
        nv = self.info()["nv"]
        out = np.empty((nv, 3), dtype=np.float64)
        self.ctx.check(self.ctx._lib.gi_mesh_download(self.handle, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                       "gi_mesh_download")
        return out

    def release(self):
        if self.handle and self.ctx.handle:
            self.ctx._lib.gi_mesh_release(self.ctx.handle, self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class _ResultOwner:
    """Holds a gi_result handle; frees it when the last view of its arrays is gone."""

    __slots__ = ("handle",)

    def __init__(self, handle):
        self.handle = handle

    def __del__(self):
        try:
            lib().gi_result_free(self.handle)
        except Exception:
            pass


class _View:
    """numpy array interface over memory owned by a gi_result (keeps it alive)."""

    __slots__ = ("__array_interface__", "owner")

    def __init__(self, owner, addr, shape, dtype):
        self.owner = owner
        self.__array_interface__ = {"shape": shape, "typestr": np.dtype(dtype).str, "data": (addr, False),
                                    "version": 3}


class Result:
    """Pairs (n, 2) int32 sorted by (a, b); segments (m, 6) float64; seg_pair (m,).

    Results up to ZERO_COPY_BYTES are numpy views of the library's pinned result
    block (no copy; the block is released when the last view is dropped);
    larger ones are copied out and the block is released at once, so holding
    many large results pins no host memory."""

    ZERO_COPY_BYTES = 4 << 20

    __slots__ = ("_owner", "_stats", "_npairs", "_pairs", "_segments", "_seg_pair")

    def __init__(self, handle):
        # the device work and the copy to the host are done when the library
        # returns the handle; the Python views and the stats dict are built on
        # first use, so a batch of thousands of results returns at once
        self._owner = _ResultOwner(handle)
        self._stats = None
        self._pairs = None

    @property
    def stats(self):
        if self._stats is None:
            if self._owner is None:
                raise RuntimeError("result handle already released")
            st = _abi.Stats()
            lib().gi_result_stats(self._owner.handle, ctypes.byref(st))
            self._stats = st.as_dict()
        return self._stats

    def _load(self):
        if self._pairs is not None:
            return
        L = lib()
        handle = self._owner.handle
        p = ctypes.POINTER(ctypes.c_int32)()
        n = ctypes.c_uint64()
        L.gi_result_pairs(handle, ctypes.byref(p), ctypes.byref(n))
        sp = ctypes.POINTER(ctypes.c_double)()
        spp = ctypes.POINTER(ctypes.c_int32)()
        m = ctypes.c_uint64()
        L.gi_result_segments(handle, ctypes.byref(sp), ctypes.byref(spp), ctypes.byref(m))
        npairs, nsegs = n.value, m.value
        owner = self._owner
        zero_copy = 8 * npairs + 52 * nsegs <= self.ZERO_COPY_BYTES
        if not zero_copy:
            self.stats  # read now: the handle is released once the arrays are copied

        def arr(ptr, shape, dtype, count):
            if count == 0:
                return np.zeros(shape, dtype=dtype)
            a = np.asarray(_View(owner, ctypes.cast(ptr, ctypes.c_void_p).value, shape, dtype))
            return a if zero_copy else a.copy()

        self._npairs = npairs
        self._segments = arr(sp, (nsegs, 6), np.float64, nsegs)
        self._seg_pair = arr(spp, (nsegs,), np.int32, nsegs)
        self._pairs = arr(p, (npairs, 2), np.int32, npairs)
        if not zero_copy:
            self._owner = None  # freed here: every array was copied
        del owner

    @property
    def npairs(self):
        self._load()
        return self._npairs

    @property
    def pairs(self):
        self._load()
        return self._pairs

    @property
    def segments(self):
        self._load()
        return self._segments

    @property
    def seg_pair(self):
        self._load()
        return self._seg_pair

    def curves(self, drop_coplanar_interior=True):
        """The segments chained into polylines (see curves())."""
        return curves(self.segments, self.seg_pair, self.npairs, drop_coplanar_interior)


class _CurvesOwner:
    """Keeps a gi_curves alive while views of its arrays exist."""

    __slots__ = ("handle",)

    def __init__(self, handle):
        self.handle = handle

    def __del__(self):
        if self.handle:
            lib().gi_curves_free(self.handle)
            self.handle = None


def curves_of_jobs(segments, seg_pair, pair_offsets, drop_coplanar_interior=True):
    """The curves of every job of a batch in one call (gi_curves_build_jobs):
    segments (M, 6) ordered by pair, seg_pair (M,) batch-wide pair indices,
    pair_offsets (njobs + 1,).  Returns flat arrays: vertices (V, 3), curve
    offsets (C + 1,) into idx, idx (vertex ids), closed (C,) flags and
    job_curves (njobs + 1,): job j owns curves job_curves[j] .. job_curves[j + 1].
    The arrays are views of the library's (no copy), released with the last of them."""
    L = lib()
    seg = np.ascontiguousarray(segments, dtype=np.float64).reshape(-1, 6)
    sp = np.ascontiguousarray(seg_pair, dtype=np.int64).reshape(-1)
    po = np.ascontiguousarray(pair_offsets, dtype=np.int64).reshape(-1)
    h = ctypes.c_void_p()
    rc = L.gi_curves_build_jobs(seg.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                sp.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), seg.shape[0],
                                po.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), max(po.shape[0] - 1, 0),
                                1 if drop_coplanar_interior else 0, ctypes.byref(h))
    if rc:
        raise GIError(rc, "gi_curves_build_jobs")
    owner = _CurvesOwner(h)
    addr = lambda ptr: ctypes.cast(ptr, ctypes.c_void_p).value or 0

    def view(ptr, shape, dtype):
        if int(np.prod(shape)) == 0:
            return np.zeros(shape, dtype=dtype)
        return np.asarray(_View(owner, addr(ptr), shape, dtype))

    vp = ctypes.POINTER(ctypes.c_double)()
    nv = ctypes.c_uint64()
    L.gi_curves_vertices(h, ctypes.byref(vp), ctypes.byref(nv))
    off = ctypes.POINTER(ctypes.c_uint64)()
    idx = ctypes.POINTER(ctypes.c_uint32)()
    cl = ctypes.POINTER(ctypes.c_uint8)()
    nc = ctypes.c_uint64()
    L.gi_curves_polylines(h, ctypes.byref(off), ctypes.byref(idx), ctypes.byref(cl), ctypes.byref(nc))
    jo = ctypes.POINTER(ctypes.c_uint64)()
    nj = ctypes.c_uint64()
    L.gi_curves_job_offsets(h, ctypes.byref(jo), ctypes.byref(nj))
    o = view(off, (nc.value + 1,), np.uint64)
    return dict(vertices=view(vp, (nv.value, 3), np.float64), offsets=o,
                idx=view(idx, (int(o[-1]),), np.uint32),
                closed=view(cl, (nc.value,), np.uint8).view(np.bool_),
                job_curves=view(jo, (nj.value + 1,), np.uint64))


class _BatchOwner:
    """Keeps every result handle of a batch alive while views of their shared block exist."""

    __slots__ = ("owners",)

    def __init__(self, owners):
        self.owners = owners


class BatchResult:
    """Whole-batch arrays of one gi_intersect_batch call (see Context.intersect_batch_flat)."""

    def __init__(self, owners):
        L = lib()
        n = len(owners)
        p = ctypes.POINTER(ctypes.c_int32)()
        cnt = ctypes.c_uint64()
        sp = ctypes.POINTER(ctypes.c_double)()
        spp = ctypes.POINTER(ctypes.c_int32)()
        m = ctypes.c_uint64()
        pa, sa, qa = np.zeros(n, np.uint64), np.zeros(n, np.uint64), np.zeros(n, np.uint64)
        npairs, nsegs = np.zeros(n, np.int64), np.zeros(n, np.int64)
        for i, ow in enumerate(owners):
            L.gi_result_pairs(ow.handle, ctypes.byref(p), ctypes.byref(cnt))
            L.gi_result_segments(ow.handle, ctypes.byref(sp), ctypes.byref(spp), ctypes.byref(m))
            pa[i] = ctypes.cast(p, ctypes.c_void_p).value or 0
            sa[i] = ctypes.cast(sp, ctypes.c_void_p).value or 0
            qa[i] = ctypes.cast(spp, ctypes.c_void_p).value or 0
            npairs[i], nsegs[i] = cnt.value, m.value
        self.offsets = np.concatenate([[0], np.cumsum(npairs)]).astype(np.int64)
        soff = np.concatenate([[0], np.cumsum(nsegs)]).astype(np.int64)
        st = _abi.Stats()
        if n:
            L.gi_result_stats(owners[0].handle, ctypes.byref(st))
        self.stats = st.as_dict()
        holder = _BatchOwner(owners)

        def whole(addr, counts, starts, width, dtype):
            total = int(starts[-1])
            item = np.dtype(dtype).itemsize * width
            nz = np.nonzero(counts)[0]
            if total == 0:
                return np.zeros((0, width) if width > 1 else (0,), dtype=dtype)
            shape = (total, width) if width > 1 else (total,)
            first = int(nz[0])
            base = int(addr[first]) - item * int(starts[first])
            if np.all(addr[nz].astype(np.int64) == base + item * starts[nz]):  # back to back in one block
                return np.asarray(_View(holder, base + item * int(starts[0]), shape, dtype))
            parts = [np.asarray(_View(holder, int(addr[i]), (int(counts[i]),) + shape[1:], dtype)) for i in nz]
            return np.concatenate(parts)

        self.pairs = whole(pa, npairs, self.offsets, 2, np.int32)
        self.segments = whole(sa, nsegs, soff, 6, np.float64)
        local = whole(qa, nsegs, soff, 1, np.int32)  # per job, relative to the job's first pair
        self.seg_pair = local.astype(np.int64) + np.repeat(self.offsets[:-1], nsegs)
        self.job = np.repeat(np.arange(n, dtype=np.uint32), npairs)

    def curves(self, drop_coplanar_interior=True):
        """Every job's curves in one call (see curves_of_jobs)."""
        return curves_of_jobs(self.segments, self.seg_pair, self.offsets, drop_coplanar_interior)


class Server:
    """Pose-update serving loop with continuous batching (gi_server_*)."""

    def __init__(self, ctx, max_inflight, want_segments, precision):
        self.ctx = ctx
        o = _abi.ServerOpts()
        o.max_inflight = max_inflight
        o.opts = Context._opts(want_segments, precision, True)
        h = ctypes.c_void_p()
        ctx.check(ctx._lib.gi_server_start(ctx.handle, ctypes.byref(o), ctypes.byref(h)), "gi_server_start")
        self.handle = h

    def submit(self, A, pose_a, B, pose_b):
        t = ctypes.c_uint64()
        self.ctx.check(self.ctx._lib.gi_server_submit(self.handle, A.handle,
                                                      ctypes.byref(pose_a) if pose_a is not None else None,
                                                      B.handle, ctypes.byref(pose_b) if pose_b is not None else None,
                                                      ctypes.byref(t)), "gi_server_submit")
        return t.value

    def poll(self, ticket):
        r = ctypes.c_void_p()
        rc = self.ctx._lib.gi_server_poll(self.handle, ticket, ctypes.byref(r))
        if rc == _abi.GI_ERR_NOT_READY:
            return None
        self.ctx.check(rc, "gi_server_poll")
        return Result(r)

    def wait(self, ticket, timeout_ms=60000):
        r = ctypes.c_void_p()
        rc = self.ctx._lib.gi_server_wait(self.handle, ticket, timeout_ms, ctypes.byref(r))
        self.ctx.check(rc, "gi_server_wait")
        return Result(r)

    def stop(self):
        if self.handle:
            self.ctx._lib.gi_server_stop(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


# ---------------------------------------------------------------- reference-shaped mirrors
class KernelBVHController:
    """Mirror of the reference class (KernelBVHController.h:36-95).

    construct(...) uploads both meshes and builds their BVHs once; the level /
    leafThreshold arguments of the reference's level-cut builder are accepted
    and not needed (the LBVH has no level cut).  setTransformBoth stores the
    Euler poses about the stored centres; runIntersectionPipeline intersects
    under them on the device and returns the (faceA, faceB) pairs as an
    (n, 2) int32 array (the reference returns a malloc'd int2*)."""

    def __init__(self, device=0):
        self.ctx = Context(device)
        self.A = self.B = None
        self.centerA = np.zeros(3)
        self.centerB = np.zeros(3)
        self.rotA = np.zeros(3)
        self.transA = np.zeros(3)
        self.rotB = np.zeros(3)
        self.transB = np.zeros(3)
        self._host = None
        self.last_stats = None

    def construct(self, vertsA, trisA, levelA, vertsB, trisB, levelB, leafThreshold=4, centerA=None,
                  centerB=None):
        self._host = (np.array(vertsA, dtype=np.float64), np.array(trisA, dtype=np.uint32),
                      np.array(vertsB, dtype=np.float64), np.array(trisB, dtype=np.uint32))
        self.clearGPU()
        self.A = self.ctx.upload(self._host[0], self._host[1])
        self.B = self.ctx.upload(self._host[2], self._host[3])
        if centerA is not None:
            self.centerA = np.asarray(centerA, dtype=np.float64)
        if centerB is not None:
            self.centerB = np.asarray(centerB, dtype=np.float64)

    def setTransformBoth(self, rotDegA, transA, rotDegB, transB):
        self.rotA, self.transA = np.asarray(rotDegA, float), np.asarray(transA, float)
        self.rotB, self.transB = np.asarray(rotDegB, float), np.asarray(transB, float)

    def poses(self):
        return (pose_from_euler_deg(self.rotA, self.centerA, self.transA),
                pose_from_euler_deg(self.rotB, self.centerB, self.transB))

    def runIntersectionPipeline(self, batchMultiplier=1, numberOfDualTreeSteps=0, activateAsyncDownload=0,
                                gpuDouble=1, want_segments=False):
        pa, pb = self.poses()
        r = self.ctx.intersect(self.A, self.B, pa, pb, want_segments=want_segments)
        self.last_stats = r.stats
        self.last_result = r
        return r.pairs

    def clearGPU(self):
        for m in (self.A, self.B):
            if m is not None:
                m.release()
        self.A = self.B = None

    def reconstructGPU(self):
        if self._host is not None:
            self.A = self.ctx.upload(self._host[0], self._host[1])
            self.B = self.ctx.upload(self._host[2], self._host[3])

    def cleanup(self):
        self.clearGPU()

    def getCenterA(self):
        return self.centerA

    def getCenterB(self):
        return self.centerB

    def isGPUAllocated(self):
        return self.A is not None and self.B is not None


def run_grid_forest_intersection_pipeline(vertsA, trisA, vertsB, trisB, centerA=(0, 0, 0), centerB=(0, 0, 0),
                                          rotA=(0, 0, 0), transA=(0, 0, 0), rotB=(0, 0, 0), transB=(0, 0, 0),
                                          ctx=None, want_segments=False):
    """One-shot path (StandaloneBVHPipeline.h:27-43): upload, build, intersect, release."""
    own = ctx is None
    ctx = ctx or Context()
    try:
        r = ctx.intersect_oneshot(vertsA, trisA, vertsB, trisB, pose_from_euler_deg(rotA, centerA, transA),
                                  pose_from_euler_deg(rotB, centerB, transB), want_segments=want_segments)
    finally:
        if own:
            ctx.close()
    return r


def compute_exact_intersection_curves(ctx, A, B, pose_a=None, pose_b=None):
    """Segments of the intersecting pairs (MeshIntersectionCurves.h:24-29), on the device."""
    return ctx.intersect(A, B, pose_a, pose_b, want_segments=True).segments
