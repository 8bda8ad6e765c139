"""ctypes binding of the CPU exact oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py import this module, as the checker.  The product
path (the CUDA library) never calls it.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

NONE, POINT, SEGMENT, TRIANGLE, POLYGON = 0, 1, 2, 3, 4


class Pose(ctypes.Structure):
    _fields_ = [("R", ctypes.c_double * 9), ("C", ctypes.c_double * 3), ("T", ctypes.c_double * 3),
                ("identity", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("candidates", ctypes.c_uint64), ("pairs", ctypes.c_uint64), ("segments", ctypes.c_uint64),
                ("filter_failures", ctypes.c_uint64), ("ms_total", ctypes.c_double)]


def build(force=False):
    """Compile liboracle.so with its Makefile (gcc)."""
    if force or not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) < max(os.path.getmtime(os.path.join(_HERE, f))
                                              for f in ("gi_oracle.c", "gi_oracle.h"))):
        subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        up = ctypes.POINTER(ctypes.c_uint32)
        L.oc_orient3d.argtypes = [dp, dp, dp, dp]
        L.oc_orient3d.restype = ctypes.c_int
        L.oc_orient2d.argtypes = [dp, dp, dp, ctypes.c_int]
        L.oc_orient2d.restype = ctypes.c_int
        L.oc_tri_tri_intersect.argtypes = [dp, dp]
        L.oc_tri_tri_intersect.restype = ctypes.c_int
        L.oc_tri_tri_construct.argtypes = [dp, dp, dp, ctypes.POINTER(ctypes.c_int)]
        L.oc_tri_tri_construct.restype = ctypes.c_int
        L.oc_pose_from_euler_deg.argtypes = [dp, dp, dp, ctypes.POINTER(Pose)]
        L.oc_pose_identity.argtypes = [ctypes.POINTER(Pose)]
        L.oc_transform_vertices.argtypes = [ctypes.POINTER(Pose), dp, ctypes.c_size_t, dp]
        L.oc_intersect_meshes.argtypes = [
            dp, ctypes.c_uint32, up, ctypes.c_uint32, ctypes.POINTER(Pose),
            dp, ctypes.c_uint32, up, ctypes.c_uint32, ctypes.POINTER(Pose),
            ctypes.c_int, ctypes.c_int, ctypes.c_uint32,
            ctypes.POINTER(ctypes.POINTER(ctypes.c_int32)), ctypes.POINTER(ctypes.c_uint64),
            ctypes.POINTER(dp), ctypes.POINTER(ctypes.POINTER(ctypes.c_int32)), ctypes.POINTER(ctypes.c_uint64),
            ctypes.POINTER(Stats)]
        L.oc_intersect_meshes.restype = ctypes.c_int
        L.oc_intersect_meshes_bruteforce.argtypes = [
            dp, ctypes.c_uint32, up, ctypes.c_uint32, ctypes.POINTER(Pose),
            dp, ctypes.c_uint32, up, ctypes.c_uint32, ctypes.POINTER(Pose),
            ctypes.POINTER(ctypes.POINTER(ctypes.c_int32)), ctypes.POINTER(ctypes.c_uint64)]
        L.oc_intersect_meshes_bruteforce.restype = ctypes.c_int
        L.oc_classify_pairs.argtypes = [
            dp, ctypes.c_uint32, up, ctypes.c_uint32, ctypes.POINTER(Pose),
            dp, ctypes.c_uint32, up, ctypes.c_uint32, ctypes.POINTER(Pose),
            ctypes.POINTER(ctypes.c_int32), ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint8), ctypes.c_int]
        L.oc_classify_pairs.restype = ctypes.c_int
        L.oc_free.argtypes = [ctypes.c_void_p]
        L.oc_sign_log_begin.argtypes = [ctypes.c_uint64]
        L.oc_sign_log_begin.restype = ctypes.c_int
        L.oc_sign_log_end.argtypes = [ctypes.POINTER(dp), ctypes.POINTER(ctypes.POINTER(ctypes.c_int32))]
        L.oc_sign_log_end.restype = ctypes.c_uint64
        L.oc_hw_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _up(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def pose_identity():
    p = Pose()
    lib().oc_pose_identity(ctypes.byref(p))
    return p


def pose_from_euler_deg(rot, center, trans):
    p = Pose()
    r = np.ascontiguousarray(rot, dtype=np.float64)
    c = np.ascontiguousarray(center, dtype=np.float64)
    t = np.ascontiguousarray(trans, dtype=np.float64)
    lib().oc_pose_from_euler_deg(_dp(r), _dp(c), _dp(t), ctypes.byref(p))
    return p


def pose_raw(R, C, T, identity=False):
    p = Pose()
    for i in range(9):
        p.R[i] = float(np.asarray(R, dtype=np.float64).reshape(9)[i])
    for i in range(3):
        p.C[i] = float(C[i])
        p.T[i] = float(T[i])
    p.identity = 1 if identity else 0
    return p


def transform(pose, verts):
    v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 3)
    out = np.empty_like(v)
    lib().oc_transform_vertices(ctypes.byref(pose), _dp(v), v.shape[0], _dp(out))
    return out


def orient3d(a, b, c, d):
    arr = [np.ascontiguousarray(x, dtype=np.float64) for x in (a, b, c, d)]
    return lib().oc_orient3d(*[_dp(x) for x in arr])


def orient2d(a, b, c, drop):
    arr = [np.ascontiguousarray(x, dtype=np.float64) for x in (a, b, c)]
    return lib().oc_orient2d(*[_dp(x) for x in arr], int(drop))


def record_signs(fn, cap=1 << 22):
    """Runs fn() with the oracle's sign log on: every orient3d / orient2d call it
    makes is returned with its exact sign as (pts (n, 12) float64, kind (n,),
    drop (n,), sign (n,)), plus fn's return value.  Use nthreads=1 inside fn so
    that the calls are logged in order."""
    L = lib()
    if L.oc_sign_log_begin(int(cap)) != 0:
        raise MemoryError("oc_sign_log_begin")
    pp = ctypes.POINTER(ctypes.c_double)()
    mp = ctypes.POINTER(ctypes.c_int32)()
    try:
        ret = fn()
    finally:
        n = L.oc_sign_log_end(ctypes.byref(pp), ctypes.byref(mp))
    pts = np.ctypeslib.as_array(pp, shape=(n * 12,)).reshape(n, 12).copy() if n else np.zeros((0, 12))
    meta = np.ctypeslib.as_array(mp, shape=(n * 3,)).reshape(n, 3).copy() if n else np.zeros((0, 3), np.int32)
    L.oc_free(ctypes.cast(pp, ctypes.c_void_p))
    L.oc_free(ctypes.cast(mp, ctypes.c_void_p))
    return (pts, meta[:, 0], meta[:, 1], meta[:, 2]), ret


def tri_tri_intersect(t1, t2):
    a = np.ascontiguousarray(t1, dtype=np.float64).reshape(9)
    b = np.ascontiguousarray(t2, dtype=np.float64).reshape(9)
    return bool(lib().oc_tri_tri_intersect(_dp(a), _dp(b)))


def tri_tri_construct(t1, t2):
    a = np.ascontiguousarray(t1, dtype=np.float64).reshape(9)
    b = np.ascontiguousarray(t2, dtype=np.float64).reshape(9)
    pts = np.zeros(18, dtype=np.float64)
    n = ctypes.c_int(0)
    kind = lib().oc_tri_tri_construct(_dp(a), _dp(b), _dp(pts), ctypes.byref(n))
    return kind, [tuple(pts[3 * i:3 * i + 3]) for i in range(n.value)]


def intersect_meshes(vA, tA, pA, vB, tB, pB, want_segments=True, nthreads=0, a_limit=0):
    """Returns dict(pairs=(n,2) int32 sorted, segs=(m,6), seg_pair=(m,), stats=Stats)."""
    L = lib()
    vA = np.ascontiguousarray(vA, dtype=np.float64).reshape(-1, 3)
    vB = np.ascontiguousarray(vB, dtype=np.float64).reshape(-1, 3)
    tA = np.ascontiguousarray(tA, dtype=np.uint32).reshape(-1, 3)
    tB = np.ascontiguousarray(tB, dtype=np.uint32).reshape(-1, 3)
    pp = ctypes.POINTER(ctypes.c_int32)()
    npairs = ctypes.c_uint64(0)
    sp = ctypes.POINTER(ctypes.c_double)()
    spp = ctypes.POINTER(ctypes.c_int32)()
    nseg = ctypes.c_uint64(0)
    st = Stats()
    rc = L.oc_intersect_meshes(_dp(vA), vA.shape[0], _up(tA), tA.shape[0], ctypes.byref(pA),
                               _dp(vB), vB.shape[0], _up(tB), tB.shape[0], ctypes.byref(pB),
                               1 if want_segments else 0, int(nthreads), int(a_limit),
                               ctypes.byref(pp), ctypes.byref(npairs), ctypes.byref(sp), ctypes.byref(spp),
                               ctypes.byref(nseg), ctypes.byref(st))
    if rc != 0:
        raise RuntimeError("oc_intersect_meshes failed: %d" % rc)
    n = npairs.value
    pairs = (np.ctypeslib.as_array(pp, shape=(n * 2,)).reshape(n, 2).copy() if n
             else np.zeros((0, 2), dtype=np.int32))
    if pp:
        L.oc_free(ctypes.cast(pp, ctypes.c_void_p))
    segs = np.zeros((0, 6))
    seg_pair = np.zeros((0,), dtype=np.int32)
    m = nseg.value
    if want_segments and m:
        segs = np.ctypeslib.as_array(sp, shape=(m * 6,)).reshape(m, 6).copy()
        seg_pair = np.ctypeslib.as_array(spp, shape=(m,)).copy()
    if sp:
        L.oc_free(ctypes.cast(sp, ctypes.c_void_p))
    if spp:
        L.oc_free(ctypes.cast(spp, ctypes.c_void_p))
    return dict(pairs=pairs, segs=segs, seg_pair=seg_pair, stats=st)


def classify_pairs(vA, tA, pA, vB, tB, pB, pairs, nthreads=0):
    """Exact test of each (a, b) of a pair list on host threads: uint8 per pair."""
    vA = np.ascontiguousarray(vA, dtype=np.float64).reshape(-1, 3)
    vB = np.ascontiguousarray(vB, dtype=np.float64).reshape(-1, 3)
    tA = np.ascontiguousarray(tA, dtype=np.uint32).reshape(-1, 3)
    tB = np.ascontiguousarray(tB, dtype=np.uint32).reshape(-1, 3)
    p = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
    out = np.empty(p.shape[0], dtype=np.uint8)
    rc = lib().oc_classify_pairs(_dp(vA), vA.shape[0], _up(tA), tA.shape[0], ctypes.byref(pA),
                                 _dp(vB), vB.shape[0], _up(tB), tB.shape[0], ctypes.byref(pB),
                                 p.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), p.shape[0],
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), int(nthreads))
    if rc != 0:
        raise ValueError("oc_classify_pairs: index out of range")
    return out


def intersect_meshes_bruteforce(vA, tA, pA, vB, tB, pB):
    L = lib()
    vA = np.ascontiguousarray(vA, dtype=np.float64).reshape(-1, 3)
    vB = np.ascontiguousarray(vB, dtype=np.float64).reshape(-1, 3)
    tA = np.ascontiguousarray(tA, dtype=np.uint32).reshape(-1, 3)
    tB = np.ascontiguousarray(tB, dtype=np.uint32).reshape(-1, 3)
    pp = ctypes.POINTER(ctypes.c_int32)()
    npairs = ctypes.c_uint64(0)
    L.oc_intersect_meshes_bruteforce(_dp(vA), vA.shape[0], _up(tA), tA.shape[0], ctypes.byref(pA),
                                     _dp(vB), vB.shape[0], _up(tB), tB.shape[0], ctypes.byref(pB),
                                     ctypes.byref(pp), ctypes.byref(npairs))
    n = npairs.value
    pairs = (np.ctypeslib.as_array(pp, shape=(n * 2,)).reshape(n, 2).copy() if n
             else np.zeros((0, 2), dtype=np.int32))
    if pp:
        L.oc_free(ctypes.cast(pp, ctypes.c_void_p))
    return pairs


def hw_threads():
    return lib().oc_hw_threads()
