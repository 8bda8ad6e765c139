"""ctypes declarations of the C ABI in include/gi/gi.h (libgi.so)."""
import ctypes
import os

_PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG_DIR, "libgi.so")

GI_OK = 0
GI_ERR_INVALID_ARG = 1
GI_ERR_OOM = 2
GI_ERR_CAPACITY = 3
GI_ERR_TIMEOUT = 4
GI_ERR_CUDA = 5
GI_ERR_RANGE = 6
GI_ERR_NOT_READY = 7
GI_ERR_NO_DEVICE = 8

GI_FLAG_TINY_BUFFERS = 1
GI_FLAG_FIXED_SHAPE = 0x100


GI_TRAVERSE_SHAPES = 8


def GI_FLAG_SHAPE(k):
    return (int(k) & 7) << 9


GI_PREC_FP32_CASCADE = 0
GI_PREC_FP64 = 1
GI_NOALLOC_MAX_PAIRS = 1 << 20
GI_PRED_ORIENT3D = 0
GI_PRED_ORIENT2D = 1
GI_SIGN_UNDECIDED = 2
GI_SIGN_NA = 3
GI_BRANCH_INT128 = 0
GI_BRANCH_MULTILIMB = 1
GI_BRANCH_CAPACITY = 2

# every symbol include/gi/gi.h declares (checked by the CPU tests)
EXPORTED = [
    "gi_create", "gi_destroy", "gi_status_string", "gi_last_error", "gi_device_count", "gi_wait_stream",
    "gi_mesh_upload", "gi_mesh_upload_device", "gi_mesh_release", "gi_mesh_info", "gi_mesh_build_ms",
    "gi_pose_identity", "gi_pose_from_euler_deg", "gi_pose_apply",
    "gi_intersect_opts_default", "gi_intersect", "gi_intersect_oneshot", "gi_intersect_batch",
    "gi_classify_pairs", "gi_classify_pairs_noalloc", "gi_predicate_signs",
    "gi_off_load", "gi_off_arrays", "gi_off_free", "gi_scene_load", "gi_mesh_download",
    "gi_curves_build", "gi_result_curves", "gi_curves_vertices", "gi_curves_polylines", "gi_curves_free",
    "gi_curves_build_jobs", "gi_curves_job_offsets",
    "gi_records_write_csv", "gi_pairs_diff", "gi_sweep_poses",
    "gi_result_pairs", "gi_result_segments", "gi_result_stats", "gi_result_free",
    "gi_server_start", "gi_server_submit", "gi_server_poll", "gi_server_wait", "gi_server_stop",
]


class OffReport(ctypes.Structure):
    _fields_ = [("file_vertices", ctypes.c_uint64), ("file_polygons", ctypes.c_uint64),
                ("extra_fan_triangles", ctypes.c_uint64), ("dropped_degenerate", ctypes.c_uint64),
                ("dropped_duplicate", ctypes.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class RecordMesh(ctypes.Structure):
    _fields_ = [("verts_xyz", ctypes.POINTER(ctypes.c_double)), ("nv", ctypes.c_uint32),
                ("tris", ctypes.POINTER(ctypes.c_uint32)), ("nt", ctypes.c_uint32)]


class Scene(ctypes.Structure):
    _fields_ = [("center", ctypes.c_double * 3), ("scale", ctypes.c_double), ("max_span", ctypes.c_double),
                ("center_a", ctypes.c_double * 3), ("center_b", ctypes.c_double * 3)]

    def as_dict(self):
        return dict(center=list(self.center), scale=self.scale, max_span=self.max_span,
                    center_a=list(self.center_a), center_b=list(self.center_b))


class Options(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("flags", ctypes.c_uint32), ("hbm_budget_bytes", ctypes.c_uint64)]


class Pose(ctypes.Structure):
    _fields_ = [("R", ctypes.c_double * 9), ("center", ctypes.c_double * 3), ("trans", ctypes.c_double * 3),
                ("identity", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class IntersectOpts(ctypes.Structure):
    _fields_ = [("want_segments", ctypes.c_int32), ("precision_mode", ctypes.c_int32),
                ("sort_output", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class Stats(ctypes.Structure):
    _fields_ = [("tris_a", ctypes.c_uint64), ("tris_b", ctypes.c_uint64), ("nodes_a", ctypes.c_uint64),
                ("nodes_b", ctypes.c_uint64), ("node_pairs", ctypes.c_uint64), ("candidates", ctypes.c_uint64),
                ("filter_decided", ctypes.c_uint64), ("escalated", ctypes.c_uint64),
                ("exact_signs", ctypes.c_uint64), ("exact_points", ctypes.c_uint64), ("pairs", ctypes.c_uint64),
                ("segments", ctypes.c_uint64), ("levels", ctypes.c_uint32), ("retries", ctypes.c_uint32),
                ("launches", ctypes.c_uint32), ("traverse_shape", ctypes.c_uint32),
                ("ms_traverse", ctypes.c_double), ("ms_exact", ctypes.c_double), ("ms_segments", ctypes.c_double),
                ("ms_sort", ctypes.c_double), ("ms_total", ctypes.c_double),
                ("level_times", ctypes.c_uint32), ("reserved2", ctypes.c_uint32),
                ("level_end_ms", ctypes.c_double * 32),
                ("finish_phases", ctypes.c_uint32), ("reserved3", ctypes.c_uint32),
                ("finish_ms", ctypes.c_double * 4)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_
             if k not in ("level_end_ms", "reserved2", "finish_ms", "reserved3")}
        d["level_end_ms"] = [self.level_end_ms[i] for i in range(min(self.level_times, 32))]
        d["finish_ms"] = [self.finish_ms[i] for i in range(min(self.finish_phases, 4))]
        return d


class PairJob(ctypes.Structure):
    _fields_ = [("A", ctypes.c_void_p), ("B", ctypes.c_void_p), ("pose_a", Pose), ("pose_b", Pose)]


class ServerOpts(ctypes.Structure):
    _fields_ = [("max_inflight", ctypes.c_uint32), ("flags", ctypes.c_uint32), ("opts", IntersectOpts)]


_lib = None


def load(path=None):
    """Load libgi.so.  Raises if it is missing: there is no fallback path."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError("libgi.so not built (%s); run __graft_entry__.build() or make in %s" % (p, _PKG_DIR))
    L = ctypes.CDLL(p)
    vp = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    up = ctypes.POINTER(ctypes.c_uint32)
    st = ctypes.c_int
    sig = {
        "gi_create": ([ctypes.POINTER(Options), ctypes.POINTER(vp)], st),
        "gi_destroy": ([vp], st),
        "gi_status_string": ([ctypes.c_int], ctypes.c_char_p),
        "gi_last_error": ([vp], ctypes.c_char_p),
        "gi_device_count": ([ctypes.POINTER(ctypes.c_int32)], st),
        "gi_wait_stream": ([vp, vp], st),
        "gi_mesh_upload": ([vp, dp, ctypes.c_uint32, up, ctypes.c_uint32, ctypes.POINTER(vp)], st),
        "gi_mesh_upload_device": ([vp, vp, ctypes.c_uint32, vp, ctypes.c_uint32, ctypes.POINTER(vp)], st),
        "gi_mesh_release": ([vp, vp], st),
        "gi_mesh_info": ([vp, up, up, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)], st),
        "gi_mesh_build_ms": ([vp, dp], st),
        "gi_pose_identity": ([ctypes.POINTER(Pose)], st),
        "gi_pose_from_euler_deg": ([dp, dp, dp, ctypes.POINTER(Pose)], st),
        "gi_pose_apply": ([ctypes.POINTER(Pose), dp, ctypes.c_uint64, dp], st),
        "gi_intersect_opts_default": ([ctypes.POINTER(IntersectOpts)], st),
        "gi_intersect": ([vp, vp, ctypes.POINTER(Pose), vp, ctypes.POINTER(Pose), ctypes.POINTER(IntersectOpts),
                          ctypes.POINTER(vp)], st),
        "gi_intersect_oneshot": ([vp, dp, ctypes.c_uint32, up, ctypes.c_uint32, ctypes.POINTER(Pose),
                                  dp, ctypes.c_uint32, up, ctypes.c_uint32, ctypes.POINTER(Pose),
                                  ctypes.POINTER(IntersectOpts), ctypes.POINTER(vp)], st),
        "gi_intersect_batch": ([vp, ctypes.POINTER(PairJob), ctypes.c_uint32, ctypes.POINTER(IntersectOpts),
                                ctypes.POINTER(vp)], st),
        "gi_classify_pairs": ([vp, vp, ctypes.POINTER(Pose), vp, ctypes.POINTER(Pose), vp, ctypes.c_uint32,
                               ctypes.c_int32, vp], st),
        "gi_classify_pairs_noalloc": ([vp, vp, ctypes.POINTER(Pose), vp, ctypes.POINTER(Pose), vp, ctypes.c_uint32,
                                       ctypes.c_int32, vp], st),
        "gi_predicate_signs": ([vp, ctypes.c_int32, dp, ctypes.POINTER(ctypes.c_int32), ctypes.c_uint64,
                                ctypes.POINTER(ctypes.c_int8)], st),
        "gi_off_load": ([ctypes.c_char_p, ctypes.c_uint32, ctypes.POINTER(vp), ctypes.POINTER(OffReport)], st),
        "gi_off_arrays": ([vp, ctypes.POINTER(dp), ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(up),
                           ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(up)], st),
        "gi_off_free": ([vp], st),
        "gi_scene_load": ([vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(vp),
                           ctypes.POINTER(vp), ctypes.POINTER(Scene), ctypes.POINTER(OffReport),
                           ctypes.POINTER(OffReport)], st),
        "gi_mesh_download": ([vp, dp], st),
        "gi_curves_build": ([dp, ctypes.POINTER(ctypes.c_int32), ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int32,
                             ctypes.POINTER(vp)], st),
        "gi_result_curves": ([vp, ctypes.c_int32, ctypes.POINTER(vp)], st),
        "gi_curves_vertices": ([vp, ctypes.POINTER(dp), ctypes.POINTER(ctypes.c_uint64)], st),
        "gi_curves_polylines": ([vp, ctypes.POINTER(ctypes.POINTER(ctypes.c_uint64)), ctypes.POINTER(up),
                                 ctypes.POINTER(ctypes.POINTER(ctypes.c_uint8)), ctypes.POINTER(ctypes.c_uint64)], st),
        "gi_curves_free": ([vp], st),
        "gi_curves_build_jobs": ([dp, ctypes.POINTER(ctypes.c_int64), ctypes.c_uint64, ctypes.POINTER(ctypes.c_int64),
                                  ctypes.c_uint32, ctypes.c_int32, ctypes.POINTER(vp)], st),
        "gi_curves_job_offsets": ([vp, ctypes.POINTER(ctypes.POINTER(ctypes.c_uint64)), ctypes.POINTER(ctypes.c_uint64)],
                                  st),
        "gi_records_write_csv": ([ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_char_p,
                                  ctypes.POINTER(RecordMesh), ctypes.POINTER(RecordMesh),
                                  ctypes.POINTER(ctypes.c_int32), ctypes.c_uint64, ctypes.c_uint32], st),
        "gi_sweep_poses": ([ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double, ctypes.c_double, dp, dp, dp, dp], st),
        "gi_pairs_diff": ([ctypes.POINTER(ctypes.c_int32), ctypes.c_uint64, ctypes.POINTER(ctypes.c_int32),
                           ctypes.c_uint64, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_uint64),
                           ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_uint64),
                           ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_uint64)], st),
        "gi_result_pairs": ([vp, ctypes.POINTER(ctypes.POINTER(ctypes.c_int32)), ctypes.POINTER(ctypes.c_uint64)], st),
        "gi_result_segments": ([vp, ctypes.POINTER(dp), ctypes.POINTER(ctypes.POINTER(ctypes.c_int32)),
                                ctypes.POINTER(ctypes.c_uint64)], st),
        "gi_result_stats": ([vp, ctypes.POINTER(Stats)], st),
        "gi_result_free": ([vp], st),
        "gi_server_start": ([vp, ctypes.POINTER(ServerOpts), ctypes.POINTER(vp)], st),
        "gi_server_submit": ([vp, vp, ctypes.POINTER(Pose), vp, ctypes.POINTER(Pose),
                              ctypes.POINTER(ctypes.c_uint64)], st),
        "gi_server_poll": ([vp, ctypes.c_uint64, ctypes.POINTER(vp)], st),
        "gi_server_wait": ([vp, ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(vp)], st),
        "gi_server_stop": ([vp], st),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L
