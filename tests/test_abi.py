"""CPU tests of the C-ABI boundary: libgi.so loads, exports every entry point
include/gi/gi.h declares, and its host-only entry points behave without a GPU."""
import ctypes
import os
import re
import subprocess

import numpy as np

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "gi", "gi.h")


def header_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:gi_status|const char\*)\s+(gi_\w+)\s*\(", src, re.M)))


def test_header_declares_expected_entry_points(gi):
    from gpuintersector import _abi

    assert header_functions() == sorted(_abi.EXPORTED)


def test_library_exports_every_declared_symbol(gi):
    lib = gi.lib()
    for name in header_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", gi._abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (gi_\w+)", out))
    assert set(header_functions()) <= exported


def test_status_strings(gi):
    lib = gi.lib()
    for s in range(9):
        assert lib.gi_status_string(s)
    assert lib.gi_status_string(99) == b"unknown status"


def test_host_only_entry_points(gi, oc):
    p = gi.pose_identity()
    assert p.identity == 1 and list(p.R) == [1, 0, 0, 0, 1, 0, 0, 0, 1]
    o = gi._abi.IntersectOpts()
    assert gi.lib().gi_intersect_opts_default(ctypes.byref(o)) == 0
    assert o.want_segments == 1 and o.sort_output == 1 and o.precision_mode == 0
    # Euler pose identical to the oracle (RotationTools.h:28-53)
    for rot in ([0, 0, 0], [90, 0, 0], [12.5, -7.25, 181.0], [1e-9, 359.0, 45.0]):
        a = gi.pose_from_euler_deg(rot, [1, 2, 3], [0.1, 0.2, 0.3])
        b = oc.pose_from_euler_deg(rot, [1, 2, 3], [0.1, 0.2, 0.3])
        assert list(a.R) == list(b.R)
        assert a.identity == b.identity
    # invalid arguments are reported, not crashed on
    assert gi.lib().gi_pose_identity(None) == 1
    assert gi.lib().gi_result_free(None) == 1


def test_create_without_device_fails_cleanly(gi):
    import torch

    if torch.cuda.is_available():
        return
    n = ctypes.c_int32(-1)
    assert gi.lib().gi_device_count(ctypes.byref(n)) == gi._abi.GI_ERR_NO_DEVICE
    h = ctypes.c_void_p()
    assert gi.lib().gi_create(None, ctypes.byref(h)) == gi._abi.GI_ERR_NO_DEVICE
