"""Shared fixtures.  `-m gpu` tests need a CUDA device and call libgi.so through
its C ABI; everything else runs on the CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gpu-cubql-intersector-standalone_b200")
for p in (PKG, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libgi.so")


@pytest.fixture(scope="session")
def oc():
    import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def gi():
    import gpuintersector

    return gpuintersector


@pytest.fixture(scope="session")
def ctx(gi):
    c = gi.Context(0)
    yield c
    c.close()


def canonical(segs, seg_pair):
    """Segments with lexicographically ordered endpoints, rows sorted by (pair, p0, p1)."""
    from __graft_entry__ import canonical_segments

    return canonical_segments(segs, seg_pair)


def oracle_pose(oc, p):
    if p is None:
        return oc.pose_identity()
    R, C, T = p
    return oc.pose_raw(R, C, T)


def gi_pose(gi, p):
    if p is None:
        return None
    R, C, T = p
    return gi.pose_raw(R, C, T)
