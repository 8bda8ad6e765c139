"""Mesh uploads from host memory and the two-stream one-shot call.

Large pageable sources are copied through pinned chunks filled by the
context's copy helpers; pinned sources go straight to the DMA engine; the
one-shot call builds its second mesh on a helper thread and a second stream.
These tests pin the bytes that arrive on the device and the error paths."""
import numpy as np
import pytest

# vertex counts around the staging threshold (8 MB of vertices) and the 4 MB chunks
SIZES = [349525, 349526, 524288, 699051]


def _mesh(rng, nv):
    v = rng.uniform(-1.0, 1.0, (nv, 3))
    v[::7] *= 1e-3  # a spread of magnitudes
    v[5] = (-0.0, 0.0, 2.0 ** -90)
    i = np.arange(nv, dtype=np.uint32)
    t = np.stack([i, (i + 1) % nv, (i + 2) % nv], 1).astype(np.uint32)
    return v, t


def _pinned(a):
    import torch

    dt = {np.dtype(np.float64): torch.float64, np.dtype(np.uint32): torch.int32}[a.dtype]
    h = torch.empty(a.shape, dtype=dt, pin_memory=True)
    h.numpy().view(a.dtype)[...] = a
    return h, h.numpy().view(a.dtype)


@pytest.mark.gpu
@pytest.mark.parametrize("nv", SIZES)
def test_upload_bytes_pageable_and_pinned(ctx, gi, nv):
    rng = np.random.default_rng(nv)
    v, t = _mesh(rng, nv)
    hold_v, pv = _pinned(v)
    hold_t, pt = _pinned(t)
    for src_v, src_t in ((v, t), (pv, pt)):
        m = ctx.upload(src_v, src_t)
        got = m.download()
        assert np.array_equal(got.view(np.uint64), v.view(np.uint64))  # bit for bit, -0.0 included
        info = m.info()
        assert info["nv"] == nv and info["nt"] == nv
        m.release()


@pytest.mark.gpu
def test_pageable_and_pinned_uploads_intersect_alike(ctx, gi):
    from gpuintersector import meshgen as mg

    c = mg.config2(level=6)
    hv, pv = _pinned(np.ascontiguousarray(c["vB"]))
    ht, pt = _pinned(np.ascontiguousarray(c["tB"], dtype=np.uint32))
    pose = gi.pose_raw(*c["poseB"])
    r1 = ctx.intersect_oneshot(c["vA"], c["tA"], c["vB"], c["tB"], None, pose)
    r2 = ctx.intersect_oneshot(c["vA"], c["tA"], pv, pt, None, pose)
    A, B = ctx.upload(c["vA"], c["tA"]), ctx.upload(pv, pt)
    r3 = ctx.intersect(A, B, None, pose)
    assert len(r1.pairs) > 0
    assert np.array_equal(r1.pairs, r2.pairs) and np.array_equal(r1.pairs, r3.pairs)
    assert np.array_equal(r1.segments, r3.segments)
    A.release()
    B.release()


@pytest.mark.gpu
def test_oneshot_error_on_either_mesh_leaves_context_usable(ctx, gi):
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], float)
    good = np.array([[0, 1, 2]], np.uint32)
    bad = np.array([[0, 1, 7]], np.uint32)
    far = np.array([[0, 0, np.inf], [1, 0, 0], [0, 1, 0]])
    for args, status in (((v, bad, v, good), 1), ((v, good, v, bad), 1), ((v, bad, v, bad), 1),
                         ((v, good, far, good), 6), ((far, good, v, good), 6)):
        with pytest.raises(gi.GIError) as e:
            ctx.intersect_oneshot(*args)
        assert e.value.status == status
    # the context (both of its streams) still works
    w = v + np.array([0.25, 0.25, 0.0])
    r = ctx.intersect_oneshot(v, good, w, good)
    A, B = ctx.upload(v, good), ctx.upload(w, good)
    r2 = ctx.intersect(A, B)
    assert len(r.pairs) == 1 and np.array_equal(r.pairs, r2.pairs)
    A.release()
    B.release()


@pytest.mark.parametrize("nv", [1, 2, 3, 4, 7, 8, 1001])
def test_vertex_vector_reads_stay_in_the_padding(nv):
    """The build's box kernel reads vertex i as the two aligned 16-byte vectors
    that hold it (load_vertex in csrc/gi_classify.cuh): doubles [o & ~1, (o & ~1) + 4)
    with o = 3i, the vertex being the first three of them for even i and the
    last three for odd i.  A restatement of that arithmetic on the CPU: every
    vertex comes out right, each vector starts on a 16-byte boundary, and no read
    passes the 16 bytes (two doubles) of padding that mesh uploads allocate after
    the last vertex."""
    rng = np.random.default_rng(nv)
    v = rng.uniform(-1.0, 1.0, (nv, 3))
    flat = np.concatenate([v.ravel(), [np.nan, np.nan]])  # the padding
    for i in range(nv):
        base = (3 * i) & ~1
        assert (8 * base) % 16 == 0
        assert base + 4 <= 3 * nv + 2
        a, b = flat[base:base + 2], flat[base + 2:base + 4]
        got = (a[1], b[0], b[1]) if i & 1 else (a[0], a[1], b[0])
        assert np.array_equal(np.array(got), v[i])
