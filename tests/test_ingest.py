"""Mesh ingestion: OFF loading (host, no device needed) and scene normalisation
on the device, against the reference's rules (src/CPU/RobustOffLoader.h:120-186,
apps/mainApplication.cpp:166-187, 637-680) restated in numpy."""
import numpy as np
import pytest

from conftest import oracle_pose


def _write_off(path, verts, faces, header="OFF", counts_on_header=False, crlf=False, comments=True, colors=False):
    nl = "\r\n" if crlf else "\n"
    out = []
    if counts_on_header:
        out.append("%s %d %d 0" % (header, len(verts), len(faces)))
    else:
        out.append(header)
        if comments:
            out.append("# a comment line")
            out.append("")
        out.append("%d %d 0" % (len(verts), len(faces)))
    for v in verts:
        out.append(" ".join(repr(float(x)) for x in v) + (" 0.5 0.5 0.5 1" if colors else ""))
        if comments:
            out.append("   # between vertices")
    for f in faces:
        out.append("%d %s" % (len(f), " ".join(str(int(i)) for i in f)) + (" 255 0 0" if colors else ""))
    open(path, "w", newline="").write(nl.join(out) + nl)


def _reference_triangles(faces):
    """Fan triangulation, repeated-index and duplicate removal, as the reference."""
    tris, rows, seen, degen, extra, dup = [], [], set(), 0, 0, 0
    for r, p in enumerate(faces):
        if len(p) < 3:
            degen += 1
            continue
        for k in range(1, len(p) - 1):
            t = (p[0], p[k], p[k + 1])
            if k > 1:
                extra += 1
            if len(set(t)) < 3:
                degen += 1
                continue
            key = tuple(sorted(t))
            if key in seen:
                dup += 1
                continue
            seen.add(key)
            tris.append(t)
            rows.append(r)
    return np.array(tris, dtype=np.uint32).reshape(-1, 3), np.array(rows, dtype=np.uint32), degen, extra, dup


@pytest.mark.parametrize("variant", [dict(), dict(counts_on_header=True), dict(crlf=True), dict(comments=False),
                                     dict(header="COFF", colors=True)])
def test_off_polygons_degenerate_duplicates(gi, tmp_path, variant):
    rng = np.random.default_rng(1)
    verts = rng.normal(size=(12, 3)) * 1e3
    faces = [(0, 1, 2), (2, 1, 0), (3, 4, 5, 6), (7, 8, 9, 10, 11), (1, 1, 2), (4, 5), (0, 2, 1),
             (5, 6, 7), (3, 3, 4, 5), (8, 9, 10)]
    p = tmp_path / "m.off"
    _write_off(p, verts, faces, **variant)
    v, t, rows, rep = gi.load_off(str(p))
    et, erows, edeg, eextra, edup = _reference_triangles(faces)
    assert np.array_equal(v, verts)  # exact: repr() round trips
    assert np.array_equal(t, et) and np.array_equal(rows, erows)
    assert rep["file_vertices"] == 12 and rep["file_polygons"] == len(faces)
    assert rep["extra_fan_triangles"] == eextra
    assert rep["dropped_degenerate"] == edeg
    assert rep["dropped_duplicate"] == edup == 3  # (2,1,0), (0,2,1), and (3,4,5) from the degenerate quad


def test_off_large_roundtrip_and_threads(gi, tmp_path):
    from gpuintersector import meshgen as mg

    u, t = mg.geodesic_sphere(100)  # 200k triangles
    verts = mg.displace(u, mg.displacement_params(np.random.default_rng(2)))
    p = tmp_path / "big.off"
    _write_off(p, verts, t.tolist(), comments=False)
    for nthreads in (1, 0):
        v, tt, rows, rep = gi.load_off(str(p), nthreads=nthreads)
        assert np.array_equal(v, verts) and np.array_equal(tt, t)
        assert np.array_equal(rows, np.arange(t.shape[0], dtype=np.uint32))
        assert rep["dropped_duplicate"] == rep["dropped_degenerate"] == 0


def test_off_errors(gi, tmp_path):
    bad = {"noheader.off": "3 1 0\n0 0 0\n1 0 0\n0 1 0\n3 0 1 2\n",
           "range.off": "OFF\n3 1 0\n0 0 0\n1 0 0\n0 1 0\n3 0 1 7\n",
           "short.off": "OFF\n4 2 0\n0 0 0\n1 0 0\n0 1 0\n",
           "badnum.off": "OFF\n3 1 0\n0 0 x\n1 0 0\n0 1 0\n3 0 1 2\n"}
    for name, text in bad.items():
        (tmp_path / name).write_text(text)
        with pytest.raises(gi.GIError) as e:
            gi.load_off(str(tmp_path / name))
        assert e.value.status == 1
    with pytest.raises(gi.GIError):
        gi.load_off(str(tmp_path / "missing.off"))


@pytest.mark.gpu
def test_scene_load_normalise_and_intersect(gi, oc, tmp_path):
    """load_scene: normalised vertices bit-identical to (x - c) * s with the
    reference's centre and scale, rotation centres the normalised box centres,
    and an intersect under Euler poses about them equal to the oracle."""
    from gpuintersector import meshgen as mg

    cfg = mg.config1(seed=4)
    vA = cfg["vA"] * 37.5 + np.array([1000.0, -20.0, 3.25])
    vB = cfg["vB"] * 37.5 + np.array([1018.0, -20.0, 3.25])
    pa, pb = tmp_path / "a.off", tmp_path / "b.off"
    _write_off(pa, vA, cfg["tA"].tolist(), comments=False)
    _write_off(pb, vB, cfg["tB"].tolist(), comments=False)
    for unit in (True, False):
        with gi.Context(0) as ctx:
            A, B, sc, ra, rb = ctx.load_scene(str(pa), str(pb), scale_to_unit=unit)
            lo = np.minimum(vA.min(0), vB.min(0))
            hi = np.maximum(vA.max(0), vB.max(0))
            c = 0.5 * (lo + hi)
            span = float((hi - lo).max())
            s = 2.0 / span if unit else 1.0
            nA, nB = (vA - c) * s, (vB - c) * s
            assert np.array_equal(np.array(sc["center"]), c) and sc["scale"] == s and sc["max_span"] == span
            assert np.array_equal(A.download(), nA) and np.array_equal(B.download(), nB)
            assert np.array_equal(np.array(sc["center_a"]), 0.5 * (nA.min(0) + nA.max(0)))
            assert np.array_equal(np.array(sc["center_b"]), 0.5 * (nB.min(0) + nB.max(0)))
            rot, tr = (10.0, -25.0, 40.0), (0.01, 0.0, -0.02)
            pose_b = gi.pose_from_euler_deg(rot, sc["center_b"], tr)
            r = ctx.intersect(A, B, None, pose_b)
            ob = oc.pose_from_euler_deg(rot, sc["center_b"], tr)
            ref = oc.intersect_meshes(nA, cfg["tA"], oc.pose_identity(), nB, cfg["tB"], ob, want_segments=True)
            assert np.array_equal(r.pairs, ref["pairs"]) and len(ref["pairs"]) > 0
            A.release()
            B.release()
