"""Intersection curves: segments chained into polylines (gi_curves_build),
against an independent restatement of the rules in Python."""
import numpy as np
import pytest


def _canon(verts, curves):
    """Curves as coordinate tuples: closed loops up to rotation and direction,
    open chains up to direction; a sorted list."""
    out = []
    for idx, closed in curves:
        pts = [tuple(verts[i]) for i in idx]
        if closed:
            cands = []
            for seq in (pts, pts[::-1]):
                for r in range(len(seq)):
                    cands.append(tuple(seq[r:] + seq[:r]))
            out.append(("c", min(cands)))
        else:
            out.append(("o", min(tuple(pts), tuple(pts[::-1]))))
    return sorted(out)


def _reference(segs, seg_pair, npairs, drop=True):
    """The same rules in plain Python (dicts and lists)."""
    key = lambda p: tuple(0.0 if x == 0.0 else float(x) for x in p)
    per_pair = [0] * npairs
    for k in seg_pair:
        per_pair[k] += 1
    vid, verts, edges = {}, [], {}

    def vertex(p):
        k = key(p)
        if k not in vid:
            vid[k] = len(verts)
            verts.append(k)
        return vid[k]

    for s, k in zip(segs, seg_pair):
        u, v = vertex(s[:3]), vertex(s[3:])
        if u == v:
            continue
        e = edges.setdefault((min(u, v), max(u, v)), [0, 0])
        e[0 if per_pair[k] == 3 else 1] += 1
    el = sorted(e for e, (cop, oth) in edges.items() if not (drop and oth == 0 and cop >= 2))
    adj = {v: [] for v in range(len(verts))}
    for i, (a, b) in enumerate(el):
        adj[a].append((b, i))
        adj[b].append((a, i))
    used, curves = set(), []

    def walk(v0, first):
        seq, (w, e) = [v0], first
        while True:
            used.add(e)
            if w == v0 and len(adj[v0]) == 2:
                return seq, True
            seq.append(w)
            if len(adj[w]) != 2:
                return seq, False
            nxt = [x for x in adj[w] if x[1] not in used]
            if not nxt:
                return seq, False
            w, e = nxt[0]

    for v in range(len(verts)):
        if len(adj[v]) == 0:
            curves.append(([v], False))
        elif len(adj[v]) != 2:
            for x in adj[v]:
                if x[1] not in used:
                    curves.append(walk(v, x))
    for v in range(len(verts)):
        for x in adj[v]:
            if x[1] not in used:
                curves.append(walk(v, x))
    return np.array(verts), curves


def _soup(rng):
    """A random soup: closed loops, open chains, a branch, points, coplanar outlines."""
    segs, pairs = [], []
    base = 0

    def add(p, q, pair):
        segs.append(list(p) + list(q))
        pairs.append(pair)

    pts = rng.normal(size=(200, 3)).round(3)
    # loops and chains, random directions, with duplicated edges
    for L, closed in ((5, True), (7, True), (4, False), (6, False)):
        ids = list(range(base, base + L))
        base += L
        ring = ids + ids[:1] if closed else ids
        for a, b in zip(ring[:-1], ring[1:]):
            p, q = (pts[a], pts[b]) if rng.random() < 0.5 else (pts[b], pts[a])
            add(p, q, len(pairs))
        add(pts[ring[0]], pts[ring[1]], len(pairs))  # duplicate of an edge
    # a branch point (degree 3)
    c = pts[base]
    for k in range(1, 4):
        add(c, pts[base + k], len(pairs))
    base += 4
    # touching points, one of them at -0.0 vs 0.0
    add([0.0, 1.0, 2.0], [0.0, 1.0, 2.0], len(pairs))
    add([-0.0, 1.0, 2.0], [-0.0, 1.0, 2.0], len(pairs))
    # two coplanar overlap triangles sharing an edge (pairs with three segments)
    t = pts[base:base + 4]
    for tri in ((0, 1, 2), (1, 3, 2)):
        pair = len(pairs)
        for a, b in ((0, 1), (1, 2), (2, 0)):
            add(t[tri[a]], t[tri[b]], pair)
    seg = np.array(segs, dtype=np.float64)
    sp = np.array(pairs, dtype=np.int32)
    return seg, sp, int(sp.max()) + 1


@pytest.mark.parametrize("seed", range(5))
@pytest.mark.parametrize("drop", [True, False])
def test_curves_match_reference(gi, seed, drop):
    rng = np.random.default_rng(seed)
    seg, sp, npairs = _soup(rng)
    perm = rng.permutation(len(seg))
    # pair indices are per pair: keep them consistent under the permutation
    v, cv = gi.curves(seg[perm], sp[perm], npairs, drop_coplanar_interior=drop)
    rv, rc = _reference(seg[perm], sp[perm], npairs, drop)
    assert _canon(v, cv) == _canon(rv, rc)
    n_closed = sum(1 for _, c in cv if c)
    assert n_closed == (3 if drop else 2)  # two loops, plus the coplanar region's boundary when interiors drop


@pytest.mark.parametrize("drop", [True, False])
def test_curves_of_jobs_equal_per_job(gi, drop):
    """gi_curves_build_jobs on a batch of soups (some jobs empty) gives, per
    job, exactly what gi_curves_build gives for the job alone."""
    rng = np.random.default_rng(11)
    segs, gpair, offsets, jobs = [], [], [0], []
    for j in range(40):
        if j % 7 == 3:  # a job without segments, and one with pairs but no segments
            jobs.append((np.zeros((0, 6)), np.zeros(0, np.int32), 2 if j % 2 else 0))
        else:
            seg, sp, npairs = _soup(rng)
            order = np.argsort(sp, kind="stable")  # a result's segments are ordered by pair
            jobs.append((seg[order], sp[order], npairs))
        seg, sp, npairs = jobs[-1]
        segs.append(seg)
        gpair.append(sp.astype(np.int64) + offsets[-1])
        offsets.append(offsets[-1] + npairs)
    out = gi.curves_of_jobs(np.concatenate(segs), np.concatenate(gpair), np.array(offsets), drop)
    assert len(out["job_curves"]) == len(jobs) + 1
    for j, (seg, sp, npairs) in enumerate(jobs):
        v, cv = gi.curves(seg, sp, npairs, drop_coplanar_interior=drop)
        c0, c1 = int(out["job_curves"][j]), int(out["job_curves"][j + 1])
        assert c1 - c0 == len(cv)
        for k, (ids, closed) in enumerate(cv):
            a, b = int(out["offsets"][c0 + k]), int(out["offsets"][c0 + k + 1])
            assert bool(out["closed"][c0 + k]) == closed
            assert np.array_equal(out["vertices"][out["idx"][a:b]], v[ids])


def test_curves_empty_and_points(gi):
    v, cv = gi.curves(np.zeros((0, 6)), np.zeros(0, np.int32), 0)
    assert v.shape == (0, 3) and cv == []
    seg = np.array([[1.0, 2.0, 3.0, 1.0, 2.0, 3.0]])
    v, cv = gi.curves(seg, np.array([0], np.int32), 1)
    assert v.shape == (1, 3) and len(cv) == 1 and list(cv[0][0]) == [0] and not cv[0][1]


@pytest.mark.gpu
def test_curves_of_sphere_intersections_close(ctx, gi):
    """Two closed surfaces meet along closed curves: every curve of config 1 and
    config 2 is closed and every endpoint is on a curve."""
    from gpuintersector import meshgen as mg
    from conftest import gi_pose

    for cfg in (mg.config1(seed=6), mg.config2(level=6)):
        A, B = ctx.upload(cfg["vA"], cfg["tA"]), ctx.upload(cfg["vB"], cfg["tB"])
        r = ctx.intersect(A, B, None, gi_pose(gi, cfg["poseB"]))
        v, cv = r.curves()
        assert len(cv) >= 1 and all(closed for _, closed in cv)
        assert sum(len(i) for i, _ in cv) == v.shape[0]
        A.release()
        B.release()
