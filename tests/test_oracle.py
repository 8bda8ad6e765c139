"""CPU tests of the checker: the C oracle is pinned against hand-derived known
answers, the independent Fraction clipper, and the committed golden fixtures.
Mirrors the reference's verification semantics: exact set equality of
(faceA, faceB) pairs with FP/FN counts (src/CPU/TestSuite.cpp:24-32, 285-296)."""
import json
import os
import random
from fractions import Fraction

import numpy as np
import pytest

from conftest import GOLDEN, canonical, oracle_pose

import fraction_ref as fr


def _hexpts(pts):
    return sorted(tuple(float.fromhex(x) for x in p) for p in pts)


def test_known_answers(oc):
    cases = json.load(open(os.path.join(GOLDEN, "known_answers.json")))
    assert len(cases) >= 12
    for c in cases:
        exp = sorted(tuple(float(Fraction(v)) for v in p) for p in c["pts"])
        k, p = oc.tri_tri_construct(np.array(c["t1"], float), np.array(c["t2"], float))
        assert k == c["kind"], c["name"]
        assert sorted(tuple(q) for q in p) == exp, c["name"]
        assert oc.tri_tri_intersect(np.array(c["t1"], float), np.array(c["t2"], float)) == (c["kind"] != 0)
        # symmetric in the argument order
        k2, p2 = oc.tri_tri_construct(np.array(c["t2"], float), np.array(c["t1"], float))
        assert k2 == c["kind"] and sorted(tuple(q) for q in p2) == exp, c["name"]


def test_random_pairs_golden(oc):
    cases = json.load(open(os.path.join(GOLDEN, "random_pairs.json")))
    kinds = [0] * 5
    for c in cases:
        t1 = np.array([[float.fromhex(x) for x in p] for p in c["t1"]])
        t2 = np.array([[float.fromhex(x) for x in p] for p in c["t2"]])
        k, p = oc.tri_tri_construct(t1, t2)
        assert k == c["kind"]
        assert sorted(tuple(q) for q in p) == _hexpts(c["pts"])
        kinds[k] += 1
    assert min(kinds) > 0, "every result kind is covered"


@pytest.mark.parametrize("seed", [11, 12])
def test_oracle_vs_fraction_fresh(oc, seed):
    """Fresh random near-degenerate cases, beyond the committed fixture."""
    rng = random.Random(seed)
    for it in range(250):
        mode = it % 3
        if mode == 0:
            t = [[[rng.randint(0, 2) for _ in range(3)] for _ in range(3)] for _ in range(2)]
        elif mode == 1:
            s = 10 ** rng.uniform(-5, 5)
            o = rng.uniform(-100, 100)
            t = [[[o + s * rng.uniform(-1, 1) for _ in range(3)] for _ in range(3)] for _ in range(2)]
        else:
            base = [[rng.randint(-2, 2) for _ in range(3)] for _ in range(3)]
            t = [base, [[x + rng.choice([0.0, 2.0 ** -45]) for x in p] for p in base[::-1]]]
        t1 = [[float(v) for v in p] for p in t[0]]
        t2 = [[float(v) for v in p] for p in t[1]]
        kf, pf = fr.tri_tri_float(t1, t2)
        ko, po = oc.tri_tri_construct(np.array(t1), np.array(t2))
        assert ko == kf
        assert sorted(tuple(q) for q in po) == sorted(pf)


def test_orient_signs_exact(oc):
    # a point 2^-52 above a plane through integer points
    a, b, c = [0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]
    assert oc.orient3d(a, b, c, [0.25, 0.25, 2.0 ** -52]) == -oc.orient3d(a, b, c, [0.25, 0.25, -2.0 ** -52])
    assert oc.orient3d(a, b, c, [0.25, 0.25, 0.0]) == 0
    # far from the origin, cancellation-heavy but exactly coplanar
    o = 2.0 ** 30
    assert oc.orient3d([o, o, o], [o + 1, o, o], [o, o + 1, o], [o + 3, o + 7, o]) == 0
    # orient2d: exactly collinear vs. one ulp off the line
    assert oc.orient2d([1.0, 2.0, 0.0], [2.0, 4.0, 0.0], [3.0, 6.0, 0.0], 2) == 0
    assert oc.orient2d([1.0, 2.0, 0.0], [2.0, 4.0, 0.0], [3.0, np.nextafter(6.0, 7.0), 0.0], 2) != 0


def test_pose_semantics(oc, gi):
    """FP64 pose order of RotationTools.h:135-143, bit-identical host paths."""
    rng = np.random.default_rng(1)
    v = rng.standard_normal((500, 3))
    rot, cen, tr = [10.0, -20.0, 33.0], [0.1, -0.2, 0.3], [0.5, 0.25, -1.0]
    po = oc.pose_from_euler_deg(rot, cen, tr)
    pg = gi.pose_from_euler_deg(rot, cen, tr)
    assert list(po.R) == list(pg.R)
    w_or = oc.transform(po, v)
    w_gi = gi.pose_apply(pg, v)
    assert np.array_equal(w_or, w_gi)
    R = np.array(po.R).reshape(3, 3)
    x = v - np.array(cen)
    rx = (R[0, 0] * x[:, 0] + R[0, 1] * x[:, 1]) + R[0, 2] * x[:, 2]
    assert np.array_equal(w_or[:, 0], (rx + cen[0]) + tr[0])
    # identity pose leaves vertices unchanged
    assert np.array_equal(oc.transform(oc.pose_identity(), v), v)


def test_config1_golden(oc):
    g = np.load(os.path.join(GOLDEN, "config1.npz"))
    pb = oc.pose_raw(g["poseB_R"], g["poseB_C"], g["poseB_T"])
    r = oc.intersect_meshes(g["vA"], g["tA"], oc.pose_identity(), g["vB"], g["tB"], pb, want_segments=True)
    assert np.array_equal(r["pairs"], g["pairs"])
    gp, gs = canonical(r["segs"], r["seg_pair"])
    ep, es = canonical(g["segs"], g["seg_pair"])
    assert np.array_equal(gp, ep) and np.array_equal(gs, es)


def test_grid64_golden(oc):
    g = np.load(os.path.join(GOLDEN, "grid64.npz"))
    ip = oc.pose_identity()
    r = oc.intersect_meshes(g["vA"], g["tA"], ip, g["vB"], g["tB"], ip, want_segments=True, nthreads=2)
    assert np.array_equal(r["pairs"], g["pairs"])
    gp, gs = canonical(r["segs"], r["seg_pair"])
    ep, es = canonical(g["segs"], g["seg_pair"])
    assert np.array_equal(gp, ep) and np.array_equal(gs, es)


def test_bvh_vs_bruteforce(oc, gi):
    from gpuintersector import meshgen as mg

    v, t = mg.uv_sphere(12, 8)
    R = mg.random_rotation(np.random.default_rng(3))
    pb = oc.pose_raw(R, (0, 0, 0), (0.4, 0.2, 0.0))
    r = oc.intersect_meshes(v, t, oc.pose_identity(), v, t, pb, want_segments=False, nthreads=3)
    bf = oc.intersect_meshes_bruteforce(v, t, oc.pose_identity(), v, t, pb)
    bf = bf[np.lexsort((bf[:, 1], bf[:, 0]))]
    assert len(r["pairs"]) > 0 and np.array_equal(r["pairs"], bf)


def test_empty_and_bad_meshes(oc):
    ip = oc.pose_identity()
    v = np.zeros((3, 3))
    t = np.array([[0, 1, 2]], dtype=np.uint32)
    r = oc.intersect_meshes(v, np.zeros((0, 3), np.uint32), ip, v, t, ip)
    assert len(r["pairs"]) == 0
    with pytest.raises(RuntimeError):
        oc.intersect_meshes(v, np.array([[0, 1, 5]], np.uint32), ip, v, t, ip)


def test_oracle_classify_pairs_list(oc):
    """oc_classify_pairs (a pair list on host threads) agrees with the per-pair
    exact test, and rejects an index out of range."""
    from gpuintersector import meshgen as mg

    cfg = mg.config1(seed=5)
    R, C, T = cfg["poseB"]
    pB = oc.pose_raw(R, C, T)
    ref = oc.intersect_meshes(cfg["vA"], cfg["tA"], oc.pose_identity(), cfg["vB"], cfg["tB"], pB, want_segments=False)
    hits = ref["pairs"]
    nt = cfg["tB"].shape[0]
    d = np.arange(-6, 6)
    pairs = np.stack([np.repeat(hits[:, 0], d.size), (np.repeat(hits[:, 1], d.size) + np.tile(d, len(hits))) % nt], 1)
    out = oc.classify_pairs(cfg["vA"], cfg["tA"], oc.pose_identity(), cfg["vB"], cfg["tB"], pB, pairs, nthreads=3)
    wA = oc.transform(oc.pose_identity(), cfg["vA"])
    wB = oc.transform(pB, cfg["vB"])
    sample = range(0, len(pairs), 7)
    exp = [oc.tri_tri_intersect(wA[cfg["tA"][pairs[i, 0]]], wB[cfg["tB"][pairs[i, 1]]]) for i in sample]
    assert np.array_equal(out[list(sample)], np.array(exp, dtype=np.uint8))
    # every known intersecting pair is classified as such; the counts agree with the mesh run
    assert out[d.size // 2::d.size].all()
    hit_set = set(map(tuple, hits.tolist()))
    assert int(out.sum()) == sum(1 for p in map(tuple, pairs.tolist()) if p in hit_set)
    with pytest.raises(ValueError):
        oc.classify_pairs(cfg["vA"], cfg["tA"], oc.pose_identity(), cfg["vB"], cfg["tB"], pB, np.array([[0, nt]]))


def test_oracle_signs_vs_fractions_per_call(oc):
    """Every orient3d / orient2d call the oracle's decision procedure makes on the
    frozen and fresh near-degenerate pairs (its sign log), and its signs on
    exactly degenerate point sets with exponent spans beyond 2^40 / 2^60 and
    their one-unit perturbations, equal the exact rational signs.  These are the
    signs the device sign test (test_gpu_signs.py) is held to."""
    import sign_families as sf

    for tris in (sf.frozen_pairs(GOLDEN), sf.fresh_pairs(21)):
        (pts, kind, drop, sign), _ = oc.record_signs(lambda: [oc.tri_tri_construct(a, b) for a, b in tris])
        assert len(sign) > 2000 and np.count_nonzero(sign == 0) > 100
        for k in (sf.O3, sf.O2):
            sel = kind == k
            assert np.array_equal(sf.exact_signs(pts[sel], k, drop[sel]), sign[sel])
    rng = random.Random(44)
    p3 = sf.wide_span_o3(rng, 100)
    assert np.all(sf.expected_branch(p3, sf.O3) == 1)
    got = np.array([oc.orient3d(r[0:3], r[3:6], r[6:9], r[9:12]) for r in p3])
    assert np.array_equal(got, sf.exact_signs(p3, sf.O3, None))
    p2, d2 = sf.wide_span_o2(rng, 100)
    assert np.all(sf.expected_branch(p2, sf.O2, d2) == 1)
    got = np.array([oc.orient2d(r[0:3], r[3:6], r[6:9], int(d)) for r, d in zip(p2, d2)])
    assert np.array_equal(got, sf.exact_signs(p2, sf.O2, d2))
