"""Generates the committed golden fixtures under tests/golden/.

The reference ships no golden vectors or stored expected outputs (its only
verification is a live CGAL comparison, src/CPU/TestSuite.cpp:235-321), so the
fixtures are derived here:

  known_answers.json  hand-derived triangle pairs with their exact intersection
                      (kind and points, written as rationals); every entry is
                      re-checked against the Fraction clipper below.
  random_pairs.json   seeded random and near-degenerate pairs whose exact answer
                      comes from the Fraction clipper (tests/fraction_ref.py);
                      points are stored as float.hex of the correctly rounded value.
  config1.npz         UV spheres 128x80 (the small configuration): inputs, pose,
                      sorted pair set and canonical segments from the C oracle,
                      written only after every intersecting pair and a sample of
                      candidate pairs agreed with the Fraction clipper.
  grid64.npz          a 64x64-quad version of the coplanar integer-grid stress
                      case, the same way.

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import random
import sys
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "gpu-cubql-intersector-standalone_b200"))

import fraction_ref as fr  # noqa: E402
import oracle as oc  # noqa: E402
from gpuintersector import meshgen as mg  # noqa: E402

KIND = {"none": 0, "point": 1, "segment": 2, "triangle": 3, "polygon": 4}

T1 = [[0, 0, 0], [2, 0, 0], [0, 2, 0]]  # x, y >= 0, x + y <= 2, z = 0
KNOWN = [
    # coplanar
    dict(name="coplanar identical", t1=T1, t2=T1, kind="triangle", pts=[[0, 0, 0], [2, 0, 0], [0, 2, 0]]),
    dict(name="coplanar disjoint", t1=T1, t2=[[3, 0, 0], [5, 0, 0], [3, 2, 0]], kind="none", pts=[]),
    # T2 = conv{(2,0),(4,0),(4,2)} meets x+y<=2 only where x = 2, y = 0
    dict(name="coplanar vertex touch", t1=T1, t2=[[2, 0, 0], [4, 0, 0], [4, 2, 0]], kind="point", pts=[[2, 0, 0]]),
    # mirror image below the shared edge
    dict(name="coplanar shared edge", t1=T1, t2=[[0, 0, 0], [2, 0, 0], [0, -2, 0]], kind="segment",
         pts=[[0, 0, 0], [2, 0, 0]]),
    # T2 = conv{(0,1),(2,1),(1,3)}: y >= 1 inside T1 gives (0,1), (1,1) and
    # x + y = 2 meeting y = 2x + 1 at (1/3, 5/3)
    dict(name="coplanar triangle overlap", t1=T1, t2=[[0, 1, 0], [2, 1, 0], [1, 3, 0]], kind="triangle",
         pts=[[0, 1, 0], [1, 1, 0], ["1/3", "5/3", 0]]),
    # big T2 with right edge x = 1.5 cuts one corner off T1: (0,0), (1.5,0), (1.5,0.5), (0,2)
    dict(name="coplanar quad overlap", t1=T1, t2=[[1.5, -10, 0], [1.5, 10, 0], [-20, 0, 0]], kind="polygon",
         pts=[[0, 0, 0], [1.5, 0, 0], [1.5, 0.5, 0], [0, 2, 0]]),
    # non-coplanar: T2 in the plane y = 1/2 meets z = 0 on x in [1/2, 2]; T1 covers x in [0, 3/2]
    dict(name="crossing segment", t1=T1, t2=[[0.5, 0.5, -1], [0.5, 0.5, 1], [2, 0.5, 0]], kind="segment",
         pts=[[0.5, 0.5, 0], [1.5, 0.5, 0]]),
    dict(name="vertex touching interior", t1=T1, t2=[[0.5, 0.5, 0], [0, 0, 1], [1, 0, 1]], kind="point",
         pts=[[0.5, 0.5, 0]]),
    dict(name="parallel planes", t1=T1, t2=[[0, 0, 1], [2, 0, 1], [0, 2, 1]], kind="none", pts=[]),
    # T2 in the plane x = 1 through T1's hypotenuse point (1,1,0) only along z = 0: the
    # segment of T2 on z = 0 is x = 1, y in [1, 3]; T1 reaches y <= 1 there
    dict(name="edge touching edge", t1=T1, t2=[[1, 1, -1], [1, 1, 1], [1, 3, 0]], kind="point", pts=[[1, 1, 0]]),
    # degenerate (collinear) T2: the segment (0,0)-(2,2) clipped by x + y <= 2
    dict(name="degenerate segment in plane", t1=T1, t2=[[0, 0, 0], [1, 1, 0], [2, 2, 0]], kind="segment",
         pts=[[0, 0, 0], [1, 1, 0]]),
    dict(name="degenerate point inside", t1=T1, t2=[[0.5, 0.5, 0]] * 3, kind="point", pts=[[0.5, 0.5, 0]]),
    dict(name="degenerate segment piercing", t1=T1, t2=[[0.5, 0.5, -1], [0.5, 0.5, 1], [0.5, 0.5, 0]],
         kind="point", pts=[[0.5, 0.5, 0]]),
    dict(name="degenerate segment missing", t1=T1, t2=[[3, 3, -1], [3, 3, 1], [3, 3, 0]], kind="none", pts=[]),
]


def _q(x):
    return Fraction(x) if not isinstance(x, str) else Fraction(x)


def canon_pts(pts):
    return sorted(tuple(float(v) for v in p) for p in pts)


def check_known():
    for c in KNOWN:
        k, p = fr.tri_tri(c["t1"], c["t2"])
        exp = sorted(tuple(_q(v) for v in q) for q in c["pts"])
        assert k == KIND[c["kind"]], (c["name"], k)
        assert sorted(p) == exp, (c["name"], p, exp)
        ko, po = oc.tri_tri_construct(np.array(c["t1"], float), np.array(c["t2"], float))
        assert ko == k and canon_pts(po) == canon_pts(exp), (c["name"], ko, po)
    return [dict(name=c["name"], t1=c["t1"], t2=c["t2"], kind=KIND[c["kind"]],
                 pts=[[str(_q(v)) for v in q] for q in c["pts"]]) for c in KNOWN]


def random_cases(n=600, seed=20261203):
    rng = random.Random(seed)
    out = []
    for it in range(n):
        mode = it % 6
        if mode == 0:
            t = [[[rng.randint(0, 3) for _ in range(3)] for _ in range(3)] for _ in range(2)]
        elif mode == 1:
            t = [[[rng.randint(-2, 2), rng.randint(-2, 2), 0] for _ in range(3)] for _ in range(2)]
        elif mode == 2:
            t = [[[rng.uniform(-1, 1) for _ in range(3)] for _ in range(3)] for _ in range(2)]
        elif mode == 3:
            t = []
            for _ in range(2):
                tri = []
                for _ in range(3):
                    x, y = rng.randint(-3, 3), rng.randint(-3, 3)
                    tri.append([x, y, 2 - x - y])
                t.append(tri)
        elif mode == 4:
            a = [[rng.randint(0, 2) for _ in range(3)] for _ in range(3)]
            t = [a, [a[rng.randint(0, 2)], [rng.randint(0, 2) for _ in range(3)],
                     [rng.randint(0, 2) for _ in range(3)]]]
        else:
            eps = [0.0, 0.0, 2.0 ** -40, -2.0 ** -40, 2.0 ** -52]
            t = [[[rng.randint(0, 2) + rng.choice(eps) for _ in range(3)] for _ in range(3)] for _ in range(2)]
        t1 = [[float(v) for v in p] for p in t[0]]
        t2 = [[float(v) for v in p] for p in t[1]]
        k, p = fr.tri_tri_float(t1, t2)
        out.append(dict(t1=[[x.hex() for x in q] for q in t1], t2=[[x.hex() for x in q] for q in t2], kind=k,
                        pts=sorted([[x.hex() for x in q] for q in p])))
    return out


def pose_of(p):
    if p is None:
        return oc.pose_identity()
    R, C, T = p
    return oc.pose_raw(R, C, T)


def mesh_golden(cfg, sample=600, seed=5):
    pa, pb = pose_of(cfg["poseA"]), pose_of(cfg["poseB"])
    r = oc.intersect_meshes(cfg["vA"], cfg["tA"], pa, cfg["vB"], cfg["tB"], pb, want_segments=True)
    wA = oc.transform(pa, cfg["vA"])
    wB = oc.transform(pb, cfg["vB"])
    tA, tB = cfg["tA"], cfg["tB"]
    rng = np.random.default_rng(seed)
    pairs = r["pairs"]
    idx = rng.choice(len(pairs), size=min(sample, len(pairs)), replace=False)
    for i in idx:
        a, b = pairs[i]
        k, _ = fr.tri_tri(wA[tA[a]].tolist(), wB[tB[b]].tolist())
        assert k != 0, ("oracle pair not confirmed by the Fraction clipper", a, b)
        ko, po = oc.tri_tri_construct(wA[tA[a]], wB[tB[b]])
        kf, pf = fr.tri_tri_float(wA[tA[a]].tolist(), wB[tB[b]].tolist())
        assert ko == kf and canon_pts(po) == canon_pts(pf), ("construction mismatch", a, b)
    # random non-reported pairs with overlapping boxes must be disjoint
    pset = set(map(tuple, pairs.tolist()))
    loA, hiA = wA[tA].min(axis=1), wA[tA].max(axis=1)
    loB, hiB = wB[tB].min(axis=1), wB[tB].max(axis=1)
    checked = 0
    for a in rng.choice(len(tA), size=min(4000, len(tA)), replace=False):
        ov = np.nonzero(np.all(loB <= hiA[a], axis=1) & np.all(hiB >= loA[a], axis=1))[0]
        for b in ov[:4]:
            if (int(a), int(b)) in pset:
                continue
            k, _ = fr.tri_tri(wA[tA[a]].tolist(), wB[tB[b]].tolist())
            assert k == 0, ("pair missed by the oracle", a, b)
            checked += 1
    return r, checked


def main():
    os.makedirs(HERE, exist_ok=True)
    known = check_known()
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(known, f, indent=1)
    rc = random_cases()
    with open(os.path.join(HERE, "random_pairs.json"), "w") as f:
        json.dump(rc, f)
    c1 = mg.config1()
    r1, n1 = mesh_golden(c1)
    R, C, T = c1["poseB"]
    np.savez_compressed(os.path.join(HERE, "config1.npz"), vA=c1["vA"], tA=c1["tA"], vB=c1["vB"], tB=c1["tB"],
                        poseB_R=R, poseB_C=C, poseB_T=T, pairs=r1["pairs"], segs=r1["segs"],
                        seg_pair=r1["seg_pair"])
    g = mg.config3(n=64)
    r3, n3 = mesh_golden(g, sample=800)
    np.savez_compressed(os.path.join(HERE, "grid64.npz"), vA=g["vA"], tA=g["tA"], vB=g["vB"], tB=g["tB"],
                        pairs=r3["pairs"], segs=r3["segs"], seg_pair=r3["seg_pair"])
    print("known %d, random %d, config1 pairs %d (non-pairs checked %d), grid64 pairs %d (non-pairs checked %d)"
          % (len(known), len(rc), len(r1["pairs"]), n1, len(r3["pairs"]), n3))


if __name__ == "__main__":
    main()
