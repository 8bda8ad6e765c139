"""Input families for sign-by-sign tests of the orientation predicates.

Test infrastructure: seeded point sets on and around exact degeneracies, their
exact signs from Python fractions (tests/fraction_ref.py), and the triangle
pairs whose predicate calls the oracle logs.  Used by the CPU pin of the oracle
(tests/test_oracle.py) and by the device sign test (tests/test_gpu_signs.py).
"""
import json
import math
import os
import random

import numpy as np

import fraction_ref as fr

O3, O2 = 0, 1


def exact_signs(pts, kind, drop):
    """Exact orient3d (kind 0, 12 doubles a b c d) or orient2d (kind 1, 9 doubles
    a b c and a drop axis) signs of each row."""
    if kind == O3:
        return np.array([fr.orient3d(p[0:3], p[3:6], p[6:9], p[9:12]) for p in pts.tolist()], dtype=np.int8)
    return np.array([fr.orient2d(p[0:3], p[3:6], p[6:9], int(d)) for p, d in zip(pts.tolist(), drop)], dtype=np.int8)


def frozen_pairs(golden_dir):
    """The 600 frozen near-degenerate triangle pairs of random_pairs.json."""
    cases = json.load(open(os.path.join(golden_dir, "random_pairs.json")))
    tr = lambda t: np.array([[float.fromhex(x) for x in p] for p in t])
    return [(tr(c["t1"]), tr(c["t2"])) for c in cases]


def fresh_pairs(seed, n=300):
    """Seeded near-degenerate triangle pairs: small integer grids, clustered
    coordinates far from the origin, copies shifted by 2^-45, and coordinates
    whose magnitudes differ by up to 2^120 between axes (exponent spans beyond
    the int128 range of the exact stage)."""
    rng = random.Random(seed)
    tris = []
    for it in range(n):
        mode = it % 4
        if mode == 0:
            t = [[[rng.randint(0, 2) for _ in range(3)] for _ in range(3)] for _ in range(2)]
        elif mode == 1:
            s = 10 ** rng.uniform(-5, 5)
            o = rng.uniform(-100, 100)
            t = [[[o + s * rng.uniform(-1, 1) for _ in range(3)] for _ in range(3)] for _ in range(2)]
        elif mode == 2:
            base = [[rng.randint(-2, 2) for _ in range(3)] for _ in range(3)]
            t = [base, [[x + rng.choice([0.0, 2.0 ** -45]) for x in p] for p in base[::-1]]]
        else:
            e = [rng.randint(-60, 60) for _ in range(3)]
            base = [[rng.randint(-8, 8) * 2.0 ** e[k] for k in range(3)] for _ in range(3)]
            t = [base, [[x + rng.choice([0.0, 2.0 ** (e[k] - 1)]) for k, x in enumerate(p)]
                        for p in base[1:] + base[:1]]]
        tris.append((np.array(t[0], dtype=np.float64), np.array(t[1], dtype=np.float64)))
    return tris


def wide_span_o3(rng, n):
    """Exactly coplanar (a, b, c, d) with per-axis scales 2^ex, 2^ey, 2^ez far
    apart (span > 40 bits), and one-unit perturbations of d along each axis."""
    rows = []
    for _ in range(n):
        ex = rng.sample(range(-80, 81), 3)
        while max(ex) - min(ex) <= 44:
            ex = rng.sample(range(-80, 81), 3)
        sc = [2.0 ** e for e in ex]
        a, b, c = [[rng.randint(-2000, 2000) for _ in range(3)] for _ in range(3)]
        i, j = rng.randint(-9, 9), rng.randint(-9, 9)
        d = [a[k] + i * (b[k] - a[k]) + j * (c[k] - a[k]) for k in range(3)]
        for pert in ((0, 0, 0), (1, 0, 0), (0, -1, 0), (0, 0, 1)):
            dd = [d[k] + pert[k] for k in range(3)]
            rows.append([x * sc[k] for p in (a, b, c, dd) for k, x in enumerate(p)])
    pts = np.array(rows, dtype=np.float64)
    assert np.all((pts == 0) | ((np.abs(pts) >= 2.0 ** -100) & (np.abs(pts) <= 2.0 ** 100)))
    return pts


def wide_span_o2(rng, n):
    """Exactly collinear (a, b, c) in the (u, v) plane of a random drop axis with
    scales 2^eu, 2^ev more than 60 bits apart, and one-unit perturbations of c."""
    rows, drops = [], []
    for _ in range(n):
        drop = rng.randint(0, 2)
        u, v = (drop + 1) % 3, (drop + 2) % 3
        lo = rng.randint(-80, 16)
        hi = lo + rng.randint(64, min(90, 80 - lo))
        eu, ev = (lo, hi) if rng.random() < 0.5 else (hi, lo)
        sc = [1.0, 1.0, 1.0]
        sc[u], sc[v] = 2.0 ** eu, 2.0 ** ev
        a, b = [[rng.randint(-4000, 4000) for _ in range(3)] for _ in range(2)]
        k = rng.randint(-7, 7)
        c = [a[q] + k * (b[q] - a[q]) for q in range(3)]
        for pert in ((0, 0), (1, 0), (0, -1)):
            cc = list(c)
            cc[u] += pert[0]
            cc[v] += pert[1]
            rows.append([x * sc[q] for p in (a, b, cc) for q, x in enumerate(p)])
            drops.append(drop)
    pts = np.array(rows, dtype=np.float64)
    assert np.all((pts == 0) | ((np.abs(pts) >= 2.0 ** -100) & (np.abs(pts) <= 2.0 ** 100)))
    return pts, np.array(drops, dtype=np.int32)


def grid_span(row):
    """Bits between the lowest and the highest set bit over the nonzero
    coordinates of one query: the exact stage takes its int128 branch when this
    is at most 40 (orient3d) or 60 (orient2d), its multi-limb branch otherwise."""
    lo, hi = None, None
    for x in row:
        if x == 0.0:
            continue
        m, e = math.frexp(abs(x))
        mant = int(m * 2.0 ** 53)
        tz = (mant & -mant).bit_length() - 1
        elow, ehigh = e - 53 + tz, e
        lo = elow if lo is None else min(lo, elow)
        hi = ehigh if hi is None else max(hi, ehigh)
    return 0 if lo is None else hi - lo


def expected_branch(pts, kind, drop=None):
    """Integer branch (0 int128, 1 multi-limb) the exact stage must take per row."""
    if kind == O3:
        return np.array([0 if grid_span(r) <= 40 else 1 for r in pts[:, :12].tolist()], dtype=np.int8)
    out = []
    for r, d in zip(pts[:, :9].tolist(), drop):
        u, v = (int(d) + 1) % 3, (int(d) + 2) % 3
        out.append(0 if grid_span([r[3 * i + u] for i in range(3)] + [r[3 * i + v] for i in range(3)]) <= 60 else 1)
    return np.array(out, dtype=np.int8)
