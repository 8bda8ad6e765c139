"""Sign-by-sign parity of the device predicates.

Every decision of the intersection path is made from orient3d / orient2d signs
(the reference's device predicates: src/GPU_exact_predicates/
GPUPredicatesCommon.h:38-100 orient3d_interval, DoublePredicate.cu:75-93
orient3d_double_interval, ExactBigIntPredicate.cu:180-212 orient2d/orient3d_
exact_V2, and CGAL's exact predicates behind src/CPU/YellowFilter.h:80-137).
gi_predicate_signs runs, through the C ABI, the same device functions the
traversal's filter and the exact stage call, and returns each stage's answer.
Here every answer is compared with the exact rational sign (tests/fraction_ref.py)
and with the oracle's sign on the same inputs:

  * the integer sign and the exact stage's answer equal the exact sign, always;
  * a filter that decides (FP32 or FP64, either form) gives the exact sign;
  * both integer branches run: int128 (coordinates on a grid of <= 40 bits,
    60 for orient2d) and the multi-limb integers (wider exponent spans).

Inputs: the predicate calls that the oracle's decision procedure makes on the
600 frozen near-degenerate pairs, on fresh seeded near-degenerate families and
on sampled candidate pairs of the coplanar-grid stress configuration (the
pairs the device escalates), plus constructed exactly-degenerate point sets
with exponent spans beyond the int128 range and one-unit perturbations of them.
"""
import random

import numpy as np
import pytest

import sign_families as sf
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

O3, O2 = sf.O3, sf.O2
UNDECIDED, NA = 2, 3
INT128, MULTILIMB = 0, 1


def check_signs(ctx, kind, pts, drop, exact, what):
    """Device stages against the exact signs; returns the integer branches used."""
    pts = np.ascontiguousarray(pts[:, :12 if kind == O3 else 9], dtype=np.float64)
    out = ctx.predicate_signs(kind, pts, drop)
    exact = np.asarray(exact, dtype=np.int8)
    for col, name in ((5, "exact integer sign"), (6, "exact stage")):
        bad = np.nonzero(out[:, col] != exact)[0]
        assert bad.size == 0, "%s: %s differs on %d of %d queries, first %s: %d vs %d" % (
            what, name, bad.size, len(exact), pts[bad[0]].tolist(), out[bad[0], col], exact[bad[0]])
    names = ("FP32 filter (line form)", "FP32 filter (plane form)", "FP64 semi-static filter (line form)",
             "FP64 semi-static filter (plane form)", "FP64 filter of the exact stage")
    for col, name in enumerate(names):
        v = out[:, col]
        if kind == O2 and col < 4:
            assert np.all(v == NA), "%s: %s should be n/a for orient2d" % (what, name)
            continue
        dec = v != UNDECIDED
        assert np.all(np.isin(v[dec], (-1, 1))), "%s: %s gives a zero or an unknown code" % (what, name)
        bad = np.nonzero(dec & (v != exact))[0]
        assert bad.size == 0, "%s: %s decided wrongly on %d queries, first %s" % (
            what, name, bad.size, pts[bad[0]].tolist())
    assert np.all(np.isin(out[:, 7], (INT128, MULTILIMB))), "%s: integer capacity exceeded" % what
    exp_branch = sf.expected_branch(pts, kind, drop)
    bad = np.nonzero(out[:, 7] != exp_branch)[0]
    assert bad.size == 0, "%s: integer branch differs from the span rule on %d queries" % (what, bad.size)
    return out


def logged_calls(oc, fn):
    (pts, kind, drop, sign), _ = oc.record_signs(fn)
    return pts, kind, drop, sign


def replay(ctx, pts, kind, drop, sign, what, fraction_sample=None, rng=None):
    """Device signs of the oracle's logged calls: equal to the oracle's signs, and
    (on all calls or a sample) to the exact rational signs."""
    branches = []
    for k in (O3, O2):
        sel = np.nonzero(kind == k)[0]
        if sel.size == 0:
            continue
        p, d, s = pts[sel], drop[sel], sign[sel]
        if fraction_sample is not None and sel.size > fraction_sample:
            sub = rng.choice(sel.size, fraction_sample, replace=False)
            assert np.array_equal(sf.exact_signs(p[sub], k, d[sub]), s[sub]), "%s: oracle log vs fractions" % what
        else:
            assert np.array_equal(sf.exact_signs(p, k, d), s), "%s: oracle log vs fractions" % what
        out = check_signs(ctx, k, p, d, s, "%s (%s)" % (what, "orient3d" if k == O3 else "orient2d"))
        branches.append(out[:, 7])
    return np.concatenate(branches) if branches else np.zeros(0, np.int8)


def test_signs_of_frozen_near_degenerate_pairs(ctx, oc):
    tris = sf.frozen_pairs(GOLDEN)

    def run():
        for t1, t2 in tris:
            oc.tri_tri_construct(t1, t2)

    pts, kind, drop, sign = logged_calls(oc, run)
    assert len(sign) > 5000
    assert np.count_nonzero(sign == 0) > 500, "the family must hold exactly degenerate signs"
    br = replay(ctx, pts, kind, drop, sign, "frozen pairs")
    assert np.count_nonzero(br == INT128) > 0


@pytest.mark.parametrize("seed", [21, 22])
def test_signs_of_fresh_near_degenerate_pairs(ctx, oc, seed):
    tris = sf.fresh_pairs(seed)

    def run():
        for t1, t2 in tris:
            oc.tri_tri_construct(np.array(t1), np.array(t2))

    pts, kind, drop, sign = logged_calls(oc, run)
    br = replay(ctx, pts, kind, drop, sign, "fresh pairs seed %d" % seed)
    assert np.count_nonzero(br == INT128) > 0 and np.count_nonzero(br == MULTILIMB) > 0


def test_signs_of_coplanar_grid_escalations(ctx, gi, oc):
    """Candidate pairs of the coplanar-grid stress configuration (512 x 512 quads
    on a 2^20 grid, B coplanar and shifted half a cell, tiles at z = -1, 0, +1):
    every pair the device escalates is coplanar or touching, so these are the
    calls of the exact stage on the int128 branch."""
    from gpuintersector import meshgen as mg

    cfg = mg.config3()
    ref = oc.intersect_meshes(cfg["vA"], cfg["tA"], oc.pose_identity(), cfg["vB"], cfg["tB"], oc.pose_identity(),
                              want_segments=False)
    rng = np.random.default_rng(33)
    sel = ref["pairs"][rng.choice(len(ref["pairs"]), 2000, replace=False)]
    nb = np.stack([sel[:, 0], (sel[:, 1] + rng.integers(-3, 4, len(sel))) % cfg["tB"].shape[0]], 1)
    pairs = np.concatenate([sel, nb]).astype(np.int32)
    pts, kind, drop, sign = logged_calls(oc, lambda: oc.classify_pairs(
        cfg["vA"], cfg["tA"], oc.pose_identity(), cfg["vB"], cfg["tB"], oc.pose_identity(), pairs, nthreads=1))
    assert len(sign) > 50000 and np.count_nonzero(sign == 0) > 10000
    br = replay(ctx, pts, kind, drop, sign, "coplanar grid", fraction_sample=6000, rng=rng)
    assert np.all(br == INT128), "grid coordinates stay on the int128 branch"


def test_signs_beyond_int128_spans(ctx):
    rng = random.Random(44)
    p3 = sf.wide_span_o3(rng, 400)
    e3 = sf.exact_signs(p3, O3, None)
    assert np.count_nonzero(e3 == 0) >= 400 and np.count_nonzero(e3 != 0) > 400
    out3 = check_signs(ctx, O3, p3, None, e3, "wide-span orient3d")
    assert np.all(out3[:, 7] == MULTILIMB), "spans beyond 40 bits take the multi-limb branch"
    p2, d2 = sf.wide_span_o2(rng, 400)
    e2 = sf.exact_signs(p2, O2, d2)
    assert np.count_nonzero(e2 == 0) >= 400 and np.count_nonzero(e2 != 0) > 400
    out2 = check_signs(ctx, O2, p2, d2, e2, "wide-span orient2d")
    assert np.all(out2[:, 7] == MULTILIMB), "spans beyond 60 bits take the multi-limb branch"


def test_signs_entry_point_errors(ctx, gi):
    with pytest.raises(gi.GIError) as e:
        ctx.predicate_signs(O3, np.full((1, 12), 2.0 ** 101))
    assert e.value.status == gi._abi.GI_ERR_RANGE
    with pytest.raises(gi.GIError) as e:
        ctx.predicate_signs(O2, np.zeros((1, 9)), np.array([3], np.int32))
    assert e.value.status == gi._abi.GI_ERR_INVALID_ARG
    assert ctx.predicate_signs(O3, np.zeros((0, 12))).shape == (0, 8)
