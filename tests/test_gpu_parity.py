"""GPU parity tests: libgi.so through its C ABI versus the exact CPU oracle and
the committed golden fixtures.  Bit-exact pair sets (the reference's criterion,
src/CPU/TestSuite.cpp:285-306: set equality, zero false positives / negatives)
and bit-exact segment endpoints (both sides round the exact point to nearest)."""
import json
import os
from fractions import Fraction

import numpy as np
import pytest

from conftest import GOLDEN, canonical, gi_pose, oracle_pose

pytestmark = pytest.mark.gpu


def assert_same(res, ref, segments=True):
    got, exp = res.pairs, ref["pairs"]
    if not np.array_equal(got, exp):
        gs, es = set(map(tuple, got.tolist())), set(map(tuple, exp.tolist()))
        raise AssertionError("pair sets differ: %d false positives, %d false negatives (of %d)"
                             % (len(gs - es), len(es - gs), len(es)))
    if segments:
        gp, gs = canonical(res.segments, res.seg_pair)
        ep, es = canonical(ref["segs"], ref["seg_pair"])
        assert np.array_equal(gp, ep), "segment grouping differs"
        if not np.array_equal(gs, es):
            bad = np.nonzero(np.any(gs != es, axis=1))[0]
            raise AssertionError("%d of %d segment endpoints differ, first: %s vs %s"
                                 % (len(bad), len(es), gs[bad[0]], es[bad[0]]))


def run_cfg(ctx, gi, oc, cfg, precision=0, want_segments=True, nthreads=0):
    A = ctx.upload(cfg["vA"], cfg["tA"])
    B = ctx.upload(cfg["vB"], cfg["tB"])
    r = ctx.intersect(A, B, gi_pose(gi, cfg["poseA"]), gi_pose(gi, cfg["poseB"]), want_segments=want_segments,
                      precision=precision)
    ref = oc.intersect_meshes(cfg["vA"], cfg["tA"], oracle_pose(oc, cfg["poseA"]), cfg["vB"], cfg["tB"],
                              oracle_pose(oc, cfg["poseB"]), want_segments=want_segments, nthreads=nthreads)
    A.release()
    B.release()
    return r, ref


def test_smoke():
    import __graft_entry__

    __graft_entry__.smoke()


def _single_tri_jobs(ctx, cases):
    meshes, jobs = [], []
    for t1, t2 in cases:
        A = ctx.upload(np.array(t1, float), np.array([[0, 1, 2]], np.uint32))
        B = ctx.upload(np.array(t2, float), np.array([[0, 1, 2]], np.uint32))
        meshes += [A, B]
        jobs.append((A, None, B, None))
    return meshes, jobs


NSEG = {0: 0, 1: 1, 2: 1, 3: 3, 4: 0}


def test_known_answers_gpu(ctx, gi):
    cases = json.load(open(os.path.join(GOLDEN, "known_answers.json")))
    meshes, jobs = _single_tri_jobs(ctx, [(c["t1"], c["t2"]) for c in cases])
    res = ctx.intersect_batch(jobs, want_segments=True)
    for c, r in zip(cases, res):
        assert (r.pairs.shape[0] == 1) == (c["kind"] != 0), c["name"]
        assert r.segments.shape[0] == NSEG[c["kind"]], c["name"]
        pts = sorted(tuple(float(Fraction(v)) for v in p) for p in c["pts"])
        if c["kind"] in (1, 2, 3):
            got = sorted(set(tuple(s[:3]) for s in r.segments) | set(tuple(s[3:]) for s in r.segments))
            assert got == pts, c["name"]
    for m in meshes:
        m.release()


def test_random_pairs_gpu(ctx, gi):
    cases = json.load(open(os.path.join(GOLDEN, "random_pairs.json")))
    tr = lambda t: [[float.fromhex(x) for x in p] for p in t]
    meshes, jobs = _single_tri_jobs(ctx, [(tr(c["t1"]), tr(c["t2"])) for c in cases])
    res = ctx.intersect_batch(jobs, want_segments=True)
    for c, r in zip(cases, res):
        assert (r.pairs.shape[0] == 1) == (c["kind"] != 0)
        assert r.segments.shape[0] == NSEG[c["kind"]]
        if c["kind"] in (1, 2, 3):
            exp = sorted(tuple(float.fromhex(x) for x in p) for p in c["pts"])
            got = sorted(set(tuple(s[:3]) for s in r.segments) | set(tuple(s[3:]) for s in r.segments))
            assert got == exp
    for m in meshes:
        m.release()


def test_config1_golden_gpu(ctx, gi):
    g = np.load(os.path.join(GOLDEN, "config1.npz"))
    A, B = ctx.upload(g["vA"], g["tA"]), ctx.upload(g["vB"], g["tB"])
    for prec in (0, 1):
        r = ctx.intersect(A, B, None, gi.pose_raw(g["poseB_R"], g["poseB_C"], g["poseB_T"]), precision=prec)
        assert_same(r, dict(pairs=g["pairs"], segs=g["segs"], seg_pair=g["seg_pair"]))
    A.release()
    B.release()


def test_grid64_golden_gpu(ctx, gi):
    g = np.load(os.path.join(GOLDEN, "grid64.npz"))
    A, B = ctx.upload(g["vA"], g["tA"]), ctx.upload(g["vB"], g["tB"])
    for prec in (0, 1):
        r = ctx.intersect(A, B, None, None, precision=prec)
        assert_same(r, dict(pairs=g["pairs"], segs=g["segs"], seg_pair=g["seg_pair"]))
    A.release()
    B.release()


def test_config2_full_vs_oracle(ctx, gi, oc):
    from gpuintersector import meshgen as mg

    cfg = mg.config2()
    r, ref = run_cfg(ctx, gi, oc, cfg)
    assert_same(r, ref)
    st = r.stats
    assert st["pairs"] == len(ref["pairs"]) and st["candidates"] >= ref["stats"].candidates
    assert st["filter_decided"] >= 0.99 * st["candidates"]


def test_config3_full_vs_oracle(ctx, gi, oc):
    from gpuintersector import meshgen as mg

    cfg = mg.config3()
    r, ref = run_cfg(ctx, gi, oc, cfg)
    assert len(ref["pairs"]) > 1_000_000
    assert_same(r, ref)


def test_ordering_paths_and_redo(gi, oc):
    """Both ordering paths on a fresh context.  The path follows the previous
    call's result count: the first call predicts a small result and takes the
    one-launch path; a large result then overruns it, the kernel refuses and the
    call reruns on the radix path; the next (small) call takes the radix path,
    the one after it the one-launch path again.  All equal the oracle, sorted
    and unsorted."""
    from gpuintersector import meshgen as mg

    small = mg.config1(seed=21)
    large = mg.config3(n=256, seed=5)

    def unsorted_same(c, A, B, ref):
        ru = c.intersect(A, B, None, gi_pose(gi, small["poseB"]), sort_output=False)
        assert set(map(tuple, ru.pairs.tolist())) == set(map(tuple, ref["pairs"].tolist()))
        # segments: renumber the unsorted pair indices to the oracle's order, then compare canonically
        index = {ab: k for k, ab in enumerate(map(tuple, ref["pairs"].tolist()))}
        remap = np.array([index[ab] for ab in map(tuple, ru.pairs.tolist())], dtype=np.int64)
        gp, gs = canonical(ru.segments, remap[np.asarray(ru.seg_pair, dtype=np.int64)])
        ep, es = canonical(ref["segs"], ref["seg_pair"])
        assert np.array_equal(gp, ep) and np.array_equal(gs, es)

    with gi.Context(0) as c:
        r1, ref1 = run_cfg(c, gi, oc, small)          # one-launch path
        assert_same(r1, ref1)
        r2, ref2 = run_cfg(c, gi, oc, large)          # one-launch refused -> radix path
        assert len(ref2["pairs"]) > 65536
        assert_same(r2, ref2)
        A, B = c.upload(small["vA"], small["tA"]), c.upload(small["vB"], small["tB"])
        unsorted_same(c, A, B, ref1)                   # radix path, unsorted
        unsorted_same(c, A, B, ref1)                   # one-launch path, unsorted
        r3 = c.intersect(A, B, None, gi_pose(gi, small["poseB"]))
        assert_same(r3, ref1)
        A.release()
        B.release()


def _crowded_pair(n_grid, corner):
    """A: 2,048 triangles, the first a large triangle in the plane z = 0, the
    others tiny and far away; B: an n_grid x n_grid unit grid at z = 0.  Every
    result has a = 0, so the keys crowd into the partitions of the first a."""
    big = [[0.25, 0.25, 0.0], [corner + 0.25, 0.25, 0.0], [0.25, corner + 0.25, 0.0]]
    tiny = []
    for k in range(2047):
        x = 1000.0 + 3.0 * k
        tiny += [[x, 0.0, 500.0], [x + 1.0, 0.0, 500.0], [x, 1.0, 500.0]]
    vA = np.array(big + tiny, dtype=np.float64)
    tA = np.arange(vA.shape[0], dtype=np.uint32).reshape(-1, 3)
    from gpuintersector import meshgen as mg

    vB, tB = mg.grid_mesh(n=n_grid, cell=1.0)
    return dict(vA=vA, tA=tA, vB=vB, tB=tB, poseA=None, poseB=None)


def test_finish_block_partitions_and_crowded_refusal(gi, oc):
    """The one-launch finish with partitions above 32 keys (sorted by a whole
    block), with escalated coplanar pairs (its exact phase), and with a
    partition above its limit (refused, rerun on the general path, kept off the
    finish for the next calls).  All equal the oracle, segments included."""
    with gi.Context(0) as c:
        mid = _crowded_pair(64, 18.0)       # a few hundred keys per partition
        r, ref = run_cfg(c, gi, oc, mid)
        assert 64 < len(ref["pairs"]) < 4096
        assert r.stats["escalated"] > 0
        assert r.stats["launches"] == 2      # traversal + the finish
        assert_same(r, ref)
        crowded = _crowded_pair(128, 88.0)  # ~15 k keys, most in one partition
        r, ref = run_cfg(c, gi, oc, crowded)
        assert 4096 < len(ref["pairs"]) < 24000
        assert r.stats["launches"] > 2       # refused, rerun on the general path
        assert_same(r, ref)
        r, ref = run_cfg(c, gi, oc, mid)     # the next call stays off the finish
        assert r.stats["launches"] > 2
        assert_same(r, ref)


@pytest.mark.parametrize("shape", list(range(8)))
def test_every_traversal_shape(gi, oc, shape):
    """Each traversal shape the autotuner may pick (work queue or level-synchronous
    with grid barriers, expansion per lane or per quad, all resident blocks or
    one per SM) gives the oracle's pairs and segments, in both precision forms
    and in a batch."""
    from gpuintersector import meshgen as mg

    flags = gi._abi.GI_FLAG_FIXED_SHAPE | gi._abi.GI_FLAG_SHAPE(shape)
    cfg = mg.config1(seed=30 + shape)
    with gi.Context(0, flags=flags) as c:
        for prec in (0, 1):
            r, ref = run_cfg(c, gi, oc, cfg, precision=prec)
            assert_same(r, ref)
            assert r.stats["traverse_shape"] == shape
        A, B = c.upload(cfg["vA"], cfg["tA"]), c.upload(cfg["vB"], cfg["tB"])
        rs = c.intersect_batch([(A, None, B, gi_pose(gi, cfg["poseB"])), (B, None, A, None)])
        assert_same(rs[0], ref)
        A.release()
        B.release()


def test_fp64_form_identical(ctx, gi, oc):
    from gpuintersector import meshgen as mg

    cfg = mg.config2(level=6)
    r32, ref = run_cfg(ctx, gi, oc, cfg, precision=0)
    r64, _ = run_cfg(ctx, gi, oc, cfg, precision=1)
    assert_same(r32, ref)
    assert_same(r64, ref)


def test_unsorted_output_same_set(ctx, gi, oc):
    from gpuintersector import meshgen as mg

    cfg = mg.config1(seed=9)
    A, B = ctx.upload(cfg["vA"], cfg["tA"]), ctx.upload(cfg["vB"], cfg["tB"])
    r1 = ctx.intersect(A, B, None, gi_pose(gi, cfg["poseB"]), sort_output=True)
    r2 = ctx.intersect(A, B, None, gi_pose(gi, cfg["poseB"]), sort_output=False)
    assert set(map(tuple, r1.pairs.tolist())) == set(map(tuple, r2.pairs.tolist()))
    A.release()
    B.release()


def test_pose_sweep_like_runsuite(ctx, gi, oc):
    """Seeded random rotations (+-15 deg) and translations (+-0.5) of B about a
    centre, as TestSuite::runSuite (src/CPU/TestSuite.cpp:455-505); FP = FN = 0."""
    from gpuintersector import meshgen as mg

    v, t = mg.uv_sphere(64, 40)
    rng = np.random.default_rng(1337)
    A, B = ctx.upload(v, t), ctx.upload(v, t)
    for step in range(8):
        rot = rng.uniform(-15, 15, 3)
        tr = rng.uniform(-0.5, 0.5, 3)
        cen = [0.01, -0.02, 0.03]
        r = ctx.intersect(A, B, None, gi.pose_from_euler_deg(rot, cen, tr))
        ref = oc.intersect_meshes(v, t, oc.pose_identity(), v, t, oc.pose_from_euler_deg(rot, cen, tr))
        assert_same(r, ref)
    A.release()
    B.release()


def test_both_meshes_posed(ctx, gi, oc):
    from gpuintersector import meshgen as mg

    v, t = mg.icosphere(4)
    rng = np.random.default_rng(5)
    v = mg.displace(v, mg.displacement_params(rng))
    pa = (mg.random_rotation(rng), np.array([0.1, 0.0, -0.2]), np.array([1.0, -2.0, 0.5]))
    pb = (mg.random_rotation(rng), np.array([0.0, 0.3, 0.0]), np.array([1.3, -1.9, 0.4]))
    r, ref = run_cfg(ctx, gi, oc, dict(vA=v, tA=t, vB=v, tB=t, poseA=pa, poseB=pb))
    assert len(ref["pairs"]) > 0
    assert_same(r, ref)


def test_identical_meshes_coplanar_everywhere(ctx, gi, oc):
    """A == B under the identity pose: every pair of neighbours touches or overlaps
    coplanarly -- the exact stage decides almost every candidate."""
    from gpuintersector import meshgen as mg

    v, t = mg.uv_sphere(16, 10)
    r, ref = run_cfg(ctx, gi, oc, dict(vA=v, tA=t, vB=v, tB=t, poseA=None, poseB=None))
    assert len(ref["pairs"]) > t.shape[0]
    assert_same(r, ref)
    assert r.stats["escalated"] > 0


def test_batch_equals_individual(ctx, gi, oc):
    from gpuintersector import meshgen as mg

    jobs = mg.config4(seed=8, pairs=6, t_min=200, t_max=4000)
    meshes, bjobs, refs = [], [], []
    for j in jobs:
        A, B = ctx.upload(j["vA"], j["tA"]), ctx.upload(j["vB"], j["tB"])
        meshes += [A, B]
        bjobs.append((A, None, B, gi_pose(gi, j["poseB"])))
        refs.append(oc.intersect_meshes(j["vA"], j["tA"], oc.pose_identity(), j["vB"], j["tB"],
                                        oracle_pose(oc, j["poseB"])))
    res = ctx.intersect_batch(bjobs)
    assert sum(len(r["pairs"]) for r in refs) > 0
    for r, ref, (A, pa, B, pb) in zip(res, refs, bjobs):
        assert_same(r, ref)
        single = ctx.intersect(A, B, pa, pb)
        assert_same(single, ref)
    for m in meshes:
        m.release()


def test_config4_full_batch_sampled_vs_oracle(ctx, gi, oc):
    """The full batched configuration (4,096 mesh pairs of displaced geodesic
    spheres, 1k-200k triangles per mesh, B offset by 0.2-1.5 radius and rotated)
    in one gi_intersect_batch call; 64 jobs spread evenly over the size range
    are compared with the oracle (pair sets and endpoints), as the reference's
    suite compares every step with its ground truth (src/CPU/TestSuite.cpp:235-321)."""
    from types import SimpleNamespace

    from gpuintersector import meshgen as mg

    sizes = np.array([a + b for a, b in mg.config4_sizes(seed=4)])
    order = np.argsort(sizes, kind="stable")
    pick = set(order[np.linspace(0, len(sizes) - 1, 64).astype(int)].tolist())
    meshes, jobs, kept = [], [], {}
    for p, j in enumerate(mg.config4_iter(seed=4)):
        A, B = ctx.upload(j["vA"], j["tA"]), ctx.upload(j["vB"], j["tB"])
        meshes += [A, B]
        jobs.append((A, None, B, gi_pose(gi, j["poseB"])))
        if p in pick:
            kept[p] = j
    assert len(jobs) == 4096 and len(kept) == 64
    flat = ctx.intersect_batch_flat(jobs, want_segments=True)
    assert len(flat.pairs) > 1_000_000
    nonempty = 0
    for p in sorted(kept):
        j = kept[p]
        ref = oc.intersect_meshes(j["vA"], j["tA"], oc.pose_identity(), j["vB"], j["tB"],
                                  oracle_pose(oc, j["poseB"]), want_segments=True)
        a, e = flat.offsets[p], flat.offsets[p + 1]
        sel = (flat.seg_pair >= a) & (flat.seg_pair < e)
        got = SimpleNamespace(pairs=flat.pairs[a:e], segments=flat.segments[sel], seg_pair=flat.seg_pair[sel] - a)
        assert_same(got, ref)
        nonempty += len(ref["pairs"]) > 0
    assert nonempty >= 32
    del flat
    for m in meshes:
        m.release()


def test_classify_pairs_after_wait_stream(ctx, gi, oc):
    """Inputs produced on a side stream of the caller reach gi_classify_pairs
    through gi_wait_stream (the library's stream waits for the caller's work)."""
    import torch
    from gpuintersector import meshgen as mg

    cfg = mg.config1(seed=12)
    rng = np.random.default_rng(4)
    pairs, _ = _candidate_pairs(cfg, oc, rng, n_random=20000)
    exp = oc.classify_pairs(cfg["vA"], cfg["tA"], oc.pose_identity(), cfg["vB"], cfg["tB"],
                            oracle_pose(oc, cfg["poseB"]), pairs)
    A, B = ctx.upload(cfg["vA"], cfg["tA"]), ctx.upload(cfg["vB"], cfg["tB"])
    side = torch.cuda.Stream()
    host = torch.from_numpy(pairs).pin_memory()
    with torch.cuda.stream(side):
        d_pairs = host.to("cuda", non_blocking=True)
        d_out = torch.full((len(pairs),), 7, dtype=torch.uint8, device="cuda")
    ctx.wait_stream(side.cuda_stream)
    ctx.classify_pairs(A, B, None, gi_pose(gi, cfg["poseB"]), d_pairs.data_ptr(), len(pairs), d_out.data_ptr())
    assert np.array_equal(d_out.cpu().numpy(), exp)
    A.release()
    B.release()


def test_batch_flat_matches_per_job_results(ctx, gi):
    """intersect_batch_flat: the same pairs, segments and segment grouping as the
    per-job results, as whole-batch arrays (jobs with no pair included)."""
    from gpuintersector import meshgen as mg

    jobs = mg.config4(seed=9, pairs=12, t_min=200, t_max=3000)
    meshes, bjobs = [], []
    for k, j in enumerate(jobs):
        A, B = ctx.upload(j["vA"], j["tA"]), ctx.upload(j["vB"], j["tB"])
        meshes += [A, B]
        pose = gi_pose(gi, j["poseB"])
        if k % 5 == 4:  # far apart: a job with no pair
            R, C, T = j["poseB"]
            pose = gi.pose_raw(R, C, np.asarray(T) + 50.0)
        bjobs.append((A, None, B, pose))
    per = ctx.intersect_batch(bjobs)
    flat = ctx.intersect_batch_flat(bjobs)
    assert flat.offsets.shape == (len(jobs) + 1,)
    assert any(len(r.pairs) == 0 for r in per) and sum(len(r.pairs) for r in per) > 0
    for k, r in enumerate(per):
        a, e = flat.offsets[k], flat.offsets[k + 1]
        assert np.array_equal(flat.pairs[a:e], r.pairs)
        assert np.all(flat.job[a:e] == k)
        sel = (flat.seg_pair >= a) & (flat.seg_pair < e)
        assert np.array_equal(flat.segments[sel], r.segments)
        assert np.array_equal(flat.seg_pair[sel] - a, r.seg_pair)
    assert flat.stats["pairs"] == len(per[0].pairs)
    del per, flat
    for m in meshes:
        m.release()


def test_oneshot_and_controller_mirror(ctx, gi, oc):
    from gpuintersector import meshgen as mg

    v, t = mg.uv_sphere(48, 30)
    rot, cen, tr = [5.0, 10.0, -12.0], [0.0, 0.0, 0.0], [0.6, 0.05, 0.0]
    ref = oc.intersect_meshes(v, t, oc.pose_identity(), v, t, oc.pose_from_euler_deg(rot, cen, tr))
    r = ctx.intersect_oneshot(v, t, v, t, None, gi.pose_from_euler_deg(rot, cen, tr))
    assert_same(r, ref)
    r2 = gi.run_grid_forest_intersection_pipeline(v, t, v, t, rotB=rot, transB=tr, ctx=ctx, want_segments=True)
    assert_same(r2, ref)
    kc = gi.KernelBVHController()
    kc.construct(v, t, 12, v, t, 12, 4)
    kc.setTransformBoth([0, 0, 0], [0, 0, 0], rot, tr)
    pairs = kc.runIntersectionPipeline(1, 0, 0, 1)
    assert np.array_equal(pairs, ref["pairs"])
    kc.clearGPU()
    assert not kc.isGPUAllocated()
    kc.reconstructGPU()
    assert np.array_equal(kc.runIntersectionPipeline(), ref["pairs"])
    kc.cleanup()


def test_degenerate_triangles_in_meshes(ctx, gi, oc):
    from gpuintersector import meshgen as mg

    v, t = mg.uv_sphere(20, 12)
    rng = np.random.default_rng(2)
    t = t.copy()
    # collapse some triangles to segments and points
    for k in rng.choice(t.shape[0], 30, replace=False):
        t[k, 2] = t[k, 1] if k % 2 else t[k, 0]
    v2 = np.concatenate([v, [[0.1, 0.2, 0.3], [0.3, 0.6, 0.9], [0.2, 0.4, 0.6]]])
    t2 = np.concatenate([t, [[v.shape[0], v.shape[0] + 1, v.shape[0] + 2]]]).astype(np.uint32)  # collinear
    R = mg.random_rotation(rng)
    r, ref = run_cfg(ctx, gi, oc, dict(vA=v2, tA=t2, vB=v2, tB=t2, poseA=None, poseB=(R, np.zeros(3),
                                                                                      np.array([0.3, 0, 0]))))
    assert_same(r, ref)
    r, ref = run_cfg(ctx, gi, oc, dict(vA=v2, tA=t2, vB=v2, tB=t2, poseA=None, poseB=None))
    assert_same(r, ref)


def test_empty_and_tiny_meshes(ctx, gi, oc):
    one = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], float)
    tri = np.array([[0, 1, 2]], np.uint32)
    A = ctx.upload(one, tri)
    E = ctx.upload(one, np.zeros((0, 3), np.uint32))
    r = ctx.intersect(A, E)
    assert r.pairs.shape == (0, 2)
    r = ctx.intersect(A, A)
    assert r.pairs.tolist() == [[0, 0]] and r.segments.shape[0] == 3
    for m in (A, E):
        m.release()


def test_far_from_origin_and_scaled(ctx, gi, oc):
    from gpuintersector import meshgen as mg

    v, t = mg.icosphere(3)
    v = v * 1e-3 + np.array([1e5, -3e4, 7.0])
    R = mg.random_rotation(np.random.default_rng(4))
    cen = np.array([1e5, -3e4, 7.0])
    r, ref = run_cfg(ctx, gi, oc, dict(vA=v, tA=t, vB=v, tB=t, poseA=None,
                                       poseB=(R, cen, np.array([6e-4, 0.0, 0.0]))))
    assert len(ref["pairs"]) > 0
    assert_same(r, ref)


def test_invalid_inputs_are_reported(ctx, gi):
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], float)
    with pytest.raises(gi.GIError) as e:
        ctx.upload(v, np.array([[0, 1, 7]], np.uint32))
    assert e.value.status == 1
    with pytest.raises(gi.GIError) as e:
        ctx.upload(np.array([[0, 0, np.nan], [1, 0, 0], [0, 1, 0]]), np.array([[0, 1, 2]], np.uint32))
    assert e.value.status == 6
    with pytest.raises(gi.GIError) as e:
        ctx.upload(np.array([[0, 0, 1e40], [1, 0, 0], [0, 1, 0]]), np.array([[0, 1, 2]], np.uint32))
    assert e.value.status == 6
    A = ctx.upload(v, np.array([[0, 1, 2]], np.uint32))
    bad = gi.pose_raw(np.eye(3), (0, 0, 0), (1e300, 0, 0))
    with pytest.raises(gi.GIError) as e:
        ctx.intersect(A, A, None, bad)
    assert e.value.status == 6
    A.release()


def test_capacity_retry_path(gi, oc):
    """Host-side fault injection: every buffer starts at 64 entries, so the
    overflow flags fire and the call grows its buffers and re-runs."""
    from gpuintersector import meshgen as mg

    cfg = mg.config1(seed=4)
    for shape in (None, 1, 5):  # tuned, the work-queue traversal, the level-synchronous one
        flags = gi._abi.GI_FLAG_TINY_BUFFERS
        if shape is not None:
            flags |= gi._abi.GI_FLAG_FIXED_SHAPE | gi._abi.GI_FLAG_SHAPE(shape)
        with gi.Context(0, flags=flags) as c:
            r, ref = run_cfg(c, gi, oc, cfg)
        assert r.stats["retries"] > 0
        assert_same(r, ref)


def test_hbm_budget_admission(gi):
    from gpuintersector import meshgen as mg

    v, t = mg.icosphere(5)
    with gi.Context(0, hbm_budget_bytes=1 << 20) as c:
        with pytest.raises(gi.GIError) as e:
            c.upload(v, t)
        assert e.value.status == 2


def test_server_results_alone_and_in_mix(ctx, gi):
    """Continuous batching: requests that arrive while others run are admitted
    into later device rounds; every result equals the one computed alone."""
    from gpuintersector import meshgen as mg

    v, t = mg.icosphere(4)
    v = mg.displace(v, mg.displacement_params(np.random.default_rng(6)))
    A, B = ctx.upload(v, t), ctx.upload(v, t)
    rng = np.random.default_rng(7)
    poses = []
    for R, tr in mg.pose_stream(rng, 24, 5.0, 0.05):
        poses.append(gi.pose_raw(R, (0, 0, 0), tr + np.array([0.35, 0.0, 0.0])))
    alone = [ctx.intersect(A, B, None, p) for p in poses]
    srv = ctx.server(max_inflight=5)
    tickets = [srv.submit(A, None, B, p) for p in poses]
    mixed = [srv.wait(tk) for tk in tickets]
    srv.stop()
    for a, m in zip(alone, mixed):
        assert np.array_equal(a.pairs, m.pairs)
        assert np.array_equal(a.segments, m.segments)
    A.release()
    B.release()


def _candidate_pairs(cfg, oc, rng, n_random=4000):
    """Exact-box-overlapping pairs from the oracle's BVH plus random pairs."""
    ref = oc.intersect_meshes(cfg["vA"], cfg["tA"], oracle_pose(oc, cfg["poseA"]), cfg["vB"], cfg["tB"],
                              oracle_pose(oc, cfg["poseB"]), want_segments=False)
    rand = np.stack([rng.integers(0, cfg["tA"].shape[0], n_random), rng.integers(0, cfg["tB"].shape[0], n_random)],
                    axis=1)
    return np.concatenate([ref["pairs"], rand]).astype(np.int32), ref


def test_classify_pairs_vs_oracle(ctx, gi, oc):
    """gi_classify_pairs over an explicit list equals the oracle's exact test."""
    import torch
    from gpuintersector import meshgen as mg

    cfg = mg.config1(seed=11)
    rng = np.random.default_rng(3)
    pairs, ref = _candidate_pairs(cfg, oc, rng)
    wA = oc.transform(oracle_pose(oc, cfg["poseA"]), cfg["vA"])
    wB = oc.transform(oracle_pose(oc, cfg["poseB"]), cfg["vB"])
    exp = np.array([oc.tri_tri_intersect(wA[cfg["tA"][a]], wB[cfg["tB"][b]]) for a, b in pairs], dtype=np.uint8)
    A, B = ctx.upload(cfg["vA"], cfg["tA"]), ctx.upload(cfg["vB"], cfg["tB"])
    d_pairs = torch.from_numpy(pairs).cuda()
    for prec in (0, 1):
        d_out = torch.full((len(pairs),), 7, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()  # the library's stream is not ordered after torch's
        ctx.classify_pairs(A, B, None, gi_pose(gi, cfg["poseB"]), d_pairs.data_ptr(), len(pairs), d_out.data_ptr(),
                           precision=prec)
        torch.cuda.synchronize()
        assert np.array_equal(d_out.cpu().numpy(), exp)
    assert exp[:len(ref["pairs"])].all()
    bad = torch.tensor([[0, cfg["tB"].shape[0]]], dtype=torch.int32, device="cuda")
    out = torch.zeros(1, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    with pytest.raises(gi.GIError) as e:
        ctx.classify_pairs(A, B, None, None, bad.data_ptr(), 1, out.data_ptr())
    assert e.value.status == 1
    A.release()
    B.release()
