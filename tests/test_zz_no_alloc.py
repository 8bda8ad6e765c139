"""gi_classify_pairs_noalloc against gi_classify_pairs and the oracle (GPU;
collected last).

The no-alloc entry point keeps its escalation list in a fixed per-device array
inside the library instead of the context's stream-ordered pool, for callers
that may not allocate device memory while they run.  Both entry points are
compared with each other on two calls in a row and with the exact CPU oracle
(oc.classify_pairs) on the same lists.  The library works on its context's own
stream, so the test synchronises the device after torch has filled the input
and output tensors and before the library's calls read and write them.  This
file is named to run after every other test file so that it also runs with the
library already warmed by them; it is self-contained and passes alone as well.
"""
import numpy as np
import pytest

from conftest import gi_pose, oracle_pose

pytestmark = pytest.mark.gpu


def _pairs(cfg, rng, n):
    """Candidate pairs: near pairs (A triangle i with B triangles around i) plus random ones."""
    nA, nB = cfg["tA"].shape[0], cfg["tB"].shape[0]
    a = rng.integers(0, nA, n)
    near = np.clip(a + rng.integers(-64, 64, n), 0, nB - 1)
    far = rng.integers(0, nB, n)
    b = np.where(rng.random(n) < 0.5, near, far)
    return np.stack([a, b], axis=1).astype(np.int32)


def test_noalloc_matches_classify_pairs_two_calls(ctx, gi, oc):
    import torch
    from gpuintersector import meshgen as mg

    # the coplanar grids (B coplanar with A, shifted half a cell, tiles at z = -1,
    # 0, +1) escalate most pairs, so the scratch list is used
    hits = 0
    for cfg, n in ((mg.config1(seed=5), 200000), (mg.config3(n=32, seed=2), 60000),
                   (mg.config3(n=512, seed=3), 400000)):
        rng = np.random.default_rng(17)
        A, B = ctx.upload(cfg["vA"], cfg["tA"]), ctx.upload(cfg["vB"], cfg["tB"])
        pb = gi_pose(gi, cfg["poseB"])
        pa = gi_pose(gi, cfg["poseA"])
        for prec in (gi.GI_PREC_FP32_CASCADE, gi.GI_PREC_FP64):
            for call in range(2):  # two calls in a row on the same fixed scratch
                pairs = _pairs(cfg, rng, n)
                exp = oc.classify_pairs(cfg["vA"], cfg["tA"], oracle_pose(oc, cfg["poseA"]), cfg["vB"], cfg["tB"],
                                        oracle_pose(oc, cfg["poseB"]), pairs)
                d_pairs = torch.from_numpy(pairs).cuda()
                ref = torch.full((n,), 7, dtype=torch.uint8, device="cuda")
                out = torch.full((n,), 9, dtype=torch.uint8, device="cuda")
                torch.cuda.synchronize()  # inputs and fills complete before the library's stream reads them
                ctx.classify_pairs(A, B, pa, pb, d_pairs.data_ptr(), n, ref.data_ptr(), precision=prec)
                ctx.classify_pairs_noalloc(A, B, pa, pb, d_pairs.data_ptr(), n, out.data_ptr(), precision=prec)
                torch.cuda.synchronize()
                r, o = ref.cpu().numpy(), out.cpu().numpy()
                assert set(np.unique(r)) <= {0, 1}
                assert np.array_equal(r, o), (prec, call)
                assert np.array_equal(o, exp), ("oracle", prec, call)
                hits += int(exp.sum())
        A.release()
        B.release()
    assert hits > 0, "the lists must hold intersecting pairs"


def test_noalloc_limits(ctx, gi):
    import torch
    from gpuintersector import meshgen as mg

    cfg = mg.config1(seed=5)
    A, B = ctx.upload(cfg["vA"], cfg["tA"]), ctx.upload(cfg["vB"], cfg["tB"])
    d_pairs = torch.zeros((2, 2), dtype=torch.int32, device="cuda")
    out = torch.zeros(2, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    # above the fixed limit: rejected before any access to the (short) buffers
    with pytest.raises(gi.GIError) as e:
        ctx.classify_pairs_noalloc(A, B, None, None, d_pairs.data_ptr(), gi.GI_NOALLOC_MAX_PAIRS + 1,
                                   out.data_ptr())
    assert e.value.status == 3
    # bad index: same error as the allocating entry point
    bad = torch.tensor([[0, cfg["tB"].shape[0]]], dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    with pytest.raises(gi.GIError) as e:
        ctx.classify_pairs_noalloc(A, B, None, None, bad.data_ptr(), 1, out.data_ptr())
    assert e.value.status == 1
    # an empty call and a valid call afterwards still work
    ctx.classify_pairs_noalloc(A, B, None, None, 0, 0, 0)
    ok = torch.tensor([[0, 0]], dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ctx.classify_pairs_noalloc(A, B, None, None, ok.data_ptr(), 1, out.data_ptr())
    A.release()
    B.release()
