"""Serving: HBM admission of resident mesh pairs (CPU, with a fake context) and
a short Poisson pose-update stream through the C-ABI server (GPU)."""
import numpy as np
import pytest


class _FakeMesh:
    def __init__(self, ctx, nbytes):
        self.ctx, self.nbytes = ctx, nbytes
        ctx.used += nbytes

    def release(self):
        self.ctx.used -= self.nbytes
        self.ctx.released += 1


class _FakeCtx:
    """Uploads cost 100 bytes per vertex array row; over budget -> GIError(OOM)."""

    def __init__(self, gi, budget):
        self.gi, self.budget, self.used, self.released = gi, budget, 0, 0

    def upload(self, v, t):
        nb = 100 * len(v)
        if self.used + nb > self.budget:
            raise self.gi.GIError(self.gi._abi.GI_ERR_OOM, "budget")
        return _FakeMesh(self, nb)


def test_resident_set_admits_and_evicts_lru(gi):
    from gpuintersector.serving import ResidentSet

    pairs = [(np.zeros((10, 3)), None, np.zeros((10, 3)), None) for _ in range(4)]  # 2000 bytes per pair
    ctx = _FakeCtx(gi, budget=4500)  # two pairs fit
    rs = ResidentSet(ctx, pairs)
    rs.acquire(0)
    rs.acquire(1)
    assert rs.admissions == 2 and rs.evictions == 0
    rs.release(0)
    rs.release(1)
    rs.acquire(0)  # hit: 0 becomes most recent
    rs.release(0)
    rs.acquire(2)  # evicts 1 (least recently used, idle)
    assert rs.evictions == 1 and set(rs.res) == {0, 2}
    # a pair in flight is never evicted: with 0 and 2 both in flight, 3 cannot be admitted
    rs.acquire(0)
    with pytest.raises(RuntimeError):
        rs.acquire(3, wait_s=0.01)
    rs.release(0)
    rs.release(0)
    rs.release(2)
    rs.acquire(3)
    assert 3 in rs.res and ctx.used <= ctx.budget
    rs.close()
    assert ctx.used == 0


@pytest.mark.gpu
def test_poisson_serving_with_admission(gi):
    from gpuintersector import meshgen as mg
    from gpuintersector.serving import ResidentSet, poisson_serving

    rng = np.random.default_rng(8)
    pairs, poses = [], []
    for k in range(6):
        u, t = mg.geodesic_sphere(int(rng.integers(10, 25)))
        vA = mg.displace(u, mg.displacement_params(rng))
        vB = mg.displace(u, mg.displacement_params(rng))
        pairs.append((vA, t, vB, t))
        poses.append((mg.random_rotation(rng), np.zeros(3), np.array([0.4, 0.0, 0.0])))
    with gi.Context(0) as probe:
        m = probe.upload(pairs[0][0], pairs[0][1])
        per_mesh = m.info()["bytes"]
        m.release()
    with gi.Context(0, hbm_budget_bytes=int(per_mesh * 2 * 3.5)) as ctx:  # about three of six pairs fit
        rs = ResidentSet(ctx, pairs)
        out = poisson_serving(ctx, rs, poses, rate=400.0, duration=0.5, seed=3)
        rs.close()
    assert out["completed"] == out["requests"] > 0
    assert out["evictions"] > 0 and out["admissions"] > 3
    assert out["p99_ms"] is not None
