"""Sharding of independent mesh-pair jobs across ranks (one process per GPU).

Batched and serving workloads are sets of independent mesh pairs: no pair
needs data from another, so ranks split the jobs and run them with no
collective on the data path.  The only exchange is the final gather of the
per-job results to the host of rank 0 (torch.distributed object gather, over
NCCL's host-side store or gloo).

Assignment is greedy longest-processing-time first on an estimated cost
(triangle count of both meshes, the traversal's dominant term): jobs sorted by
cost, each given to the currently least-loaded rank.  Every rank computes the
same assignment from the same inputs, so no message is needed to agree on it.
"""
import heapq


def job_cost(tris_a, tris_b):
    """Estimated cost of one pair: build-free traversal work grows with both trees."""
    return float(tris_a) + float(tris_b)


def assign(costs, world):
    """Greedy LPT: list of job-index lists, one per rank; deterministic for equal costs."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    for lst in out:
        lst.sort()
    return out


def loads(costs, parts):
    return [sum(costs[i] for i in p) for p in parts]


def run_sharded(costs, execute, rank, world, dist=None, dst=0):
    """Runs this rank's share with execute(job_indices) -> {job: result} and gathers
    every rank's results to rank `dst` (returns the merged dict there, None elsewhere).
    With world == 1 or dist None it just runs everything locally."""
    parts = assign(costs, world)
    mine = parts[rank]
    local = execute(mine) if mine else {}
    if world == 1 or dist is None:
        return local
    gathered = [None] * world if rank == dst else None
    dist.gather_object(local, gathered, dst=dst)
    if rank != dst:
        return None
    merged = {}
    for part in gathered:
        merged.update(part)
    return merged
