"""Pose-update serving over resident BVHs: HBM admission and a Poisson driver.

The reference recomputes every pose update from the host (KernelBVHController::
setTransformBoth, src/GPUIntersector/KernelBVHController.cu:289-412, followed
by runIntersectionPipeline).  Here meshes stay resident with their BVHs and a
request is only a pose: the C-ABI server (gi_server_*) admits pending requests
into device rounds as earlier rounds finish (continuous batching).

ResidentSet keeps mesh pairs uploaded within the context's HBM budget
(gi_options.hbm_budget_bytes; gi_mesh_upload returns GI_ERR_OOM past it).  A
request for a pair that is not resident admits it, evicting the least recently
used pairs that have no request in flight until the upload fits.

poisson_serving() submits pose updates at Poisson arrival times and records
each request's latency from submission to a finished result on the host.
"""
import collections
import sys
import threading
import time

import numpy as np

from . import _abi


class ResidentSet:
    """LRU set of resident mesh pairs under the context's HBM budget.

    pairs: list of (vA, tA, vB, tB) host arrays (kept by the caller)."""

    def __init__(self, ctx, pairs):
        self.ctx = ctx
        self.pairs = pairs
        self.res = collections.OrderedDict()  # k -> (A, B), least recently used first
        self.inflight = collections.Counter()
        self.lock = threading.Lock()
        self.admissions = 0
        self.evictions = 0

    def _evict_one(self):
        for k in self.res:
            if self.inflight[k] == 0:
                A, B = self.res.pop(k)
                A.release()
                B.release()
                self.evictions += 1
                return True
        return False

    def acquire(self, k, wait_s=5.0):
        """Mesh handles of pair k, resident and counted as in flight until release(k)."""
        t_end = time.perf_counter() + wait_s
        while True:
            with self.lock:
                if k in self.res:
                    self.res.move_to_end(k)
                    self.inflight[k] += 1
                    return self.res[k]
                vA, tA, vB, tB = self.pairs[k]
                A = B = None
                while True:
                    try:
                        if A is None:
                            A = self.ctx.upload(vA, tA)
                        B = self.ctx.upload(vB, tB)
                        break
                    except Exception as e:  # over budget: make room
                        if getattr(e, "status", None) != _abi.GI_ERR_OOM or not self._evict_one():
                            if A is not None:
                                A.release()
                            A = None
                            break
                if A is not None and B is not None:
                    self.res[k] = (A, B)
                    self.admissions += 1
                    self.inflight[k] += 1
                    return A, B
            if time.perf_counter() > t_end:
                raise RuntimeError("pair %d cannot be admitted within the HBM budget" % k)
            time.sleep(0.0005)  # every resident pair is in flight: wait for completions

    def release(self, k):
        with self.lock:
            self.inflight[k] -= 1

    def close(self):
        with self.lock:
            for A, B in self.res.values():
                A.release()
                B.release()
            self.res.clear()


def poisson_serving(ctx, resident, base_poses, rate, duration, seed=0, max_rot_deg=5.0, max_trans=0.05,
                    max_inflight=256, want_segments=False):
    """Serve pose updates arriving as a Poisson stream of `rate` requests/s for
    `duration` seconds, each for a uniformly chosen pair with a small rigid
    update of B around its base pose.  Returns a dict of latencies (ms), counts
    and rates."""
    from . import meshgen as mg
    from . import pose_raw

    rng = np.random.default_rng(seed)
    npairs = len(base_poses)
    n_req = max(1, int(rate * duration))
    gaps = rng.exponential(1.0 / rate, n_req)
    arrivals = np.cumsum(gaps)
    choice = rng.integers(0, npairs, n_req)
    updates = mg.pose_stream(rng, n_req, max_rot_deg, max_trans)
    server = ctx.server(max_inflight=max_inflight, want_segments=want_segments)
    submit_t = {}
    done_t = {}
    pair_of = {}
    npairs_found = [0]
    outstanding = collections.deque()
    lock = threading.Lock()
    stop = threading.Event()

    def collect():
        while not (stop.is_set() and not outstanding):
            with lock:
                pending = list(outstanding)
            finished = []
            for t in pending:
                r = server.poll(t)
                if r is not None:
                    done_t[t] = time.perf_counter()
                    npairs_found[0] += len(r.pairs)
                    resident.release(pair_of[t])
                    finished.append(t)
            if finished:
                with lock:
                    for t in finished:
                        outstanding.remove(t)
            else:
                time.sleep(0.00002)

    # the submitting loop and the collector share the interpreter lock: hand it
    # over often, and sleep (releasing it) until shortly before each arrival
    old_switch = sys.getswitchinterval()
    sys.setswitchinterval(0.0005)
    th = threading.Thread(target=collect, daemon=True)
    th.start()
    t0 = time.perf_counter()
    for q in range(n_req):
        ahead = arrivals[q] - (time.perf_counter() - t0)
        if ahead > 0.0004:
            time.sleep(ahead - 0.0003)
        while time.perf_counter() - t0 < arrivals[q]:
            pass
        k = int(choice[q])
        R0, C0, T0 = base_poses[k]
        dR, dt = updates[q]
        A, B = resident.acquire(k)
        ts = time.perf_counter()
        ticket = server.submit(A, None, B, pose_raw(dR @ R0, C0, T0 + dt))
        with lock:
            submit_t[ticket] = ts
            pair_of[ticket] = k
            outstanding.append(ticket)
    stop.set()
    th.join(timeout=60)
    wall = time.perf_counter() - t0
    sys.setswitchinterval(old_switch)
    server.stop()
    order = sorted(t for t in submit_t if t in done_t)
    lat = np.array([(done_t[t] - submit_t[t]) * 1e3 for t in order])
    half = lat.size // 2
    halves = [dict(p50_ms=float(np.percentile(h, 50)), p99_ms=float(np.percentile(h, 99)))
              for h in (lat[:half], lat[half:]) if h.size]
    return dict(requests=n_req, completed=int(lat.size), offered_rate=rate, wall_s=wall,
                achieved_rate=lat.size / wall, p50_ms=float(np.percentile(lat, 50)) if lat.size else None,
                p99_ms=float(np.percentile(lat, 99)) if lat.size else None,
                max_ms=float(lat.max()) if lat.size else None, pairs_found=npairs_found[0],
                pairs_per_s=npairs_found[0] / wall, admissions=resident.admissions, evictions=resident.evictions,
                by_half=halves)
