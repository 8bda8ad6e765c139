"""Benchmark of the mesh-mesh intersection hot path (one JSON line on rank 0).

Workload (the large precision-cascade configuration): two level-8 displaced
icospheres, 1,310,720 triangles each, FP64 vertices; B offset (0.3, 0.1, 0)
plus a seeded rotation.  A step is one intersection under a new rigid pose of
B (a seeded stream of small updates, <= 5 degrees and <= 0.05 radius, around
the base pose): the pose-update path of the reference's compute command
(KernelBVHController::setTransformBoth + runIntersectionPipeline), producing
the exact intersecting pair set and the intersection segments.

  value      device time per intersect (library CUDA events on its stream,
             traversal -> exact stage -> segments -> ordering), meshes and BVHs
             resident in HBM, L2 flushed (256 MB write) before every step.
  e2e        the one-shot C-ABI call with HOST arrays
             (gi_intersect_oneshot = runGridForestIntersectionPipeline):
             H2D of both meshes, BVH builds, intersect, D2H of pairs+segments.
  pose_update  wall-clock latency of gi_intersect with resident meshes
             (pose in, results on the host), p50 / p99.
  fp64_form  the same steps with FP64 boxes and FP64 filters (plain FP64 form).
  cpu_baseline  the exact CPU oracle (same semantics; the reference's own CPU
             path needs CGAL and cannot be built here) on all host cores.

--impl reference times that CPU implementation on the same workload.
Multi-GPU: replicas only (each rank runs the same independent workload, no
collective on the data path); value = max-over-ranks time / intersects done.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "gpu-cubql-intersector-standalone_b200")
sys.path.insert(0, PKG)

METRIC = "ms/intersect at 2×1.3M tris & tri-pair tests/s; pose-update p50/p99 vs FP64 path"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--level", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    return ap.parse_args()


def workload(level):
    from gpuintersector import meshgen as mg

    cfg = mg.config2(level=level)
    rng = np.random.default_rng(22)
    return cfg, rng


def step_poses(cfg, rng, n):
    """Base pose of B composed with a stream of small rigid updates."""
    from gpuintersector import meshgen as mg

    R0, C0, T0 = cfg["poseB"]
    out = []
    for dR, dt in mg.pose_stream(rng, n, 5.0, 0.05):
        out.append((dR @ R0, C0, T0 + dt))
    return out


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, n in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def cpu_oracle_run(cfg, poses, nthreads):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as oc

    oc.build()
    ms, last = [], None
    for (R, C, T) in poses:
        t0 = time.perf_counter()
        last = oc.intersect_meshes(cfg["vA"], cfg["tA"], oc.pose_identity(), cfg["vB"], cfg["tB"],
                                   oc.pose_raw(R, C, T), want_segments=True, nthreads=nthreads)
        ms.append((time.perf_counter() - t0) * 1e3)
    return ms, last


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def run_reference(args):
    """The reference path's CPU implementation (the exact oracle port) on the host cores."""
    cfg, rng = workload(args.level)
    poses = step_poses(cfg, rng, args.warmup + args.steps)
    ncores = os.cpu_count() or 1
    ms, last = cpu_oracle_run(cfg, poses[:args.warmup], ncores)
    ms, last = cpu_oracle_run(cfg, poses[args.warmup:], ncores)
    v = float(np.mean(ms))
    line = {
        "metric": METRIC, "impl": "reference", "value": v, "unit": "ms", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": v, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded displaced icospheres)",
        "config": {"workload": "icosphere L8 displaced x2 (1,310,720 tris each), pose-update stream",
                   "tris_per_mesh": int(cfg["tA"].shape[0]), "parallelism": "cpu threads"},
        "cpu_baseline": {"value": v, "unit": "ms", "cores": ncores, "kind": "port",
                         "sample": "full intersect (BVH over B + exact predicates + segments) per step, "
                                   "%d steps; CPU %s" % (args.steps, cpu_model())},
        "e2e": {"value": v, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "pairs": int(len(last["pairs"])),
        "note": "the reference's CPU/CGAL path cannot be built here (CGAL, Boost, TBB, cuBQL absent); "
                "this arm times the exact C oracle restating its semantics",
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(local)
    import gpuintersector as gi

    cfg, rng = workload(args.level)
    poses = step_poses(cfg, rng, args.warmup + args.steps)
    ctx = gi.Context(local)
    A = ctx.upload(cfg["vA"], cfg["tA"])
    B = ctx.upload(cfg["vB"], cfg["tB"])
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def one(pose, precision=0):
        R, C, T = pose
        return ctx.intersect(A, B, None, gi.pose_raw(R, C, T), want_segments=True, precision=precision)

    for k in range(args.warmup):
        one(poses[k])
        one(poses[k], precision=1)
    torch.cuda.synchronize()
    dev_ms, wall_ms, trav_ms, stats = [], [], [], []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        for k in range(args.steps):
            flush.fill_(k & 255)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = one(poses[args.warmup + k])
            wall_ms.append((time.perf_counter() - t0) * 1e3)
            dev_ms.append(r.stats["ms_total"])
            trav_ms.append(r.stats["ms_traverse"])
            stats.append(r.stats)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    total = float(np.sum(dev_ms))
    if dist:
        t = torch.tensor([total], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total = float(t.item())
    value = total / (args.steps * world)

    # plain FP64 form on the same poses
    fp64_ms = []
    for k in range(args.steps):
        flush.fill_(k & 255)
        torch.cuda.synchronize()
        r64 = one(poses[args.warmup + k], precision=1)
        fp64_ms.append(r64.stats["ms_total"])
        assert np.array_equal(r64.pairs, r.pairs) or k != args.steps - 1

    # e2e: one-shot from host arrays
    e2e_ms = []
    last_e2e = None
    for k in range(args.e2e_steps):
        R, C, T = poses[args.warmup + k]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        last_e2e = ctx.intersect_oneshot(cfg["vA"], cfg["tA"], cfg["vB"], cfg["tB"], None, gi.pose_raw(R, C, T))
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    h2d = int(cfg["vA"].nbytes + cfg["tA"].astype(np.uint32).nbytes + cfg["vB"].nbytes +
              cfg["tB"].astype(np.uint32).nbytes)
    d2h = int(last_e2e.pairs.nbytes + last_e2e.segments.nbytes + last_e2e.seg_pair.nbytes)

    st = stats[-1]
    cand = np.mean([s["candidates"] for s in stats])
    tests_per_s = float(np.sum([s["candidates"] for s in stats]) / (np.sum(trav_ms) / 1e3))
    # roofline of the dominant kernel (traversal + first filter)
    node_bytes = 2 * 128
    tri_bytes = 2 * (16 + 3 * 24)
    alg_bytes = np.mean([s["node_pairs"] * node_bytes + s["candidates"] * tri_bytes + s["pairs"] * 16
                         for s in stats])
    trav = float(np.mean(trav_ms))
    achieved = alg_bytes / (trav * 1e-3) / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    line = {
        "metric": METRIC, "value": value, "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": value, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded displaced icospheres, seeded pose stream)",
        "config": {"workload": "icosphere L%d displaced x2 (%d tris each), pose-update stream" % (
            args.level, int(cfg["tA"].shape[0])), "tris_per_mesh": int(cfg["tA"].shape[0]),
            "parallelism": "replicas" if world > 1 else "single", "l2": "flushed (256 MB write) before each step",
            "precision": "fp32 filter -> fp64 filter -> exact", "segments": True},
        "pairs": int(st["pairs"]), "segments": int(st["segments"]), "candidates": int(cand),
        "tri_pair_tests_per_s": tests_per_s,
        "filter_decided_frac": float(st["filter_decided"] / max(1, st["candidates"])),
        "escalated": int(st["escalated"]), "exact_signs": int(st["exact_signs"]),
        "levels": int(st["levels"]), "node_pairs": int(st["node_pairs"]),
        "stage_ms": {"traverse_filter": trav, "exact": float(np.mean([s["ms_exact"] for s in stats])),
                     "segments": float(np.mean([s["ms_segments"] for s in stats])),
                     "ordering": float(np.mean([s["ms_sort"] for s in stats]))},
        "pose_update": {"p50_ms": float(np.percentile(wall_ms, 50)), "p99_ms": float(np.percentile(wall_ms, 99)),
                        "what": "gi_intersect wall clock, resident meshes, results on host"},
        "fp64_form": {"value": float(np.mean(fp64_ms)), "unit": "ms",
                      "speedup_fp32_cascade": float(np.mean(fp64_ms) / max(1e-9, np.mean(dev_ms)))},
        "e2e": {"value": float(np.mean(e2e_ms)), "unit": "ms", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "what": "gi_intersect_oneshot from host arrays (upload + BVH build + intersect + results)"},
        "gpu_launches": int(np.sum([s["launches"] for s in stats])),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "kernel": "k_traverse", "peak_source": peak_src,
                     "alg_bytes_per_launch": float(alg_bytes),
                     "note": "output-sensitive traversal: bytes = node pairs x 2 nodes x 128 B + leaf pairs x "
                             "2 x (16 B record + 3 x 24 B vertices) + results x 16 B"},
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ncores = os.cpu_count() or 1
        ms, ref = cpu_oracle_run(cfg, poses[args.warmup:args.warmup + 3], ncores)
        line["cpu_baseline"] = {"value": float(np.mean(ms)), "unit": "ms", "cores": ncores, "kind": "port",
                                "sample": "3 full intersects of the same workload (same poses) with the exact "
                                          "C oracle; CPU %s" % cpu_model()}
        R, C, T = poses[args.warmup + 2]
        rchk = one((R, C, T))
        line["cpu_baseline"]["pairs_identical"] = bool(np.array_equal(rchk.pairs, ref["pairs"]))
    if rank == 0:
        print(json.dumps(line), flush=True)
    A.release()
    B.release()
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
