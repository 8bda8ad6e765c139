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
  e2e        the one-shot C-ABI call with HOST arrays in pinned memory
             (gi_intersect_oneshot = runGridForestIntersectionPipeline):
             H2D of both meshes, BVH builds, intersect, D2H of pairs+segments;
             e2e.split.pageable_inputs_ms_p50 is the same call from ordinary
             (pageable) arrays.
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
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one traversal
# launch on the level-8 pose workload with L2 flushed, from the ncu captures
# summarised in profiles/k_traverse_config2.md, per traversal shape captured
# (shape 7 with a quarter of the blocks filtering candidates)
TRAVERSE_DRAM_BYTES = {0: 11.373824e6 + 512.0, 7: 13.270784e6 + 256.0}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--level", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--workload", default="pose", choices=["pose", "batch", "serving", "ingest", "classify"],
                    help="pose: the headline pose-update stream on two 1.3M-triangle meshes; batch: many "
                         "mesh pairs of uneven size in one call; serving: resident pairs under an HBM "
                         "budget with a Poisson pose stream")
    ap.add_argument("--pairs", type=int, default=0, help="batch: 4096 pairs; serving: 64 pairs (default)")
    ap.add_argument("--classify-config", type=int, default=2, choices=[2, 3],
                    help="classify: the displaced icospheres (2) or the coplanar integer grids (3), whose "
                         "candidate pairs escalate to the exact stage")
    ap.add_argument("--rate", type=float, default=2000.0, help="serving: mean requests per second")
    ap.add_argument("--duration", type=float, default=3.0, help="serving: seconds of offered load")
    ap.add_argument("--pose-samples", type=int, default=1000,
                    help="pose-update latency: wall-clock samples of gi_intersect after the timed steps")
    ap.add_argument("--shape", type=int, default=-1,
                    help="pin the traversal shape (0..7) instead of autotuning it (for profiling runs)")
    return ap.parse_args()


def workload(level):
    from gpuintersector import meshgen as mg

    cfg = mg.config2(level=level)
    rng = np.random.default_rng(22)
    return cfg, rng


def pose_config(level, cfg):
    """The workload's identity, the same in both arms (ours and --impl reference)."""
    return {"workload": "icosphere L%d displaced x2 (%d tris each), pose-update stream" % (level, int(cfg["tA"].shape[0])),
            "tris_per_mesh": int(cfg["tA"].shape[0]), "pose_stream": "seeded 22, <= 5 deg and <= 0.05 r per step",
            "segments": True}


def step_poses(cfg, rng, n):
    """Base pose of B composed with a stream of small rigid updates."""
    from gpuintersector import meshgen as mg

    R0, C0, T0 = cfg["poseB"]
    out = []
    for dR, dt in mg.pose_stream(rng, n, 5.0, 0.05):
        out.append((dR @ R0, C0, T0 + dt))
    return out


class Clocks:
    """SM clock, power and clock-event reasons sampled through NVML every 2 ms
    while the timed region runs (nvidia-smi's fastest period, 200 ms, is longer
    than a short timed region).  Reading counters only; no setting is changed."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, cuda_index):
        self.index = cuda_index
        self.rows = []
        self.max_mhz = None
        self.stop = threading.Event()
        self.nv = None

    def _handle(self):
        import pynvml as nv
        import torch

        nv.nvmlInit()
        self.nv = nv
        try:
            pr = torch.cuda.get_device_properties(self.index)
            bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.index)

    def __enter__(self):
        try:
            self.h = self._handle()
            self.max_mhz = float(self.nv.nvmlDeviceGetMaxClockInfo(self.h, self.nv.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        except Exception as e:  # no NVML: report unsampled
            self.err = repr(e)
            self.h = None
        return self

    def _run(self):
        nv = self.nv
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                pw = nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0
                self.rows.append((float(sm), int(rs), pw))
            except Exception:
                pass
            self.stop.wait(0.002)

    def __exit__(self, *a):
        self.stop.set()
        if self.h is not None:
            self.t.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        reasons = set()
        for _, rs, _ in self.rows:
            for name, const in self.REASONS:
                if rs & getattr(self.nv, const, 0):
                    reasons.add(name)
        return {"sm_mhz": float(np.median([r[0] for r in self.rows])), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(self.rows), "source": "nvml, 2 ms period",
                "power_w_max": float(max(r[2] for r in self.rows))}


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
        "config": pose_config(args.level, cfg), "parallelism": "cpu threads",
        "cpu_baseline": {"value": v, "unit": "ms", "cores": ncores, "kind": "port",
                         "sample": "full intersect (BVH over B + exact predicates + segments) per step, "
                                   "%d steps; CPU %s" % (args.steps, cpu_model())},
        "e2e": {"value": v, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "pairs": int(len(last["pairs"])),
        "note": "the reference's CPU/CGAL path cannot be built here (CGAL, Boost, TBB, cuBQL absent); "
                "this arm times the exact C oracle restating its semantics",
    }
    print(json.dumps(line), flush=True)


def _json(line):
    print(json.dumps(line), flush=True)


def run_batch(args, gi, world, rank, dist):
    """Config 4: batched mesh pairs of uneven size (displaced geodesic spheres,
    T log-uniform in [1k, 200k] per mesh) in one call per step.  With N ranks the
    pairs are shared out by estimated cost (no collective on the data path)."""
    import torch
    from gpuintersector import meshgen as mg
    from gpuintersector import shard

    npairs = args.pairs or 4096
    ctx = gi.Context(int(os.environ.get("LOCAL_RANK", "0")))
    costs = [shard.job_cost(a, b) for a, b in mg.config4_sizes(seed=4, pairs=npairs)]
    mine = shard.assign(costs, world)[rank]
    jobs, meshes, tris = [], [], 0
    t_up = time.perf_counter()
    for j in mg.config4_iter(seed=4, pairs=npairs, which=mine):
        A, B = ctx.upload(j["vA"], j["tA"]), ctx.upload(j["vB"], j["tB"])
        meshes += [A, B]
        tris += j["tA"].shape[0] + j["tB"].shape[0]
        R, C, T = j["poseB"]
        jobs.append((A, None, B, gi.pose_raw(R, C, T)))
    upload_s = time.perf_counter() - t_up
    for k in range(2 * gi._abi.GI_TRAVERSE_SHAPES + args.warmup):  # autotuning, then warm-up (untimed)
        rs = ctx.intersect_batch(jobs, want_segments=True)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    dev, wall, st = [], [], None
    if dist:
        dist.barrier()
    with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for k in range(args.steps):
            flush.fill_(k & 255)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fr = ctx.intersect_batch_flat(jobs, want_segments=True)  # whole-batch arrays on the host
            wall.append((time.perf_counter() - t0) * 1e3)
            dev.append(fr.stats["ms_total"])
    st = fr.stats
    found = int(len(fr.pairs))
    # every job's curves from the whole-batch arrays, in one call on host threads
    t0 = time.perf_counter()
    ncurves = int(len(fr.curves()["closed"]))
    curves_ms = (time.perf_counter() - t0) * 1e3
    total = float(np.sum(dev))
    if dist:
        t = torch.tensor([total], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total = float(t.item())
    ms = total / args.steps
    line = {
        "metric": "ms per batch of %d mesh pairs (config 4) and mesh pairs/s" % npairs, "value": ms, "unit": "ms",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded displaced geodesic spheres, T log-uniform in [1k, 200k] per mesh)",
        "config": {"workload": "batch of %d mesh pairs" % npairs, "pairs_this_rank": len(jobs),
                   "tris_this_rank": tris, "l2": "flushed (256 MB write) before each step",
                   "parallelism": "pairs sharded by cost" if world > 1 else "single",
                   "traverse_shape": int(st["traverse_shape"]), "autotuned": True},
        "mesh_pairs_per_s": npairs / (ms * 1e-3), "intersecting_pairs": found,
        "node_pairs": int(st["node_pairs"]), "candidates": int(st["candidates"]),
        "tri_pair_tests_per_s": float(st["candidates"]) / (float(np.mean([st["ms_traverse"]])) * 1e-3),
        "stage_ms": {"traverse_filter": st["ms_traverse"], "exact": st["ms_exact"], "segments": st["ms_segments"],
                     "ordering": st["ms_sort"]},
        "wall_ms_p50": float(np.percentile(wall, 50)),  # intersect_batch_flat: results as whole-batch host arrays
        "generate_upload_build_s": upload_s,  # numpy generation of the meshes included
        "clocks": clk.summary(),
        "curve_assembly": {"ms": curves_ms, "curves": ncurves,
                           "what": "gi_curves_build_jobs over the whole batch, host threads"},
    }
    if rank == 0:
        _json(line)
    for m in meshes:
        m.release()
    ctx.close()


def run_serving(args, gi, world, rank, dist):
    """Config 5: resident mesh pairs (displaced geodesic spheres, T log-uniform in
    [10k, 2M]) under an HBM admission budget of about three quarters of their
    total size, served with a Poisson stream of small pose updates."""
    from gpuintersector import meshgen as mg
    from gpuintersector.serving import ResidentSet, poisson_serving

    npairs = args.pairs or 64
    sets = mg.config5(seed=5, pairs=npairs)
    pairs = [(d["vA"], d["tA"], d["vB"], d["tB"]) for d in sets]
    poses = [d["poseB"] for d in sets]
    tris = sum(d["tA"].shape[0] + d["tB"].shape[0] for d in sets)
    with gi.Context(int(os.environ.get("LOCAL_RANK", "0"))) as probe:
        m = probe.upload(sets[0]["vA"], sets[0]["tA"])
        per_tri = m.info()["bytes"] / sets[0]["tA"].shape[0]
        m.release()
    need = int(per_tri * tris)
    budget = int(0.75 * need)
    ctx = gi.Context(int(os.environ.get("LOCAL_RANK", "0")), hbm_budget_bytes=budget)
    # admission: pairs are admitted in order while the budget accepts their
    # uploads; requests go to admitted pairs only (a rejected pair is refused up
    # front instead of evicting resident ones on every request)
    admitted = []
    for k in range(npairs):
        try:
            A = ctx.upload(pairs[k][0], pairs[k][1])
        except gi.GIError:
            continue
        try:
            B = ctx.upload(pairs[k][2], pairs[k][3])
        except gi.GIError:
            A.release()
            continue
        admitted.append((k, A, B))
    sel = [k for k, _, _ in admitted]
    rs = ResidentSet(ctx, [pairs[k] for k in sel])
    for i, (k, A, B) in enumerate(admitted):
        rs.res[i] = (A, B)
    rs.admissions = len(admitted)
    sel_poses = [poses[k] for k in sel]
    warm = poisson_serving(ctx, rs, sel_poses, rate=args.rate, duration=0.5, seed=1)
    with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        out = poisson_serving(ctx, rs, sel_poses, rate=args.rate, duration=args.duration, seed=2)
    out["admitted_pairs"] = len(sel)
    out["rejected_pairs"] = npairs - len(sel)
    out["tris_admitted"] = int(sum(pairs[k][1].shape[0] + pairs[k][3].shape[0] for k in sel))
    line = {
        "metric": "pose-update latency p50/p99 under a Poisson stream (config 5) and pairs/s", "value": out["p50_ms"],
        "unit": "ms", "n_gpus": world, "steps": out["requests"], "warmup": warm["requests"],
        "ms_per_step": out["p50_ms"], "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded displaced geodesic spheres, T log-uniform in [10k, 2M])",
        "config": {"workload": "serving %d resident pairs, Poisson %.0f req/s for %.1f s" % (npairs, args.rate,
                                                                                              args.duration),
                   "tris_total": tris, "mesh_bytes_total": need, "hbm_budget_bytes": budget},
        "serving": out, "clocks": clk.summary(),
    }
    rs.close()
    ctx.close()
    if rank == 0:
        _json(line)


def run_ingest(args, gi, world, rank):
    """Ingestion upstream of the path: two config-2 meshes (1,310,720 triangles
    each) written as OFF text, then gi_off_load (host threads, mmap) and
    gi_scene_load (both files parsed, copied, normalised on the device, both
    BVHs built)."""
    import tempfile

    from gpuintersector import meshgen as mg

    cfg = mg.config2(level=args.level)
    tmp = tempfile.mkdtemp(prefix="gi_ingest_")
    paths = []
    for tag in ("A", "B"):
        v, t = cfg["v" + tag], cfg["t" + tag]
        path = os.path.join(tmp, tag + ".off")
        with open(path, "w") as f:
            f.write("OFF\n%d %d 0\n" % (v.shape[0], t.shape[0]))
            np.savetxt(f, v, fmt="%.17g")
            np.savetxt(f, np.column_stack([np.full(t.shape[0], 3), t]), fmt="%d")
        paths.append(path)
    nbytes = sum(os.path.getsize(p) for p in paths)
    load_ms, scene_ms = [], []
    ncores = os.cpu_count() or 1
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        for p in paths:
            gi.load_off(p)
        t1 = time.perf_counter()
        with gi.Context(int(os.environ.get("LOCAL_RANK", "0"))) as ctx:
            t2 = time.perf_counter()
            A, B, sc, ra, rb = ctx.load_scene(paths[0], paths[1], scale_to_unit=True)
            t3 = time.perf_counter()
            A.release()
            B.release()
        if k >= args.warmup:
            load_ms.append((t1 - t0) * 1e3)
            scene_ms.append((t3 - t2) * 1e3)
    tris = int(cfg["tA"].shape[0] + cfg["tB"].shape[0])
    line = {
        "metric": "OFF ingestion: ms to load both config-2 files; ms to load + normalise + build both meshes",
        "value": float(np.median(scene_ms)), "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": float(np.median(scene_ms)), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (config-2 icospheres written as OFF text, %.1f MB)" % (nbytes / 1e6),
        "config": {"workload": "2 OFF files, %d triangles" % tris, "host_threads": ncores},
        "off_load_ms": float(np.median(load_ms)), "off_parse_MB_per_s": nbytes / 1e6 / (np.median(load_ms) * 1e-3),
        "scene_load_ms": float(np.median(scene_ms)), "scene_tris_per_s": tris / (np.median(scene_ms) * 1e-3),
    }
    for p in paths:
        os.remove(p)
    os.rmdir(tmp)
    if rank == 0:
        _json(line)


def run_classify(args, gi, world, rank):
    """The pair-list predicate entry point (gi_classify_pairs, the reference's
    classifyPair chain FP32 -> FP64 -> exact on a candidate list): config 2's
    meshes at the base pose, a list of its intersecting pairs with index
    neighbours of B (about 1 M pairs, most not intersecting), in both precision
    forms; the exact C oracle over the same list on all host threads as the CPU
    baseline."""
    import torch

    from gpuintersector import meshgen as mg

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    cfg = mg.config2(level=args.level) if args.classify_config == 2 else mg.config3()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    ctx = gi.Context(local)
    A, B = ctx.upload(cfg["vA"], cfg["tA"]), ctx.upload(cfg["vB"], cfg["tB"])
    if cfg["poseB"] is not None:
        R, C, T = cfg["poseB"]
        pose = gi.pose_raw(R, C, T)
    else:
        R, C, T = np.eye(3), np.zeros(3), np.zeros(3)
        pose = None
    hits = ctx.intersect(A, B, None, pose, want_segments=False).pairs
    if args.classify_config == 3:  # 1.33 M intersecting pairs: a sample of them keeps the list near 1 M
        hits = hits[np.random.default_rng(3).choice(len(hits), 11000, replace=False)]
    nt = int(cfg["tB"].shape[0])
    d = np.arange(-48, 48)
    pairs = np.stack([np.repeat(hits[:, 0], d.size), (np.repeat(hits[:, 1], d.size) + np.tile(d, len(hits))) % nt], 1)
    pairs = np.ascontiguousarray(pairs.astype(np.int32))
    n = pairs.shape[0]
    d_pairs = torch.from_numpy(pairs).cuda()
    d_out = torch.empty(n, dtype=torch.uint8, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    res = {}
    for prec, name in ((0, "fp32_cascade"), (1, "fp64")):
        for k in range(args.warmup):
            ctx.classify_pairs(A, B, None, pose, d_pairs.data_ptr(), n, d_out.data_ptr(), precision=prec)
        ms = []
        for k in range(args.steps):
            flush.fill_(k & 255)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ctx.classify_pairs(A, B, None, pose, d_pairs.data_ptr(), n, d_out.data_ptr(), precision=prec)
            ms.append((time.perf_counter() - t0) * 1e3)
        res[name] = float(np.median(ms))
    out = d_out.cpu().numpy()
    # CPU baseline: the exact oracle over the same list on all host threads
    import oracle as oc

    pA, pB = oc.pose_identity(), (oc.pose_raw(R, C, T) if pose is not None else oc.pose_identity())
    reps, t0 = 0, time.perf_counter()
    while True:
        exp = oc.classify_pairs(cfg["vA"], cfg["tA"], pA, cfg["vB"], cfg["tB"], pB, pairs)
        reps += 1
        if time.perf_counter() - t0 > 2.0 or reps >= 50:
            break
    cpu_s = (time.perf_counter() - t0) / reps
    same = bool(np.array_equal(exp, out))
    per_pair = 8 + 2 * (12 + 3 * 24) + 1
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = per_pair * n / (res["fp32_cascade"] * 1e-3) / 1e9
    line = {
        "metric": "candidate pairs classified per second (gi_classify_pairs, FP32 cascade)",
        "value": n / (res["fp32_cascade"] * 1e-3), "unit": "pairs/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": res["fp32_cascade"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (%s; intersecting pairs and their B-index neighbours)" % (
            "config-2 icospheres" if args.classify_config == 2 else "config-3 coplanar integer grids"),
        "config": {"workload": "%d candidate pairs, 2 x %d triangles" % (n, nt), "intersecting": int(out.sum()),
                   "l2": "flushed (256 MB write) before each step", "timing": "host wall of the blocking call"},
        "fp64_form_ms": res["fp64"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "alg_bytes_per_pair": per_pair,
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        "cpu_baseline": {"value": n / cpu_s, "unit": "pairs/s", "cores": os.cpu_count() or 1, "kind": "port",
                         "sample": "the whole list, %d runs, exact C oracle on all host threads (vertices posed "
                                   "once per run); CPU %s" % (reps, cpu_model()),
                         "outputs_identical": same},
    }
    A.release()
    B.release()
    if rank == 0:
        _json(line)


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

    if args.workload == "batch":
        run_batch(args, gi, world, rank, dist)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.workload == "ingest":
        run_ingest(args, gi, world, rank)
        return
    if args.workload == "classify":
        run_classify(args, gi, world, rank)
        return
    if args.workload == "serving":
        run_serving(args, gi, world, rank, dist)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    cfg, rng = workload(args.level)
    # the pose-update samples take the poses after the timed steps' (the stream
    # is drawn pose by pose, so the first warmup + steps poses do not depend on it)
    poses = step_poses(cfg, rng, args.warmup + args.steps + args.pose_samples)
    flags = 0 if args.shape < 0 else (gi._abi.GI_FLAG_FIXED_SHAPE | gi._abi.GI_FLAG_SHAPE(args.shape))
    ctx = gi.Context(local, flags=flags)
    A = ctx.upload(cfg["vA"], cfg["tA"])
    B = ctx.upload(cfg["vB"], cfg["tB"])
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def one(pose, precision=0):
        R, C, T = pose
        return ctx.intersect(A, B, None, gi.pose_raw(R, C, T), want_segments=True, precision=precision)

    # autotuning: the library times each traversal shape (expansion form x
    # blocks per SM) twice per workload class on its own calls, then keeps the
    # fastest; these calls precede the warm-up and are not timed
    for k in range(2 * gi._abi.GI_TRAVERSE_SHAPES if args.shape < 0 else 0):
        one(poses[0])
        one(poses[0], precision=1)
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
            r.pairs  # the result's arrays are made usable inside the timing
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

    # pose-update latency (the serving loop's steady state): resident meshes, a
    # new pose in, the pairs and segments usable on the host; no L2 flush.
    # Collections of Python's garbage collector are logged with their times, so
    # that a slow sample can be put down to the host or to the device.
    import gc

    gc_log = []

    def _gc_cb(phase, info):
        gc_log.append((phase, info.get("generation", -1), time.perf_counter()))

    pu_wall, pu_dev, pu_span = [], [], []
    gc.callbacks.append(_gc_cb)
    try:
        base = args.warmup + args.steps
        for k in range(args.pose_samples):
            t0 = time.perf_counter()
            rr = one(poses[base + k])
            rr.pairs
            t1 = time.perf_counter()
            pu_wall.append((t1 - t0) * 1e3)
            pu_dev.append(rr.stats["ms_total"])
            pu_span.append((t0, t1))
        del rr
    finally:
        gc.callbacks.remove(_gc_cb)
    pose_update = {"what": "gi_intersect wall clock, resident meshes, a new pose per call, results on the host",
                   "samples": len(pu_wall)}
    if pu_wall:
        w = np.array(pu_wall)
        slow = np.nonzero(w > 1.0)[0]
        gc_starts = [t for ph, g, t in gc_log if ph == "start"]
        slow_gc = sum(1 for i in slow if any(pu_span[i][0] <= t <= pu_span[i][1] for t in gc_starts))
        pose_update.update({
            "p50_ms": float(np.percentile(w, 50)), "p99_ms": float(np.percentile(w, 99)),
            "p999_ms": float(np.percentile(w, 99.9)), "max_ms": float(w.max()),
            "device_p50_ms": float(np.percentile(pu_dev, 50)), "device_max_ms": float(np.max(pu_dev)),
            "over_1ms": int(slow.size), "over_1ms_with_gc": int(slow_gc),
            "over_1ms_device_over_1ms": int(sum(1 for i in slow if pu_dev[i] > 1.0)),
            "gc_collections": len(gc_starts)})

    # e2e: one-shot from host arrays in pinned memory (the inputs' H2D, both
    # builds, the intersect and the D2H of its results are inside the timing)
    def pinned(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        t = torch.empty(a.shape, dtype={np.float64: torch.float64, np.uint32: torch.int32}[dt], pin_memory=True)
        t.numpy().view(dt)[...] = a
        return t, t.numpy().view(dt)

    hold = [pinned(cfg["vA"], np.float64), pinned(cfg["tA"], np.uint32), pinned(cfg["vB"], np.float64),
            pinned(cfg["tB"], np.uint32)]
    hvA, htA, hvB, htB = (h[1] for h in hold)
    e2e_ms = []
    last_e2e = None
    for k in range(3 + args.e2e_steps):
        R, C, T = poses[args.warmup + (k % args.steps)]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        last_e2e = ctx.intersect_oneshot(hvA, htA, hvB, htB, None, gi.pose_raw(R, C, T))
        if k >= 3:  # three untimed warm-up calls first
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
    # the same call from pageable (ordinary numpy) arrays, for comparison
    pageable_ms = []
    for k in range(3):
        R, C, T = poses[args.warmup + k]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.intersect_oneshot(cfg["vA"], cfg["tA"], cfg["vB"], cfg["tB"], None, gi.pose_raw(R, C, T))
        pageable_ms.append((time.perf_counter() - t0) * 1e3)
    # where the end-to-end time goes (one extra instrumented call, not in the mean)
    R, C, T = poses[args.warmup]
    t0 = time.perf_counter()
    eA = ctx.upload(cfg["vA"], cfg["tA"])
    t1 = time.perf_counter()
    eB = ctx.upload(cfg["vB"], cfg["tB"])
    t2 = time.perf_counter()
    er = ctx.intersect(eA, eB, None, gi.pose_raw(R, C, T), want_segments=True)
    t3 = time.perf_counter()
    eA.release()
    eB.release()
    t4 = time.perf_counter()
    e2e_split = {"pageable_inputs_ms_p50": float(np.median(pageable_ms)),
                 "upload_build_a_ms": (t1 - t0) * 1e3, "upload_build_b_ms": (t2 - t1) * 1e3,
                 "intersect_ms": (t3 - t2) * 1e3, "release_ms": (t4 - t3) * 1e3,
                 "intersect_device_ms": er.stats["ms_total"]}
    h2d = int(cfg["vA"].nbytes + cfg["tA"].astype(np.uint32).nbytes + cfg["vB"].nbytes +
              cfg["tB"].astype(np.uint32).nbytes)
    d2h = int(last_e2e.pairs.nbytes + last_e2e.segments.nbytes + last_e2e.seg_pair.nbytes)

    st = stats[-1]
    # BVH build roofline: the algorithmic bytes of one build of a T-triangle,
    # V-vertex mesh (read the mesh 24V + 12T, a 32-bit key sort 64T, write 2T-1
    # nodes of 32 B and T ids, read the nodes once to refit) over the device time
    # of the build kernels (gi_mesh_build_ms), averaged over the builds above
    T, V = int(cfg["tA"].shape[0]), int(cfg["vA"].shape[0])
    build_bytes = 24 * V + 12 * T + 64 * T + 32 * (2 * T - 1) + 4 * T + 32 * (2 * T - 1)
    # warm builds only (the first launches of a process also load the kernels)
    build_ms = []
    for k in range(5):
        wm = ctx.upload(hvA, htA)
        build_ms.append(wm.info()["build_ms"])
        wm.release()
    build_ms = build_ms[1:]
    # curve assembly (downstream of the path) on the last step's result
    t0 = time.perf_counter()
    cv_verts, cv = r.curves()
    curves_ms = (time.perf_counter() - t0) * 1e3
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
        "config": pose_config(args.level, cfg),
        "parallelism": "replicas" if world > 1 else "single",
        "impl_config": {"l2": "flushed (256 MB write) before each step", "precision": "fp32 filter -> fp64 filter -> exact",
                        "traverse_shape": int(st["traverse_shape"]), "autotuned": args.shape < 0},
        "pairs": int(st["pairs"]), "segments": int(st["segments"]), "candidates": int(cand),
        "tri_pair_tests_per_s": tests_per_s,
        "filter_decided_frac": float(st["filter_decided"] / max(1, st["candidates"])),
        "escalated": int(st["escalated"]), "exact_signs": int(st["exact_signs"]),
        "levels": int(st["levels"]), "node_pairs": int(st["node_pairs"]),
        "level_end_ms": [round(x, 4) for x in st.get("level_end_ms", [])],
        "stage_ms": {"traverse_filter": trav, "exact": float(np.mean([s["ms_exact"] for s in stats])),
                     "segments": float(np.mean([s["ms_segments"] for s in stats])),
                     "ordering": float(np.mean([s["ms_sort"] for s in stats]))},
        "pose_update": pose_update,
        "curve_assembly": {"ms": curves_ms, "curves": len(cv), "closed": int(sum(1 for _, c in cv if c)),
                           "vertices": int(cv_verts.shape[0]), "what": "gi_curves_build on the host, last step"},
        "fp64_form": {"value": float(np.mean(fp64_ms)), "unit": "ms",
                      "speedup_fp32_cascade": float(np.mean(fp64_ms) / max(1e-9, np.mean(dev_ms)))},
        "e2e": {"value": float(np.mean(e2e_ms)), "unit": "ms", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "what": "gi_intersect_oneshot from pinned host arrays (H2D of both meshes + both BVH builds on two "
                        "streams + intersect + D2H of pairs and segments)",
                "samples_ms": [round(x, 3) for x in e2e_ms], "split": e2e_split},
        "gpu_launches": int(np.sum([s["launches"] for s in stats])),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": TRAVERSE_DRAM_BYTES.get(int(st["traverse_shape"])) if args.level == 8 else None,
                     "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of the "
                                       "traversal on this workload with the same shape (null: shape not captured); "
                                       "profiles/k_traverse_config2.md",
                     "kernel": "k_traverse", "peak_source": peak_src,
                     "alg_bytes_per_launch": float(alg_bytes),
                     "note": "output-sensitive traversal: bytes = node pairs x 2 nodes x 128 B + leaf pairs x "
                             "2 x (16 B record + 3 x 24 B vertices) + results x 16 B"},
        "build_roofline": {"bound": "hbm", "achieved": build_bytes / (np.mean(build_ms) * 1e-3) / 1e9, "peak": peak,
                           "unit": "GB/s", "frac": build_bytes / (np.mean(build_ms) * 1e-3) / 1e9 / peak,
                           "build_ms": float(np.mean(build_ms)), "builds": len(build_ms),
                           "what": "mean of 4 warm builds of mesh A from pinned host arrays (gi_mesh_build_ms: "
                                   "CUDA events around validation + build, the mid-build host round trip included)",
                           "alg_bytes_per_mesh": build_bytes, "peak_source": peak_src,
                           "note": "24V + 12T (mesh) + 64T (32-bit key sort) + 32(2T-1) + 4T (nodes, ids) + "
                                   "32(2T-1) (refit read) over the device time of validation + build kernels"},
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
