"""DD3 projector / backprojector throughput on B200.

One step = one branchless DD forward projection and one backprojection of
the 512x512x256 volume over 984 views onto the 888x64 detector (the
single-volume throughput workload): volume SATs + projection kernel,
projection SATs + backprojection kernel.  value = voxel-views processed by
both operators (2 * XN*YN*ZN*PN per step) per second, whole job, inputs
resident in HBM.  e2e = the same metric through the reference-facing host
entry points DD3Proj_gpu / DD3Back_gpu with pinned host buffers, copies
included.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun), the ranks share one scan (--split scan, the default):
projection split by views, backprojection by z slabs, NCCL all-gathers of the
view blocks and slabs (strong scaling); --split volumes gives every rank its
own independent volume instead (weak scaling, no data-path collective).
Timing is the max over ranks.  --impl reference times the CPU restatement of
the reference's DD path (the oracle) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DD3 proj+backproj throughput (Gvoxel-views/s)"
UNIT = "Gvoxel-views/s"
WORKLOAD = "dd3_proj_back_512x512x256_984v_888x64"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--sat", default="zprefix", choices=["fp64", "f32pair", "zprefix"])
    ap.add_argument("--cpu-views", type=int, default=4, help="views in the bounded CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="dd3", choices=["dd3", "recon", "learned", "batch", "helical"],
                    help="dd3: the projector/backprojector throughput line (default); recon: OS-SART 24x30 and "
                         "FISTA-TV 50 at 256x256x128 / 720 views with residual and RMSE per iteration; learned: "
                         "train the warm-start CNN on OS-SART 2- vs 30-iteration pairs, then time-to-residual "
                         "learned vs plain; batch: 48 uneven scans, one persistent launch vs per-scan launches; "
                         "helical: projection and backprojection of a 512x512x1024 helical scan")
    ap.add_argument("--train-volumes", type=int, default=16, help="learned workload: training phantoms")
    ap.add_argument("--train-steps", type=int, default=3000, help="learned workload: Adam steps")
    ap.add_argument("--held-out", type=int, default=8, help="learned workload: held-out phantoms evaluated")
    ap.add_argument("--cases", type=int, default=48,
                    help="batch workload: keep the first N of the 48 cases (a profiling case)")
    ap.add_argument("--recon-iters", type=int, default=0,
                    help="recon workload: iterations of each solver (0 = 30 OS-SART, 50 FISTA-TV); a smaller count "
                         "is a profiling case")
    ap.add_argument("--split", default="auto", choices=["auto", "scan", "volumes"],
                    help="'scan' splits one scan over the ranks (projection by views, backprojection by z slabs, "
                         "NCCL all-gathers of the view blocks and slabs; strong scaling); 'volumes' gives every "
                         "rank its own independent volume (weak scaling, no data-path collective); 'auto' = scan "
                         "for N > 1, the plain one-GPU path for N = 1")
    ap.add_argument("--views", type=int, default=0,
                    help="profiling case: keep only this many of the 984 views, in evenly spaced runs of 8 "
                         "adjacent views (0 = all)")
    return ap.parse_args()


def workload_geometry(args, G=None):
    if G is None:
        from ctlab_b200 import geometry as G
    g = G.config2()
    if args.views:
        runs = max(1, args.views // 8)
        starts = np.linspace(0, g.PN - 8, runs).round().astype(int)
        idx = np.unique(np.concatenate([s + np.arange(8) for s in starts]))[: args.views]
        g = g.with_views(idx)
    return g


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def config_dict(args, extra=None):
    d = {"workload": WORKLOAD if not args.views else f"{WORKLOAD}_subset{args.views}v",
         "volume": [512, 512, 256], "views": args.views or 984, "detector": [888, 64],
         "voxel_mm": [1.0, 1.0, 0.15625], "cell_mm": [1.0239, 1.0960], "sod_sdd_mm": [541, 949],
         "sat": args.sat, "l2": "inputs larger than L2 (volume 268 MB, SATs 1.08 GB)",
         "phantom": "random ellipsoids, 20-40, seed 1+rank"}
    if extra:
        d.update(extra)
    return d


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_sample(g, vol_h, prj_h, nviews):
    """Oracle (CPU restatement) proj + back over a bounded view sample."""
    import oracle
    idx = np.linspace(0, g.PN - 1, nviews).round().astype(int)
    gs = g.with_views(idx)
    threads = oracle.num_threads()
    t0 = time.perf_counter()
    oracle.dd3_proj(gs, vol_h)
    t1 = time.perf_counter()
    oracle.dd3_back(gs, prj_h[idx])
    t2 = time.perf_counter()
    vv = g.XN * g.YN * g.ZN * nviews
    return {"value": 2 * vv / (t2 - t0) / 1e9, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{nviews} evenly spaced views of the 984 (proj {t1 - t0:.1f} s + back {t2 - t1:.1f} s), "
                      "FP64 oracle with OpenMP, scaled per voxel-view"}


def geometry_records():
    """ctlab_b200/geometry.py loaded on its own (numpy only): the reference arm draws
    its scan without importing the package or loading the CUDA library."""
    import importlib.util
    name = "ctlab_scan_geometry"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "ctlab_b200", "geometry.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def run_reference(args):
    """The reference's CPU DD path, restated by the oracle (the reference's own CPU DD
    bodies are not published), on the host cores with all their threads.  Each timed step
    projects and backprojects the full 512x512x256 volume over a bounded sample of the
    984 views (evenly spaced); value = voxel-views processed / measured step time."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    import oracle
    G = geometry_records()
    g = workload_geometry(args, G)
    hx, hy, hz = G.half_extents(g)
    vol = oracle.ellipsoid_phantom(g, oracle.random_ellipsoids(1, hx, hy, hz))
    nviews = max(1, args.cpu_views)
    idx = np.linspace(0, g.PN - 1, nviews).round().astype(int)
    gs = g.with_views(idx)
    prj = oracle.dd3_proj(gs, vol).astype(np.float32)  # the sampled views' input to the backprojection
    threads = oracle.num_threads()
    # untimed warm-up: one short sample (thread pool start-up, page faults)
    if args.warmup > 0:
        g1 = g.with_views(idx[:1])
        oracle.dd3_proj(g1, vol)
        oracle.dd3_back(g1, prj[:1])
    times = []
    for _ in range(max(1, args.steps)):
        t0 = time.perf_counter()
        oracle.dd3_proj(gs, vol)
        oracle.dd3_back(gs, prj)
        times.append(time.perf_counter() - t0)
    t = float(np.median(times))
    vv2 = 2 * g.XN * g.YN * g.ZN * nviews
    v = vv2 / t / 1e9
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(args), "impl": "reference",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"each step: projection + backprojection of the full volume over {nviews} "
                                       f"evenly spaced views of {g.PN} (median of {len(times)} steps, "
                                       f"{t:.2f} s each); the full {g.PN}-view step would take "
                                       f"{t * g.PN / nviews:.0f} s at this rate (extrapolated, not run)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def kernel_counters(kernel, args):
    """Per-launch DRAM bytes and warp instructions of `kernel` at this workload from the
    committed ncu summary (profiles/kernel_counters.json), with the source hash the
    capture was made from and whether it still matches the kernel's source file."""
    path = os.path.join(ROOT, "profiles", "kernel_counters.json")
    if not os.path.exists(path) or args.views or args.sat != "zprefix":
        return None
    entry = json.load(open(path)).get(kernel)
    if not entry:
        return None
    import hashlib
    src = os.path.join(ROOT, "ctlab_b200", "csrc", entry["source"])
    cur = hashlib.sha256(open(src, "rb").read()).hexdigest()[:16] if os.path.exists(src) else None
    return dict(entry, source_matches=(cur == entry.get("source_sha16")))


def roofline_entry(dom, t_dom, alg, achieved, peak, peak_kind, clocks, args):
    """Three views of the dominant kernel against its limits:
    nominal_frac -- model bytes (8 B per voxel-view + 4 B per detector bin, a
        view-at-a-time stream of the FP64 SAT / accumulator) / time / HBM peak; this
        model is not a lower bound on traffic, so kernels that keep data on chip
        across views and slices exceed 1.0 here;
    dram_frac -- DRAM bytes one launch actually moves (ncu dram__bytes_read.sum +
        dram__bytes_write.sum, one full-size launch) / time / HBM peak;
    issue_frac -- warp instructions one launch executes (ncu smsp__inst_executed.sum)
        / (148 SMs x 4 schedulers x the median SM clock sampled during the timed region
        x time): the instruction-issue roofline of these gather kernels."""
    r = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
         "frac": achieved / peak, "nominal_frac": achieved / peak,
         "peak_source": ("measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback (6.65 TB/s, earlier measurement on this pool; no MEASURED_PEAKS.json)"),
         "algorithmic_bytes_per_launch": alg, "launch_ms": t_dom,
         "traffic": None, "dram_frac": None, "issue_frac": None}
    c = kernel_counters(dom, args)
    if c:
        t = t_dom * 1e-3
        r["traffic"] = c["dram_bytes_per_launch"]
        r["dram_achieved_gbs"] = c["dram_bytes_per_launch"] / t / 1e9
        r["dram_frac"] = r["dram_achieved_gbs"] / peak
        mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
        issue_peak = 148 * 4 * mhz * 1e6  # warp instructions per second
        r["warp_inst_per_launch"] = c["warp_inst_per_launch"]
        r["issue_frac"] = c["warp_inst_per_launch"] / t / issue_peak
        r["counters_source"] = (f"profiles/kernel_counters.json ({c['profile']}, captured {c['captured']}; "
                                f"kernel source {'unchanged' if c['source_matches'] else 'CHANGED'} since)")
        # what actually limits the kernel: HBM when it moves a good part of the
        # peak, otherwise instruction issue (and the latency issue-bound code waits on)
        r["limiter"] = "hbm" if r["dram_frac"] >= 0.5 else "instruction issue"
    return r


def run_split(args):
    """N ranks share ONE scan: rank r projects its block of the 984 views of the whole
    (replicated) volume and backprojects its z slab of the volume from the views that
    reach it; the view blocks and the slabs are all-gathered over NCCL, so every rank
    ends the step holding the whole projection and the whole backprojection.  value =
    the scan's voxel-views (2 * XN*YN*ZN*PN per step) / the max-over-ranks step time.
    e2e: the same step with the volume and the input projection uploaded from pinned
    host memory on every rank and both results read back, inside the timed region."""
    import datetime

    import torch
    import torch.distributed as dist

    import ctlab_b200 as cb
    from ctlab_b200 import geometry as G
    from ctlab_b200.multi import DistributedPlan

    ws, rank, local = dist_env()
    if "MASTER_ADDR" not in os.environ:  # a one-rank group outside torchrun
        import socket
        with socket.socket() as so:
            so.bind(("127.0.0.1", 0))
            os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(so.getsockname()[1]))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", init_method="env://", world_size=ws, rank=rank,
                            timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    g = workload_geometry(args)
    hx, hy, hz = G.half_extents(g)
    sat_mode = {"fp64": cb.CTLAB_SAT_FP64, "f32pair": cb.CTLAB_SAT_F32PAIR, "zprefix": cb.CTLAB_SAT_ZPREFIX}[args.sat]
    plans = []

    def make_plan(geom):
        plans.append(cb.Plan(geom, device=local, sat_mode=sat_mode))
        return plans[-1]

    dp = DistributedPlan(g, make_plan)
    vol = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
    cb.ellipsoid_phantom(vol, g, cb.random_ellipsoids(1, hx, hy, hz))  # the same scan on every rank
    prj_in = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
    dp.proj(vol, prj_in)
    prj = torch.zeros_like(prj_in)
    back = torch.zeros_like(vol)
    stream = torch.cuda.current_stream()

    def step():
        dp.proj(vol, prj)
        dp.back(prj_in, back)

    for _ in range(max(3, args.warmup)):
        step()
    step()
    launches_per_step = sum(p.last_launches() for p in plans)
    torch.cuda.synchronize()

    def timed(fn, steps):
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        t = torch.tensor([e0.elapsed_time(e1) / steps], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    with ClockSampler(local) as clk:
        ms_step = timed(step, args.steps)
    vv = g.voxel_views
    value = 2 * vv / (ms_step * 1e-3) / 1e9

    e2e = None
    if not args.no_e2e:
        hvol = torch.empty(g.vol_shape, dtype=torch.float32, pin_memory=True)
        hvol.copy_(vol.cpu())
        hprj_in = torch.empty(g.prj_shape, dtype=torch.float32, pin_memory=True)
        hprj_in.copy_(prj_in.cpu())
        hprj = torch.empty(g.prj_shape, dtype=torch.float32, pin_memory=True)
        hback = torch.empty(g.vol_shape, dtype=torch.float32, pin_memory=True)
        dvol, dprj_in = torch.empty_like(vol), torch.empty_like(prj_in)

        def e2e_step():
            dvol.copy_(hvol, non_blocking=True)
            dprj_in.copy_(hprj_in, non_blocking=True)
            dp.proj(dvol, prj)
            dp.back(dprj_in, back)
            hprj.copy_(prj, non_blocking=True)
            hback.copy_(back, non_blocking=True)

        for _ in range(2):
            e2e_step()
        es = timed(e2e_step, args.steps)
        nb = 4 * (g.XN * g.YN * g.ZN + g.PN * g.DNU * g.DNV) * ws
        e2e = {"value": 2 * vv / (es * 1e-3) / 1e9, "unit": UNIT, "h2d_bytes_per_step": nb,
               "d2h_bytes_per_step": nb, "ms_per_step": es,
               "path": "DistributedPlan.proj + .back (pinned host buffers on every rank)"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": max(3, args.warmup), "ms_per_step": ms_step, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None,
                "dtype": {"fp64": "f32 (f64 SAT)", "f32pair": "f32 (f32-pair SAT)",
                          "zprefix": "f32 (f64-accumulated z-prefix SAT)"}[args.sat],
                "data": "synthetic (seeded random-ellipsoid phantom)", "config": config_dict(args),
                "parallelism": f"one scan over {ws} ranks: views (projection) and z slabs (backprojection), "
                               "NCCL all-gather of view blocks and slabs",
                "clocks": clk.summary(), "e2e": e2e, "gpu_launches": launches_per_step * args.steps * ws,
                "roofline": None, "cpu_baseline": None}
        print(json.dumps(line), flush=True)
    dp.close()
    dist.barrier()
    dist.destroy_process_group()


def run_ours(args):
    import torch
    import torch.distributed as dist

    import ctlab_b200 as cb
    from ctlab_b200 import geometry as G

    ws, rank, local = dist_env()
    if args.split == "scan" or (ws > 1 and args.split == "auto"):
        return run_split(args)
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", init_method="env://", world_size=ws, rank=rank,
                                timeout=__import__("datetime").timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    g = workload_geometry(args)
    hx, hy, hz = G.half_extents(g)
    ell = cb.random_ellipsoids(1 + rank, hx, hy, hz)
    sat_mode = {"fp64": cb.CTLAB_SAT_FP64, "f32pair": cb.CTLAB_SAT_F32PAIR, "zprefix": cb.CTLAB_SAT_ZPREFIX}[args.sat]
    os.environ["CTLAB_LEGACY_SAT"] = str(sat_mode)  # the e2e arm's DD3Proj_gpu / DD3Back_gpu use the same SAT
    plan = cb.Plan(g, device=local, sat_mode=sat_mode)
    vol = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
    cb.ellipsoid_phantom(vol, g, ell)
    prj_in = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
    plan.proj(vol, prj_in)
    prj = torch.zeros_like(prj_in)
    back = torch.zeros_like(vol)
    stream = torch.cuda.current_stream()

    def step():
        plan.proj(vol, prj)
        plan.back(prj_in, back)

    def barrier():
        if ws > 1:
            dist.barrier()

    for _ in range(max(3, args.warmup)):
        step()
    launches_per_step = 0
    plan.proj(vol, prj)
    launches_per_step += plan.last_launches()
    plan.back(prj_in, back)
    launches_per_step += plan.last_launches()
    torch.cuda.synchronize()

    # timed region: K steps, barrier + synchronize on both sides
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    if ws > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    vv = g.voxel_views
    value = ws * 2 * vv / (ms_step * 1e-3) / 1e9

    # per-kernel times (CUDA events inside the plan, on the launching stream)
    plan.set_timing(True)
    proj_sat, proj_k, back_sat, back_k = [], [], [], []
    for _ in range(args.steps):
        plan.proj(vol, prj)
        a, b = plan.last_times()
        proj_sat.append(a)
        proj_k.append(b)
        plan.back(prj_in, back)
        a, b = plan.last_times()
        back_sat.append(a)
        back_k.append(b)
    plan.set_timing(False)
    t_proj, t_back = float(np.mean(proj_k)), float(np.mean(back_k))
    peak, peak_kind = peaks()
    alg = 8.0 * vv + 4.0 * g.PN * g.DNU * g.DNV  # bytes per launch (proj or back)
    zp = args.sat == "zprefix"
    if t_proj >= t_back:
        dom = "dd3_proj_t_kernel" if zp else "dd3_proj_kernel"
    else:
        dom = "dd3_back_t_kernel" if zp else "dd3_back_kernel"
    t_dom = max(t_proj, t_back)
    achieved = alg / (t_dom * 1e-3) / 1e9

    # e2e through the host entry points: pinned host buffers (the headline), and
    # pageable ones (numpy arrays, what thrust::host_vector callers pass) beside it
    e2e = None
    if not args.no_e2e:
        gargs = g.args()

        def e2e_time(hv, hp, hb):
            def e2e_step():
                cb.DD3Proj_gpu(**gargs, hvol=hv, hprj=hp, mask=None, gpunum=local, prjMode=0)
                cb.DD3Back_gpu(**gargs, hvol=hb, hprj=hp, mask=None, gpunum=local, squared=0, prjMode=0)

            for _ in range(max(2, args.warmup)):
                e2e_step()
            barrier()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                e2e_step()
            t1 = time.perf_counter()
            barrier()
            es = (t1 - t0) / args.steps
            if ws > 1:
                t = torch.tensor([es], device="cuda", dtype=torch.float64)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                es = float(t.item())
            return es

        hvol = torch.empty(g.vol_shape, dtype=torch.float32, pin_memory=True)
        hvol.copy_(vol.cpu())
        hprj = torch.empty(g.prj_shape, dtype=torch.float32, pin_memory=True)
        hback = torch.empty(g.vol_shape, dtype=torch.float32, pin_memory=True)
        es = e2e_time(hvol.numpy(), hprj.numpy(), hback.numpy())
        pv = hvol.numpy().copy()  # pageable copies, first-touched before timing
        pp, pb = np.zeros(g.prj_shape, np.float32), np.zeros(g.vol_shape, np.float32)
        es_pg = e2e_time(pv, pp, pb)
        del hvol, hprj, hback
        nvb, npb = 4 * vv // g.PN, 4 * g.PN * g.DNU * g.DNV
        e2e = {"value": ws * 2 * vv / es / 1e9, "unit": UNIT, "h2d_bytes_per_step": nvb + npb,
               "d2h_bytes_per_step": npb + nvb, "ms_per_step": es * 1e3,
               "path": "DD3Proj_gpu + DD3Back_gpu (host pointers, pinned)",
               "pageable": {"value": ws * 2 * vv / es_pg / 1e9, "ms_per_step": es_pg * 1e3,
                            "path": "DD3Proj_gpu + DD3Back_gpu (host pointers, pageable numpy arrays)"}}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(g, vol.cpu().numpy(), prj_in.cpu().numpy(), args.cpu_views)

    if rank == 0:
        clocks = clk.summary()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": {"fp64": "f32 (f64 SAT)", "f32pair": "f32 (f32-pair SAT)",
                                            "zprefix": "f32 (f64-accumulated z-prefix SAT)"}[args.sat],
            "data": "synthetic (seeded random-ellipsoid phantoms)",
            "config": config_dict(args),
            "parallelism": f"independent volume per GPU x{ws}",
            "clocks": clocks,
            "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps,
            "roofline": roofline_entry(dom, t_dom, alg, achieved, peak, peak_kind, clocks, args),
            "kernels_ms": {"proj_sat": float(np.mean(proj_sat)), "proj": t_proj,
                           "back_sat": float(np.mean(back_sat)), "back": t_back},
            "proj_gvvps": vv / (t_proj + float(np.mean(proj_sat))) / 1e6,
            "back_gvvps": vv / (t_back + float(np.mean(back_sat))) / 1e6,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    plan.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_recon(args):
    """OS-SART (24 subsets, 30 iterations, lambda 1) and FISTA-TV (lambda 1e-4, 50
    iterations) at 256x256x128 / 720 views / 384x128 detector from the projection of a
    seeded random-ellipsoid phantom with Poisson noise at I0 = 1e5 photons per ray:
    b = -ln(max(Poisson(I0 exp(-Ax)), 1) / I0).  Device times with CUDA events (the
    solves without per-iteration residuals, after one warm-up call that builds each
    solver's workspace and weights), then the residual ||Ax - b||/||b|| and the RMSE
    against the phantom after every iteration from a second, untimed pass."""
    import torch

    import ctlab_b200 as cb
    from ctlab_b200 import geometry as G

    ws, rank, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    g = G.config3()
    hx, hy, hz = G.half_extents(g)
    truth = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
    cb.ellipsoid_phantom(truth, g, cb.random_ellipsoids(11, hx, hy, hz))
    plan = cb.Plan(g, device=local)
    clean = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
    plan.proj(truth, clean)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    I0 = 1e5
    counts = torch.poisson(I0 * torch.exp(-clean), generator=gen)
    meas = -torch.log(torch.clamp(counts, min=1.0) / I0)
    stream = torch.cuda.current_stream()
    ev = lambda: torch.cuda.Event(enable_timing=True)

    def timed(fn):
        x = torch.zeros_like(truth)
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record(stream)
        fn(x, None)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), x

    def curve(fn, iters):
        x = torch.zeros_like(truth)
        res, rmse = [], []
        for _ in range(iters):
            r = fn(x, 1)
            res.append(float(r[0]))
            rmse.append(float(torch.sqrt(torch.mean((x - truth) ** 2))))
        return res, rmse

    n_os, n_fi = (args.recon_iters, args.recon_iters) if args.recon_iters else (30, 50)
    # one warm-up call of each solver builds its workspace and SART weights
    # on the plan (once per plan and mask); the timed calls reuse them
    plan.os_sart(torch.zeros_like(truth), meas, os_num=24, iter_num=1)
    plan.fista_tv(torch.zeros_like(truth), meas, iter_num=1, tv_lambda=1e-4)
    with ClockSampler(local) as clk:
        os_ms, _ = timed(lambda x, n: plan.os_sart(x, meas, os_num=24, iter_num=n_os))
        fi_ms, _ = timed(lambda x, n: plan.fista_tv(x, meas, iter_num=n_fi, tv_lambda=1e-4))
    # per-iteration curves: OS-SART restarts nothing between iterations, so one
    # iteration per call is the same solve; FISTA's momentum is not resumable, so
    # its residuals come from one call and its RMSE only at the end
    os_res, os_rmse = curve(lambda x, n: plan.os_sart(x, meas, os_num=24, iter_num=n, residuals=True), n_os)
    xf = torch.zeros_like(truth)
    fi_res = plan.fista_tv(xf, meas, iter_num=n_fi, tv_lambda=1e-4, residuals=True)
    fi_rmse = float(torch.sqrt(torch.mean((xf - truth) ** 2)))
    vv = g.voxel_views
    line = {"metric": "OS-SART / FISTA-TV time and convergence", "workload": "recon_256x256x128_720v_384x128",
            "n_gpus": 1, "data": "synthetic (seeded random-ellipsoid phantom, Poisson noise I0=1e5)",
            "os_sart": {"subsets": 24, "iterations": n_os, "lambda": 1.0, "ms_total": os_ms,
                        "ms_per_iteration": os_ms / n_os, "gvoxel_views_per_s": 2 * vv * n_os / (os_ms * 1e-3) / 1e9,
                        "residual": [round(v, 6) for v in os_res], "rmse": [round(v, 7) for v in os_rmse]},
            "fista_tv": {"iterations": n_fi, "tv_lambda": 1e-4, "ms_total": fi_ms, "ms_per_iteration": fi_ms / n_fi,
                         "residual": [round(float(v), 6) for v in fi_res], "rmse_final": fi_rmse},
            "phantom_rms": float(torch.sqrt(torch.mean(truth ** 2))), "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    plan.close()


def run_learned(args):
    """Learned warm start at 256x256x128 / 720 views / 384x128 detector, Poisson
    noise I0 = 1e5.  Training pairs: for each seeded random-ellipsoid phantom, the
    2-iteration and the 30-iteration OS-SART images (24 subsets) of its noisy
    projections; 128 slice pairs per phantom.  The CNN trains with the library's own
    kernels.  On each of --held-out phantoms (seeds 7, 8, ...): plain = 30 OS-SART
    iterations from zero (residual R30, device time T30); learned = 2 iterations + the
    CNN + the fewest further iterations whose residual reaches R30; the line reports
    every phantom and the median and worst time ratio.  Times are CUDA-event device
    times of the solver calls; residual evaluations happen in separate, untimed passes."""
    import torch

    import ctlab_b200 as cb
    from ctlab_b200 import geometry as G
    from ctlab_b200.learned import WarmStartNet

    ws, rank, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    g = G.config3()
    hx, hy, hz = G.half_extents(g)
    plan = cb.Plan(g, device=local)
    stream = torch.cuda.current_stream()
    OS, IT, I0, SCALE = 24, 30, 1e5, 1.0 / 0.03

    def event_ms(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def scan(seed):
        truth = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        cb.ellipsoid_phantom(truth, g, cb.random_ellipsoids(seed, hx, hy, hz))
        clean = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
        plan.proj(truth, clean)
        gen = torch.Generator(device="cuda")
        gen.manual_seed(seed)
        counts = torch.poisson(I0 * torch.exp(-clean), generator=gen)
        return truth, -torch.log(torch.clamp(counts, min=1.0) / I0)

    t0 = time.perf_counter()
    pairs = []
    for s in range(args.train_volumes):
        _, meas = scan(1000 + s)
        x = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        plan.os_sart(x, meas, os_num=OS, iter_num=2)
        x2 = x.clone()
        plan.os_sart(x, meas, os_num=OS, iter_num=IT - 2)
        pairs.append((x2, x))
        del meas
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0

    net = WarmStartNet(seed=0)
    rng = np.random.default_rng(0)
    losses = []
    t0 = time.perf_counter()
    for step in range(args.train_steps):
        lr = 1e-3 * 0.5 * (1 + np.cos(np.pi * step / args.train_steps))
        x2, x30 = pairs[int(rng.integers(len(pairs)))]
        losses.append(net.train_step(x2, x30, rng.integers(0, g.ZN, 8), SCALE, lr=max(lr, 2e-5)))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    net.check_kernels()

    # one untimed inference first: the first inference after training pays host-side
    # start-up (allocator, first batch-16 shapes) that grows with the training run
    _, warm_meas = scan(6)
    xw0 = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
    plan.os_sart(xw0, warm_meas, os_num=OS, iter_num=2)
    net.predict_volume(xw0, SCALE, torch.empty_like(xw0))
    del warm_meas, xw0

    def held_out(seed):
        truth, meas = scan(seed)
        # plain: 30 iterations from zero
        x = torch.zeros_like(truth)
        t30 = event_ms(lambda: plan.os_sart(x, meas, os_num=OS, iter_num=IT))
        xr = torch.zeros_like(truth)
        res_plain = plan.os_sart(xr, meas, os_num=OS, iter_num=IT, residuals=True)
        r30 = float(res_plain[-1])
        rmse_plain = float(torch.sqrt(torch.mean((x - truth) ** 2)))
        # learned: 2 iterations, the network, then iterations until the residual reaches R30
        xl = torch.zeros_like(truth)
        t2 = event_ms(lambda: plan.os_sart(xl, meas, os_num=OS, iter_num=2))
        xw = torch.zeros_like(truth)
        tcnn = event_ms(lambda: net.predict_volume(xl, SCALE, xw))
        net.check_kernels()
        rmse_warm = float(torch.sqrt(torch.mean((xw - truth) ** 2)))
        xc = xw.clone()
        res_cont = plan.os_sart(xc, meas, os_num=OS, iter_num=IT, residuals=True)
        hits = [k + 1 for k, r in enumerate(res_cont) if r <= r30]
        k = hits[0] if hits else None
        tk = 0.0
        xk = xw.clone()
        if k:
            tk = event_ms(lambda: plan.os_sart(xk, meas, os_num=OS, iter_num=k))
        rmse_learned = float(torch.sqrt(torch.mean((xk - truth) ** 2)))
        t_learned = t2 + tcnn + tk
        return {"seed": seed, "plain_ms": t30, "residual_30": r30, "rmse_plain": rmse_plain,
                "os_sart_2_ms": t2, "cnn_ms": tcnn, "continued_iterations": k, "continued_ms": tk,
                "learned_ms": t_learned if k else None, "residual_after_cnn": float(res_cont[0]),
                "rmse_after_cnn": rmse_warm, "rmse_learned": rmse_learned,
                "time_ratio": (t_learned / t30) if k else None}

    clk = ClockSampler(local).__enter__()
    evals = [held_out(seed) for seed in range(7, 7 + max(1, args.held_out))]
    clk.__exit__(None, None, None)
    ratios = [e["time_ratio"] for e in evals]
    reached = [r for r in ratios if r is not None]
    line = {"metric": "learned warm start: time to the plain 30-iteration OS-SART residual",
            "workload": "learned_warm_start_256x256x128_720v_384x128", "n_gpus": 1,
            "data": "synthetic (seeded random-ellipsoid phantoms, Poisson noise I0=1e5)",
            "network": "2.5D residual CNN, 5 slices in, 8 conv3x3 layers of 64 channels, BF16 weights / FP32 accumulate",
            "training": {"volumes": args.train_volumes, "slice_pairs": args.train_volumes * g.ZN,
                         "steps": args.train_steps, "batch_slices": 8, "data_s": t_data, "train_s": t_train,
                         "loss_first": float(np.mean(losses[:20])), "loss_last": float(np.mean(losses[-20:])),
                         "deviation": f"{args.train_volumes} method-generated volume pairs ({args.train_volumes * g.ZN} "
                                      "slice pairs), not 2000 volume pairs: 2000 x 30 OS-SART iterations would take "
                                      "about 45 min of GPU time per run"},
            "held_out": evals, "held_out_phantoms": len(evals),
            "reached_plain_residual": len(reached),
            "time_ratio_median": float(np.median(reached)) if reached else None,
            "time_ratio_worst": float(max(reached)) if len(reached) == len(evals) else None,
            "target_ratio": 0.5, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    plan.close()


def run_batch(args):
    """The uneven batch (48 scans, seed 7: volumes from {128^3, 192x192x96, 256x256x64,
    384x384x32}, 180-720 views, detectors 256-768 x 32-64, seeded random-ellipsoid
    phantoms): projection of every scan (z-prefix build + projector) as per-scan launches
    with the default staging, versus one persistent launch over all scans with autotuned
    stagings, replayed from a CUDA graph.  Device times with CUDA events."""
    import torch

    import ctlab_b200 as cb
    from ctlab_b200 import geometry as G

    ws, rank, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    geoms = G.config4()[: max(1, min(args.cases, 48))]
    vols, outs = [], []
    for i, g in enumerate(geoms):
        hx, hy, hz = G.half_extents(g)
        v = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        cb.ellipsoid_phantom(v, g, cb.random_ellipsoids(500 + i, hx, hy, hz))
        vols.append(v)
        outs.append(torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda"))
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream

    def timed(fn, reps):
        for _ in range(2):
            fn()
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
        stream.synchronize()
        return e0.elapsed_time(e1) / reps

    plans = [cb.Plan(g) for g in geoms]
    per_ms = timed(lambda: [p.proj(v, o, stream=sp) for p, v, o in zip(plans, vols, outs)], 3)
    refs = [o.clone() for o in outs]
    tune_s = time.perf_counter()
    cache = os.path.join(ROOT, "_build", "proj_tiles.jsonl")
    os.makedirs(os.path.dirname(cache), exist_ok=True)
    tuned = [p.autotune(v, o, cache) for p, v, o in zip(plans, vols, outs)]
    tune_s = time.perf_counter() - tune_s
    tuned_per_ms = timed(lambda: [p.proj(v, o, stream=sp) for p, v, o in zip(plans, vols, outs)], 3)
    batch = cb.Batch(plans)
    with ClockSampler(local) as clk:
        batch_ms = timed(lambda: batch.proj(vols, outs, graph=False, stream=sp), 3)
        graph_ms = timed(lambda: batch.proj(vols, outs, graph=True, stream=sp), 3)
    torch.cuda.synchronize()
    rel = max(float(torch.linalg.norm(o - r) / torch.linalg.norm(r)) for o, r in zip(outs, refs))
    vv = batch.voxel_views
    line = {"metric": "uneven batch projection: one persistent launch vs per-scan launches",
            "workload": "batch48_seed7" if len(geoms) == 48 else f"batch48_seed7_first{len(geoms)}",
            "n_gpus": 1, "cases": len(geoms),
            "data": "synthetic (seeded random-ellipsoid phantoms)", "voxel_views": vv,
            "per_scan_ms": per_ms, "per_scan_autotuned_ms": tuned_per_ms, "batched_ms": batch_ms,
            "batched_graph_ms": graph_ms, "speedup_vs_per_scan": per_ms / graph_ms,
            "gvoxel_views_per_s": {"per_scan": vv / (per_ms * 1e-3) / 1e9, "batched_graph": vv / (graph_ms * 1e-3) / 1e9},
            "autotune_s": tune_s, "autotuned_cases": sum(1 for t in tuned if t > 0),
            "max_rel_diff_vs_default_staging": rel, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    batch.close()
    for p in plans:
        p.close()


def run_helical(args):
    """Projection and backprojection of a long helical scan (512x512x1024 at 1 x 1 x 0.5
    mm, 14 turns of 984 views, pitch 1, the 888x64 detector): each view's cone meets a
    short z slab of the volume, so backprojector CTAs whose z range the cone misses skip
    the view.  Device times with CUDA events; inputs larger than L2."""
    import torch

    import ctlab_b200 as cb
    from ctlab_b200 import geometry as G

    ws, rank, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    g = G.helical()
    hx, hy, hz = G.half_extents(g)
    vol = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
    cb.ellipsoid_phantom(vol, g, cb.random_ellipsoids(21, hx, hy, hz))
    prj = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
    back = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
    plan = cb.Plan(g, device=local)
    plan.set_timing(True)
    steps, warm = max(1, min(args.steps, 2)), max(1, min(args.warmup, 1))
    times = []
    with ClockSampler(local) as clk:
        for it in range(warm + steps):
            plan.proj(vol, prj)
            torch.cuda.synchronize()
            ps, pg = plan.last_times()
            plan.back(prj, back)
            torch.cuda.synchronize()
            bs, bg = plan.last_times()
            if it >= warm:
                times.append((ps, pg, bs, bg))
    t = np.array(times).mean(axis=0)
    vv = g.voxel_views
    line = {"metric": "helical projection / backprojection time", "workload": "helical_512x512x1024_13776v_888x64",
            "n_gpus": 1, "data": "synthetic (seeded random-ellipsoid phantom)", "views": g.PN,
            "volume": [g.XN, g.YN, g.ZN], "voxel_mm": [g.dx, g.dx, g.dz], "pitch": 1.0,
            "proj_ms": float(t[0] + t[1]), "back_ms": float(t[2] + t[3]),
            "kernels_ms": {"proj_sat": float(t[0]), "proj": float(t[1]), "back_sat": float(t[2]), "back": float(t[3])},
            "gvoxel_views_per_s": {"proj": vv / ((t[0] + t[1]) * 1e-3) / 1e9, "back": vv / ((t[2] + t[3]) * 1e-3) / 1e9},
            "steps": steps, "warmup": warm, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    plan.close()


def main():
    args = parse()
    if args.workload == "batch":
        run_batch(args)
    elif args.workload == "helical":
        run_helical(args)
    elif args.workload == "recon":
        run_recon(args)
    elif args.workload == "learned":
        run_learned(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
