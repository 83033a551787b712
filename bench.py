#!/usr/bin/env python
"""Benchmark: forward+backward views/s of the FilterGS tile rasterizer.

Workload (one step = one view, forward + backward, plain one-view-per-call path):
  urban aerial scene, 2,000,000 Gaussians (70% ground plane, 30% faces of 400 boxes),
  SH degree 3, 1920x1080 camera at 150 m altitude, 45 deg pitch, random yaw, upstream
  gradient ~ N(0,1).  Synthetic, seeded; 8 distinct cameras cycled over the steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's own rasterizer (its CUDA sources compiled
unmodified into oracle/_ref by oracle/build_ref.py) on the same workload, through its
own `_C` entry points.  The reference has no CPU implementation of this path.

Prints ONE JSON line (rank 0).  `value` is device-timed with CUDA events over exactly K
steps (inputs resident in HBM; the 472 MB of Gaussian parameters exceed the 126 MB L2),
max over ranks.  `e2e` is the same metric through the public operator API with the
per-step camera and upstream gradient copied in from pinned host memory and the
rendered image copied back.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "fwd+bwd views/s @2M Gaussians 1080p: batched vs plain, same GPU; HBM GB/s frac"
WORKLOAD = "urban-aerial 2M Gaussians SH3, 1920x1080, fwd+bwd, plain one-view-per-call path"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--P", type=int, default=2_000_000)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--views", type=int, default=8)
    ap.add_argument("--stats", action="store_true", help="ogfs_enable_stats=True (the API default)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default render kernel shape")
    ap.add_argument("--render-config", default=None,
                    help="fwd_ppt,fwd_batch,bwd_ppt,bwd_batch (skips the autotuner)")
    return ap.parse_args()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, timeout=10.0):
        """Block until nvidia-smi produced a sample, so its start-up never overlaps the timed region."""
        t0 = time.time()
        while self.proc is not None and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.05)
        n = len(self.lines)
        # keep only samples taken from now on
        self.skip = n

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[getattr(self, "skip", 0):]:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- workload
def make_workload(args, device, rank):
    from filtergs_b200 import synthetic as S
    sc = S.urban_scene(P=args.P, seed=1001)
    rng = np.random.default_rng(2001 + 97 * rank)
    cams = [S.aerial_camera(rng, W=args.width, H=args.height) for _ in range(args.views)]
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
    scene = dict(means3D=t(sc["means3D"]), scales=t(sc["scales"]), rotations=t(sc["rotations"]),
                 opacities=t(sc["opacities"]), shs=t(sc["shs"]))
    g = torch.Generator(device="cpu").manual_seed(3001 + rank)
    views = []
    for c in cams:
        views.append(dict(cam=c, view=t(c.viewmatrix), proj=t(c.projmatrix), campos=t(c.campos),
                          dL=torch.randn(3, c.H, c.W, generator=g).to(device),
                          dL_host=torch.randn(3, c.H, c.W, generator=g).pin_memory()))
    return sc, scene, views


def step_c(mod, scene, v, bg, stats):
    """One forward + backward through the `_C` entry points (reference signature)."""
    e = torch.empty(0, device=bg.device)
    c = v["cam"]
    out = mod.rasterize_gaussians(bg, scene["means3D"], e, scene["opacities"], scene["scales"], scene["rotations"],
                                  1.0, e, v["view"], v["proj"], c.tanfovx, c.tanfovy, c.H, c.W, scene["shs"], 3,
                                  v["campos"], False, True, False, 0.2, 0.2, 0.05, 0.7, stats)
    K, color, pid, pwp, pw, radii, geom, binning, img, st = out
    grads = mod.rasterize_gaussians_backward(bg, scene["means3D"], radii, e, scene["scales"], scene["rotations"], 1.0,
                                             e, v["view"], v["proj"], c.tanfovx, c.tanfovy, v["dL"], scene["shs"], 3,
                                             v["campos"], geom, K, binning, img, False)
    return K, radii, color, grads


# algorithmic bytes per launch (per view) for each stage; K pairs, V visible, P Gaussians, N pixels
def algo_bytes(stage, P, V, K, N, T, M=16):
    if stage == "preprocess":
        return 44 * P + 4 * M * 3 * V + 56 * V + 4 * P
    if stage == "duplicate":
        return 8 * P + 12 * K
    if stage == "tile_sort":
        return 24 * K * 2
    if stage == "ranges":
        return 8 * K + 8 * T
    if stage == "render_fwd":
        return 40 * K + 28 * N
    if stage == "render_bwd":
        return 40 * K + 20 * N + 44 * V
    if stage == "preprocess_bwd":
        return V * (12 + 24 + 16 + 12 + 12 + 16 + 12 + 3 + 192) + P * 284
    if stage == "depth_sort":
        return 4 * 16 * P
    return 0


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(stage):
    """dram bytes per launch for `stage` from the committed ncu summary (None if absent)."""
    p = os.path.join(ROOT, "profiles", "traffic_urban1080.md")
    try:
        with open(p) as f:
            for ln in f:
                if ln.startswith("traffic_per_launch[") and ln.split("[")[1].split("]")[0] == stage:
                    return float(ln.split("=")[1].strip().split()[0])
    except OSError:
        pass
    return None


def cpu_baseline(sc, cam, threads):
    """The C oracle (a CPU port of the reference splat math) on the same view, all host threads.

    Sample: full preprocess, binning and per-Gaussian backward; render forward/backward on 4 evenly
    spaced slices of 1/64 of the tiles each, scaled to the full frame."""
    from oracle import oracle as O
    O.set_threads(threads)
    s = O.Scene(sc["means3D"], sc["opacities"], cam.W, cam.H, cam.tanfovx, cam.tanfovy, cam.viewmatrix.reshape(-1),
                cam.projmatrix.reshape(-1), cam.campos, shs=sc["shs"], sh_degree=3, scales=sc["scales"],
                rotations=sc["rotations"])
    t0 = time.perf_counter()
    pre = O.preprocess(s)
    t1 = time.perf_counter()
    keys, vals, ranges = O.bin_pairs(pre, cam.W, cam.H)
    t2 = time.perf_counter()
    T = ranges.shape[0]
    chunk = max(1, T // 64)
    starts = [int(T * f) for f in (0.1, 0.35, 0.6, 0.85)]
    t_r = t_b = 0.0
    dL = np.random.default_rng(0).standard_normal((3, cam.H, cam.W)).astype(np.float32)
    fwd = None
    for st in starts:
        a = time.perf_counter()
        r = O.render(s, pre, vals, ranges, tile_range=(st, min(T, st + chunk)))
        b = time.perf_counter()
        r.update(pre=pre, keys=keys, vals=vals, ranges=ranges)
        if fwd is None:
            fwd = r
        O.backward(s, r, dL, tile_range=(st, min(T, st + chunk)))
        c = time.perf_counter()
        t_r += b - a
        t_b += c - b
    covered = len(starts) * chunk
    # the per-Gaussian backward ran once per slice; count it once, the tile work scaled up
    a = time.perf_counter()
    O.backward(s, fwd, dL, tile_range=(0, 0))
    t_pb = time.perf_counter() - a
    t_tiles = (t_r + t_b - len(starts) * t_pb) * (T / covered)
    total = (t1 - t0) + (t2 - t1) + t_tiles + t_pb
    return {"value": 1.0 / total, "unit": "views/s", "cores": threads, "kind": "port",
            "sample": f"1 view: full preprocess+binning+per-Gaussian backward, render fwd+bwd on {covered}/{T} tiles "
                      f"scaled x{T / covered:.1f}; measured {(t1 - t0) + (t2 - t1) + t_r + t_b + t_pb:.1f}s CPU wall"}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = world > 1
    if dist:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.impl == "reference" and dist and rank != 0:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
        return
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)

    if args.impl == "reference":
        from oracle import build_ref
        mod = build_ref.load("ref_rasterizer_C")
        if mod is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/ref_rasterizer_C.so "
                                                                   "missing (needs the reference tree to compile)"}))
            if dist:
                torch.distributed.barrier()
                torch.distributed.destroy_process_group()
            return
    else:
        from filtergs_b200 import _C as mod
        from filtergs_b200 import _lib

    sc, scene, views = make_workload(args, device, rank)
    bg = torch.zeros(3, device=device)
    nv = len(views)
    tuned = None
    if args.impl == "ours" and args.render_config:
        _lib.set_render_config(*[int(x) for x in args.render_config.split(",")])
    elif args.impl == "ours" and not args.no_autotune:
        from filtergs_b200.autotune import tune_render
        it = iter(range(1 << 30))
        tuned, table = tune_render(lambda: step_c(mod, scene, views[next(it) % nv], bg, args.stats),
                                   key=("urban", args.P, args.width, args.height))
        if rank == 0:
            print("autotune render (ppt,batch)->(fwd ms, bwd ms): " +
                  ", ".join(f"{k}:{v[0]:.3f}/{v[1]:.3f}" for k, v in sorted(table.items())), file=sys.stderr)
    clocks = ClockSampler(local) if rank == 0 else None
    if clocks:
        clocks.start()
        clocks.wait_first()
    for i in range(args.warmup):
        step_c(mod, scene, views[i % nv], bg, args.stats)
    torch.cuda.synchronize()
    if dist and args.impl == "ours":
        torch.distributed.barrier()
    if clocks:
        clocks.skip = len(clocks.lines)
    if args.impl == "ours":
        _lib.profile_read(reset=True)
        _lib.profile_enable(True)
        l0 = _lib.launch_count()
    Ks, Vs = [], []
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    for i in range(args.steps):
        K, radii, color, grads = step_c(mod, scene, views[i % nv], bg, args.stats)
        Ks.append(K)
        Vs.append(radii)
    end.record()
    torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    if args.impl == "ours":
        launches = _lib.launch_count() - l0
        _lib.profile_enable(False)
        prof = _lib.profile_read(reset=True)
    clk = clocks.stop() if clocks else None
    Vs = [int((r > 0).sum().item()) for r in Vs]
    if dist and args.impl == "ours":
        t = torch.tensor([ms], device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    n_ranks = world if args.impl == "ours" else 1
    value = n_ranks * args.steps / (ms / 1000.0)

    # ---------------------------------------------------------------- e2e through the public API
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, mod, scene, views, bg, device, dist)

    result = None
    if rank == 0:
        cfg = {"workload": WORKLOAD, "gaussians": args.P, "width": args.width, "height": args.height, "sh_degree": 3,
               "views_cycled": nv, "path": "plain", "ogfs_enable_stats": bool(args.stats),
               "l2": "inputs larger than L2 (472 MB Gaussian parameters per step)",
               "mean_pairs_K": float(np.mean(Ks)), "mean_visible_V": float(np.mean(Vs))}
        result = {"metric": METRIC, "value": value, "unit": "views/s", "n_gpus": n_ranks, "steps": args.steps,
                  "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                  "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded urban-aerial scene)",
                  "config": cfg}
        if args.impl == "reference":
            result["impl"] = "reference"
            result["cpu_baseline"] = {"value": value, "unit": "views/s", "cores": 1, "kind": "reference",
                                      "sample": "the reference's own rasterizer (CUDA sources compiled unmodified, "
                                                "oracle/_ref) on this GPU; it has no CPU implementation"}
            if e2e:
                result["e2e"] = e2e
            else:
                result["e2e"] = {"value": value, "unit": "views/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
        else:
            P, N = args.P, args.width * args.height
            T = ((args.width + 15) // 16) * ((args.height + 15) // 16)
            Km, Vm = float(np.mean(Ks)), float(np.mean(Vs))
            stages = {k: {"ms_total": v[0], "launch_groups": v[1], "ms_per_call": (v[0] / v[1]) if v[1] else 0.0}
                      for k, v in prof.items()}
            dom = max(prof, key=lambda k: prof[k][0])
            peak, peak_kind = measured_peak()
            per_call_ms = prof[dom][0] / max(1, prof[dom][1])
            ab = algo_bytes(dom, P, Vm, Km, N, T)
            achieved = ab / (per_call_ms / 1000.0) / 1e9
            result["roofline"] = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                                  "unit": "GB/s", "frac": achieved / peak, "traffic": ncu_traffic(dom),
                                  "algorithmic_bytes_per_launch": ab, "peak_source": peak_kind,
                                  "note": "render kernels are exp/FP32-issue bound; see profiles/ for pipe utilisation"}
            result["stages"] = stages
            result["config"]["render_config"] = list(_lib.get_render_config())
            result["config"]["autotuned"] = tuned is not None
            result["gpu_launches"] = int(launches)
            if e2e:
                result["e2e"] = e2e
            if not args.no_cpu_baseline:
                result["cpu_baseline"] = cpu_baseline(sc, views[0]["cam"], os.cpu_count() or 1)
        if clk:
            result["clocks"] = clk
        print(json.dumps(result), flush=True)
    if dist:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def run_e2e(args, mod, scene, views, bg, device, dist):
    """Same metric through the public API: per step, H2D of the camera and the upstream gradient from
    pinned host memory, forward + backward, D2H of the rendered image.  The copies run on a side stream:
    step i+1's inputs are uploaded while step i computes, and step i's image is downloaded while its
    backward runs, as a pipelined caller would do; every step still moves its own bytes."""
    nv = len(views)
    c0 = views[0]["cam"]
    host_cam = [torch.from_numpy(np.concatenate([v["cam"].viewmatrix.reshape(-1), v["cam"].projmatrix.reshape(-1),
                                                 v["cam"].campos])).pin_memory() for v in views]
    out_host = [torch.empty(3, c0.H, c0.W).pin_memory() for _ in range(2)]
    dev_cam = [torch.empty(35, device=device) for _ in range(2)]
    dev_dL = [torch.empty(3, c0.H, c0.W, device=device) for _ in range(2)]
    copy = torch.cuda.Stream(device=device)
    main = torch.cuda.current_stream(device)
    if args.impl == "ours":
        from filtergs_b200.rasterization import GaussianRasterizationSettings, GaussianRasterizer
        means = scene["means3D"].clone().requires_grad_(True)
        shs = scene["shs"].clone().requires_grad_(True)
        op = scene["opacities"].clone().requires_grad_(True)
        scl = scene["scales"].clone().requires_grad_(True)
        rot = scene["rotations"].clone().requires_grad_(True)
        m2 = torch.zeros_like(means, requires_grad=True)
    ready = [torch.cuda.Event() for _ in range(2)]
    freed = [torch.cuda.Event() for _ in range(2)]

    def upload(i):
        b = i & 1
        with torch.cuda.stream(copy):
            copy.wait_event(freed[b])
            dev_cam[b].copy_(host_cam[i % nv], non_blocking=True)
            dev_dL[b].copy_(views[i % nv]["dL_host"], non_blocking=True)
            ready[b].record(copy)

    def one(i):
        b = i & 1
        v = views[i % nv]
        c = v["cam"]
        main.wait_event(ready[b])
        if i + 1 < total[0]:
            upload(i + 1)
        view, proj, cpos = dev_cam[b][:16].view(4, 4), dev_cam[b][16:32].view(4, 4), dev_cam[b][32:35]
        if args.impl == "ours":
            rs = GaussianRasterizationSettings(c.H, c.W, c.tanfovx, c.tanfovy, bg, 1.0, view, proj, 3, cpos, False,
                                               False, ogfs_enable_stats=bool(args.stats))
            for t in (means, shs, op, scl, rot, m2):
                t.grad = None
            color = GaussianRasterizer(rs)(means, m2, op, shs=shs, scales=scl, rotations=rot)[0]
            img_done = torch.cuda.Event()
            img_done.record(main)
            with torch.cuda.stream(copy):
                copy.wait_event(img_done)
                out_host[b].copy_(color.detach(), non_blocking=True)
            color.backward(dev_dL[b])
        else:
            e = torch.empty(0, device=device)
            out = mod.rasterize_gaussians(bg, scene["means3D"], e, scene["opacities"], scene["scales"],
                                          scene["rotations"], 1.0, e, view, proj, c.tanfovx, c.tanfovy, c.H, c.W,
                                          scene["shs"], 3, cpos, False, True, False, 0.2, 0.2, 0.05, 0.7, args.stats)
            K, color, pid, pwp, pw, radii, geom, binning, img, st = out
            img_done = torch.cuda.Event()
            img_done.record(main)
            with torch.cuda.stream(copy):
                copy.wait_event(img_done)
                out_host[b].copy_(color, non_blocking=True)
            mod.rasterize_gaussians_backward(bg, scene["means3D"], radii, e, scene["scales"], scene["rotations"], 1.0,
                                             e, view, proj, c.tanfovx, c.tanfovy, dev_dL[b], scene["shs"], 3, cpos,
                                             geom, K, binning, img, False)
        freed[b].record(main)

    total = [args.warmup]
    upload(0)
    for i in range(args.warmup):
        one(i)
    torch.cuda.synchronize()
    if dist and args.impl == "ours":
        torch.distributed.barrier()
    total[0] = args.steps
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    copy.wait_event(start)
    upload(0)
    for i in range(args.steps):
        one(i)
    main.wait_stream(copy)      # the last image download is inside the timed region
    end.record()
    end.synchronize()
    ms = start.elapsed_time(end)
    torch.cuda.synchronize()
    if dist and args.impl == "ours":
        t = torch.tensor([ms], device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    n_ranks = (int(os.environ.get("WORLD_SIZE", "1")) if args.impl == "ours" else 1)
    return {"value": n_ranks * args.steps / (ms / 1000.0), "unit": "views/s",
            "h2d_bytes_per_step": int(35 * 4 + 3 * c0.H * c0.W * 4), "d2h_bytes_per_step": int(3 * c0.H * c0.W * 4)}


if __name__ == "__main__":
    main()
