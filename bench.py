#!/usr/bin/env python
"""Benchmark: forward+backward views/s of the FilterGS tile rasterizer, batched vs plain.

Workload: urban aerial scene, 2,000,000 Gaussians (70% ground plane, 30% faces of 400
boxes), SH degree 3; 16 cameras at 1920x1080, fx=fy=1600, 150 m altitude, 45 deg pitch,
random position and yaw; upstream gradient ~ N(0,1) per view.  Synthetic and seeded.

One step = forward + backward of all 16 views:
  batched (headline): one CUDA-graph replay of the batched path (per-view front ends,
      one persistent compositing launch per direction over all views' tiles, gradients
      summed into shared buffers; no host synchronisation);
  plain (beside it):  16 calls of the one-view-per-call `_C` operator path.
A second workload (the mixed-resolution batch: 16 cameras with resolutions drawn from
{640x360, 1280x720, 1600x900, 1920x1080}, altitudes 80-300 m, pitch 30-75 deg) is
measured the same way and reported under `mixed_resolution`; `lod_tree` is the per-view
LoD selection + forward render of an 8M-node Gaussian tree, and `train_step` the ms per
iteration of a full training step (4M Gaussians, 4 views 1600x900, L1 + SSIM, backward,
Adam) batched vs plain.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--path batched|plain]

--impl reference times the reference's own rasterizer (its CUDA sources compiled
unmodified into oracle/_ref by oracle/build_ref.py) on the same 16 cameras, one view per
call through its own `_C` entry points (it has no batched path and no CPU implementation).

Prints ONE JSON line (rank 0).  `value` is device-timed with CUDA events over exactly K
steps (inputs resident in HBM; the 472 MB of Gaussian parameters exceed the 126 MB L2),
max over ranks; ranks render disjoint camera sets (weak scaling, no collective on the
data path).  `e2e` is the same metric through the public API with every view's camera
and upstream gradient copied in from pinned host memory and every rendered image copied
back, inside the timed region.
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
MIXED_RES = ((640, 360), (1280, 720), (1600, 900), (1920, 1080))


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--path", choices=["batched", "plain"], default="batched",
                    help="the path timed as `value` (the other one is measured beside it unless --no-plain)")
    ap.add_argument("--P", type=int, default=2_000_000)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--views", type=int, default=16, help="cameras per step")
    ap.add_argument("--stats", action="store_true", help="ogfs_enable_stats=True in the plain path (API default)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-path comparison")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-resolution workload")
    ap.add_argument("--no-lod", action="store_true", help="skip the LoD-tree filter + render workload")
    ap.add_argument("--no-train", action="store_true", help="skip the training-step workload")
    ap.add_argument("--train-gaussians", type=int, default=4_000_000)
    ap.add_argument("--lod-nodes", type=int, default=8_000_000)
    ap.add_argument("--no-autotune", action="store_true", help="keep the default render kernel shape")
    ap.add_argument("--only", choices=["lod", "train"], default=None,
                    help="run only this workload on one GPU and print its result (profiling entry point)")
    ap.add_argument("--render-config", default=None,
                    help="fwd_ppt,fwd_batch,bwd_ppt,bwd_batch (skips the autotuner)")
    return ap.parse_args(argv)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampled every 200 ms in the background; `window(t0, t1)` summarises the samples
    taken between two host times (the timed region)."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

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
            self.lines.append((time.time(), line.strip()))

    def wait_first(self, timeout=10.0):
        """Block until nvidia-smi produced a sample, so its start-up never overlaps a timed region."""
        t0 = time.time()
        while self.proc is not None and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.05)

    def window(self, t0, t1):
        sm, mx, reasons = [], [], set()
        for t, ln in list(self.lines):
            if t < t0 or t > t1 + 0.25:
                continue
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(self.REASONS, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}

    def stop(self):
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()


# ---------------------------------------------------------------- workload
def make_scene(P, device):
    from filtergs_b200 import synthetic as S
    sc = S.urban_scene(P=P, seed=1001)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
    return sc, dict(means3D=t(sc["means3D"]), scales=t(sc["scales"]), rotations=t(sc["rotations"]),
                    opacities=t(sc["opacities"]), shs=t(sc["shs"]))


def rank_cameras(n, rank, W=1920, H=1080, mixed=False):
    """n cameras of the 1080p workload, or of the mixed-resolution one (same field of view at every
    resolution: fx scales with the width).  Rank r draws its own cameras (host only)."""
    from filtergs_b200 import synthetic as S
    rng = np.random.default_rng((4001 if mixed else 2001) + 97 * rank)
    cams = []
    for _ in range(n):
        if mixed:
            w, h = MIXED_RES[int(rng.integers(len(MIXED_RES)))]
            cams.append(S.aerial_camera(rng, W=w, H=h, fx=1600.0 * w / 1920, altitude=float(rng.uniform(80, 300)),
                                        pitch_deg=float(rng.uniform(30, 75))))
        else:
            cams.append(S.aerial_camera(rng, W=W, H=H))
    return cams


def aggregate_views_per_s(n_ranks, views_per_rank, steps, ms_max):
    """Whole-job views/s: every rank renders its own views_per_rank cameras per step; the step time
    is the slowest rank's (max over ranks)."""
    return n_ranks * views_per_rank * steps / (ms_max / 1000.0)


def make_views(n, device, rank, W=1920, H=1080, mixed=False):
    """rank_cameras(...) on `device`, with a seeded upstream gradient per view (device copy and a
    pinned host copy for the end-to-end leg)."""
    cams = rank_cameras(n, rank, W, H, mixed)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
    g = torch.Generator(device="cpu").manual_seed(3001 + 7 * rank + (1 if mixed else 0))
    views = []
    for c in cams:
        views.append(dict(cam=c, view=t(c.viewmatrix), proj=t(c.projmatrix), campos=t(c.campos),
                          dL=torch.randn(3, c.H, c.W, generator=g).to(device),
                          dL_host=torch.randn(3, c.H, c.W, generator=g).pin_memory()))
    return views


def step_c(mod, scene, v, bg, stats):
    """One view forward + backward through the `_C` entry points (reference signature)."""
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


def make_batched(scene, views, bg):
    """BatchedRasterizer over `views`; its cameras live in one packed device buffer br.cam_dev
    [nv, 35] (view 16, proj 16, campos 3 per row).  Every forward output of the reference's call is
    produced per view (image, radii, point_id, point_weight_pixel, point_weight); the gradients of all
    views are summed into the shared parameter gradients."""
    from filtergs_b200.batched import BatchedRasterizer, Camera
    cam_dev = torch.stack([torch.cat([v["view"].reshape(-1), v["proj"].reshape(-1), v["campos"].reshape(-1)])
                           for v in views]).contiguous()
    cams = [Camera(v["cam"].W, v["cam"].H, v["cam"].tanfovx, v["cam"].tanfovy, cam_dev[i, :16], cam_dev[i, 16:32],
                   cam_dev[i, 32:35]) for i, v in enumerate(views)]
    br = BatchedRasterizer(scene["means3D"], scene["opacities"], scene["scales"], scene["rotations"], cams,
                           shs=scene["shs"], sh_degree=3, bg=bg, graph=True, full_outputs=True)
    br.cam_dev = cam_dev
    br.set_io_many(list(range(len(views))), list(br.images), [v["dL"] for v in views])
    return br


# algorithmic bytes per launch (per view) for each stage; K pairs, V visible, P Gaussians, N pixels, T tiles
def algo_bytes(stage, P, V, K, N, T, M=16, tile_passes=2):
    if stage == "preprocess":
        # means/scales/rotations/opacity of every Gaussian, SH rows of the visible ones; radii, tiles (and the
        # caller's radii) for all, the 48-byte record and clamp bits for the visible, compacted ids and keys
        return 44 * P + 4 * M * 3 * V + 12 * P + 49 * V + 8 * V
    if stage == "depth_sort":
        return 4 * 16 * V + 4 * V          # 4 passes of keys + ids in and out, one histogram read
    if stage == "duplicate":
        return 28 * V + 12 * V + 8 * K     # ids, tiles, record xy, radius in; pair offsets out; tile + id per pair
    if stage == "tile_sort":
        return 16 * K * tile_passes + 104 * K   # keys + ids per pass; last pass gathers 48-byte records
    if stage == "ranges":
        return 8 * K + 8 * T
    if stage == "render_fwd":
        return 40 * K + 28 * N
    if stage == "render_bwd":
        # the algorithm's own bytes: records 40 B per pair; dL/dpix, T, n_contrib per pixel; the 44-byte
        # screen-space gradient accumulators written once per visible Gaussian
        return 40 * K + 20 * N + 44 * V
    if stage == "render_bwd_design":
        return 76 * K + 20 * N  # this design's traffic: records 40 B + the per-pair gradient row 36 B per pair
    if stage == "preprocess_bwd":
        return 36 * K + V * (12 + 24 + 16 + 12 + 12 + 16 + 12 + 3 + 192) + P * 284
    return 0


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def kernel_source_digest():
    """Short digest of the render kernels' source, stamped into the ncu summaries they were captured from."""
    import hashlib
    h = hashlib.sha256()
    for f in ("render.cu", "fgs_common.cuh"):
        with open(os.path.join(ROOT, "filtergs_b200", "csrc", f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:12]


def ncu_per_pair(field, key, pairs, what):
    """`field`[key] per pair from the committed ncu summary of the CURRENT render kernels, times pairs.
    (None, reason) when the summary has no figure for this key or was captured from other kernel sources
    than the ones built now."""
    p = os.path.join(ROOT, "profiles", "render_traffic_urban1080.md")
    digest, per_pair = None, None
    try:
        with open(p) as f:
            for ln in f:
                if ln.startswith("source_digest ="):
                    digest = ln.split("=")[1].strip()
                if ln.startswith(field + "[") and ln.split("[")[1].split("]")[0] == key:
                    per_pair = float(ln.split("=")[1].strip().split()[0])
    except OSError:
        return None, "no ncu summary"
    if per_pair is None:
        return None, f"no ncu figure for {key}"
    if digest != kernel_source_digest():
        return None, "ncu summary is of other kernel sources"
    return per_pair * pairs, f"ncu {what} per pair x pairs ({os.path.relpath(p, ROOT)})"


def ncu_traffic(key, pairs):
    """DRAM bytes of one launch of `key`: the captured bytes per pair x pairs."""
    return ncu_per_pair("traffic_per_pair", key, pairs, "dram bytes")


# Warp instructions an SM can issue per cycle (four schedulers, one each), and the B200's maximum SM
# clock: the issue roof of a kernel bound by instruction issue rather than by memory.
ISSUE_PER_SM_CYCLE = 4
SM_MAX_GHZ = 1.965


def issue_roof(key, pairs, launch_ms):
    """Warp instructions of one launch (captured per pair x pairs) / its duration, against the issue roof
    of all SMs at the maximum clock; None when the ncu summary has no current figure for `key`."""
    inst, src = ncu_per_pair("inst_per_pair", key, pairs, "warp instructions")
    if inst is None:
        return {"frac": None, "source": src}
    n_sm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count \
        if torch.cuda.is_available() else 148
    peak = n_sm * ISSUE_PER_SM_CYCLE * SM_MAX_GHZ  # G warp instructions / s
    achieved = inst / (launch_ms / 1000.0) / 1e9
    return {"warp_inst_per_launch": inst, "achieved": achieved, "peak": peak, "unit": "G warp inst/s",
            "frac": achieved / peak, "sms": n_sm, "source": src,
            "peak_source": f"{ISSUE_PER_SM_CYCLE} warp instructions per SM per cycle at {SM_MAX_GHZ * 1000:.0f} MHz"}


def torch_cpu_baseline(sc, cam, threads):
    """The reference's splat math restated in PyTorch-CPU FP32 (oracle/torch_cpu.py, after its torch helpers
    LoG/model/geometry.py and sh_utils.py) on the same view, all host threads: forward + autograd backward.

    Sample: full preprocess and binning (and their backward); tile compositing forward + backward on 4 evenly
    spaced slices of 1/64 of the tiles each, scaled to the full frame."""
    from oracle import torch_cpu as TC
    prev = torch.get_num_threads()
    torch.set_num_threads(threads)
    try:
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a))  # noqa: E731
        args = (t(sc["means3D"]), t(sc["scales"]), t(sc["rotations"]), t(sc["opacities"]), t(sc["shs"]), 3, cam)
        dL = torch.from_numpy(np.random.default_rng(0).standard_normal((3, cam.H, cam.W)).astype(np.float32))
        T = ((cam.W + 15) // 16) * ((cam.H + 15) // 16)
        chunk = max(1, T // 64)
        tiles = [k for st in (int(T * f) for f in (0.1, 0.35, 0.6, 0.85)) for k in range(st, min(T, st + chunk))]
        a = time.perf_counter()
        TC.forward_backward(*args, dL, tiles=[])          # per-Gaussian forward + backward, binning
        b = time.perf_counter()
        TC.forward_backward(*args, dL, tiles=tiles)
        c = time.perf_counter()
    finally:
        torch.set_num_threads(prev)
    t_gauss, t_sample = b - a, c - b
    total = t_gauss + max(0.0, t_sample - t_gauss) * (T / len(tiles))
    return {"value": 1.0 / total, "unit": "views/s", "cores": threads, "kind": "port",
            "impl": "PyTorch-CPU FP32 restatement of the reference's splat math (oracle/torch_cpu.py)",
            "sample": f"1 view: full preprocess+binning fwd+bwd ({t_gauss:.1f}s), tile compositing fwd+bwd on "
                      f"{len(tiles)}/{T} tiles ({t_sample - t_gauss:.1f}s) scaled x{T / len(tiles):.1f}"}


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


# ---------------------------------------------------------------- timing
def _barrier(dist):
    if dist:
        torch.distributed.barrier()


def max_over_ranks(ms, device, dist):
    if not dist:
        return ms
    t = torch.tensor([ms], device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def timed(fn, steps, clocks=None):
    """Device time (ms) of `steps` calls of fn(i): CUDA events on the launching stream, synchronised
    on both sides.  Returns (ms, clock summary of the region)."""
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0 = time.time()
    a.record()
    for i in range(steps):
        fn(i)
    b.record()
    torch.cuda.synchronize()
    t1 = time.time()
    return a.elapsed_time(b), (clocks.window(t0, t1) if clocks else None)


def profiled(fn, steps):
    """Per-stage CUDA-event times of `steps` eager calls of fn(i) (events recorded around each launch
    group on the stream it runs on) and the number of kernels launched."""
    from filtergs_b200 import _lib
    torch.cuda.synchronize()
    _lib.profile_read(reset=True)
    _lib.profile_enable(True)
    l0 = _lib.launch_count()
    for i in range(steps):
        fn(i)
    torch.cuda.synchronize()
    launches = _lib.launch_count() - l0
    _lib.profile_enable(False)
    return _lib.profile_read(reset=True), launches


def autotune(args, fn, key, rank):
    from filtergs_b200 import _lib
    if args.render_config:
        vals = [int(x) for x in args.render_config.split(",")]
        _lib.set_render_config(*vals[:4])
        if len(vals) > 4:
            _lib.set_render_split(*vals[4:6])
        return None
    if args.no_autotune:
        return None
    from filtergs_b200.autotune import tune_render
    it = iter(range(1 << 30))
    tuned, table = tune_render(lambda: fn(next(it)), key=key,
                               splits=((0, 0), (512, 0), (512, 1), (512, 2), (512, 3), (4096, 2)))
    if rank == 0:
        print(f"autotune {key[0]} (ppt,batch)->(fwd ms, bwd ms), then long-tile split->fwd ms: " +
              ", ".join(f"{k}:{v[0]:.3f}/{v[1]:.3f}" for k, v in sorted(table.items(), key=lambda kv: str(kv[0]))),
              file=sys.stderr)
    return list(tuned) + list(_lib.get_render_split())


def measure_plain(args, mod, scene, views, bg, dev, dist, rank, ours=True, clocks=None, profile=False):
    """K steps of the plain path: each step renders (forward + backward) every view, one call each."""
    nv = len(views)
    tuned = None
    if ours:
        tuned = autotune(args, lambda i: step_c(mod, scene, views[i % nv], bg, args.stats),
                         ("plain", args.P, tuple((v["cam"].W, v["cam"].H) for v in views)), rank)
    for _ in range(args.warmup):
        for v in views:
            step_c(mod, scene, v, bg, args.stats)
    torch.cuda.synchronize()
    _barrier(dist)
    first = []

    def one(i):
        for v in views:
            K, radii, color, grads = step_c(mod, scene, v, bg, args.stats)
            if i == 0:
                first.append((K, radii))

    ms, clk = timed(one, args.steps, clocks)
    ms = max_over_ranks(ms, dev, dist)
    out = dict(ms=ms, clocks=clk, tuned=tuned, K=[int(k) for k, _ in first],
               vis=[int((r > 0).sum().item()) for _, r in first])
    if ours and profile:
        out["prof"], out["launches"] = profiled(one, args.steps)
    return out


def measure_batched(args, scene, views, bg, dev, dist, rank, clocks=None, profile=True):
    """K steps of the batched path: each step is one CUDA-graph replay of forward + backward of all views."""
    br = make_batched(scene, views, bg)
    tuned = autotune(args, lambda i: (br.forward(), br.backward()),
                     ("batched", args.P, tuple((v["cam"].W, v["cam"].H) for v in views)), rank)
    for _ in range(args.warmup):
        br.step()                       # the first replay captures the graph (after the autotuner)
    br.check()
    _barrier(dist)
    ms, clk = timed(lambda i: br.step(), args.steps, clocks)
    br.check()
    ms = max_over_ranks(ms, dev, dist)
    out = dict(ms=ms, clocks=clk, tuned=tuned, br=br, K=br.pair_counts(),
               vis=[int((r > 0).sum().item()) for r in br.radii])
    if profile:
        # per-launch times cannot be taken inside a graph replay: the same K steps again, eagerly
        out["prof"], out["launches"] = profiled(lambda i: (br.forward(), br.backward()), args.steps)
        br.check()
    return out


def roofline(prof, P, views, K, vis, batched):
    """Roofline of the dominant kernel: algorithmic bytes per launch / its mean CUDA-event duration.

    In the batched path the per-view front-end stages (preprocess, sorts, pair emission, ranges) run
    on concurrent streams, so their event times overlap one another and their sums overstate their
    device time; the dominant kernel is then taken among the launches that have the device to
    themselves, which is also the ranking of the serialised ncu launch list."""
    alone = [k for k in prof if not batched or k in ("render_fwd", "render_bwd", "preprocess_bwd")]
    dom = max(alone or list(prof), key=lambda k: prof[k][0])
    calls = max(1, prof[dom][1])
    per_call_ms = prof[dom][0] / calls

    def bytes_of(stage, v, k, n):
        c = views[v]["cam"]
        T = ((c.W + 15) // 16) * ((c.H + 15) // 16)
        return algo_bytes(stage, P, n, k, c.W * c.H, T)

    design = dom + "_design" if dom == "render_bwd" else dom
    if batched and dom in ("render_fwd", "render_bwd"):
        ab = sum(bytes_of(dom, v, K[v], vis[v]) for v in range(len(views)))   # one launch covers all views
        db = sum(bytes_of(design, v, K[v], vis[v]) for v in range(len(views)))
        key, pairs = "batched." + dom, float(sum(K))
    else:
        ab = float(np.mean([bytes_of(dom, v, K[v], vis[v]) for v in range(len(views))]))
        db = float(np.mean([bytes_of(design, v, K[v], vis[v]) for v in range(len(views))]))
        key, pairs = ("batched." if batched else "") + dom, float(np.mean(K))
    peak, kind = measured_peak()
    achieved = ab / (per_call_ms / 1000.0) / 1e9
    traffic, traffic_src = ncu_traffic(key, pairs)
    issue = issue_roof(key, pairs, per_call_ms)
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_src,
            "algorithmic_bytes_per_launch": ab, "bytes_formula": "per view (render bwd: 40 K + 20 N + 44 V), summed over the views",
            "design_bytes_per_launch": db, "design_frac": db / (per_call_ms / 1000.0) / 1e9 / peak,
            "launch_ms": per_call_ms, "peak_source": f"{kind} (MEASURED_PEAKS.json hbm_gbs)" if kind == "measured"
            else "fallback 6650 GB/s",
            "timing": "CUDA events around each launch, eager pass of the same K steps" if batched
            else "CUDA events around each launch over the timed steps",
            "issue": issue,
            "note": "the compositing kernels are FP32/SFU issue-bound (exp per pixel-splat pair), not DRAM-bound: "
                    "`issue` is the same launch against the instruction-issue roof"}


def stages_of(prof):
    return {k: {"ms_total": v[0], "launch_groups": v[1], "ms_per_call": (v[0] / v[1]) if v[1] else 0.0}
            for k, v in prof.items() if v[1]}


# ---------------------------------------------------------------- LoD tree: filter + render (forward)
def make_lod(args, dev):
    """8M-node Gaussian tree (branching min(Poisson(3)+1, 8), depth <= 12, child scale x0.5) over the urban
    area, and a 1920x1080 camera at 150 m altitude, 45 deg pitch, looking at the first root's subtree."""
    from filtergs_b200 import lod, synthetic as S
    tr = S.lod_tree(P=args.lod_nodes, seed=1002, roots=2, max_depth=12, half_extent=500.0)
    c = tr["xyz"][tr["roots"][0]].astype(np.float64)   # aim at the first root's subtree
    c[2] = 0.0
    cam = S.look_at_camera(c + np.array([150.0, 0.0, 150.0]), c, W=1920, H=1080, fx=1600.0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    return tr, lod.TreeScene.from_arrays(tr, device=dev), cam, t(cam.viewmatrix), t(cam.projmatrix), t(cam.campos)


def measure_lod(args, dev, impl):
    """Views/s of per-view LoD selection + forward render.  Ours: the FilterGS rule (visibility kernel,
    ordered compaction, fused gather/activation, rasterizer) and the LoG cut rule (device traversal +
    culling).  Reference: its visibility kernel, torch.nonzero, torch activations, its rasterizer."""
    from filtergs_b200 import lod
    tr, scene, cam, view, proj, cpos = make_lod(args, dev)
    bg = torch.zeros(3, device=dev)
    steps = max(3, args.steps // 2)
    out = {"nodes": int(scene.P), "unit": "views/s", "width": cam.W, "height": cam.H,
           "rules": {"filtergs": "radius_max 1.5 px, padding 0.1, threshold 700",
                     "logcut": "min_resolution 1.5 px, cull < 1 px or opacity < 1/255"}}
    if impl == "ours":
        def filtergs(_):
            idx, cnt, *_r = lod.select_filtergs(scene, view, proj, cam, 1.5, 0.1, 700.0)
            return lod.render_selected(scene, idx, cnt, view, proj, cpos, cam, bg, stats=False), cnt

        def logcut(_):
            idx, cnt = lod.select_logcut(scene, view, proj, cam, 1.5, 1.0)
            return lod.render_selected(scene, idx, cnt, view, proj, cpos, cam, bg, stats=False), cnt

        for name, fn in (("filtergs", filtergs), ("logcut", logcut)):
            # the compositing launch shape for this view (small, dense splats favour 1 pixel per thread)
            tuned = autotune(args, fn, ("lod", name), 0)
            for i in range(3):
                r, cnt = fn(i)
            ms, _ = timed(fn, steps)
            out[name] = {"value": steps / (ms / 1000.0), "selected": int(cnt.item()), "pairs_K": int(r[0]),
                         "render_config": tuned}
    else:
        from oracle import build_ref
        ref, v2 = build_ref.load("ref_rasterizer_C"), build_ref.load("ref_compute_radius_v2")
        if ref is None or v2 is None:
            return {"unavailable": "reference build oracle/_ref missing"}
        fx, fy = cam.W / (2 * cam.tanfovx), cam.H / (2 * cam.tanfovy)
        e = torch.Tensor([])
        C0, C1 = 0.28209479177387814, 0.4886025119029199

        def filtergs(_):
            m, _r, _d = v2.compute_visibility_radius(scene.xyz, scene.log_scales, scene.rotations, proj, view,
                                                     scene.node_index, scene.ancestor_path, fx, fy, cam.tanfovx,
                                                     cam.tanfovy, 0.1, 1.5, 700.0)
            ri = torch.nonzero(m, as_tuple=True)[0]
            xyz = scene.xyz[ri]
            d = xyz - cpos[None]
            d = d / torch.norm(d, dim=-1, keepdim=True)
            rest = scene.shs_rest[ri]
            col = scene.features_dc[ri] * C0 + 0.5 + (-C1 * d[:, 1:2] * rest[:, 0] + C1 * d[:, 2:3] * rest[:, 1] -
                                                      C1 * d[:, 0:1] * rest[:, 2])
            r = ref.rasterize_gaussians(bg, xyz, col, torch.sigmoid(scene.opacity_raw[ri])[:, None],
                                        torch.exp(scene.log_scales[ri]),
                                        torch.nn.functional.normalize(scene.rotations[ri]), 1.0, e, view, proj,
                                        cam.tanfovx, cam.tanfovy, cam.H, cam.W, e, 0, cpos, False, True, False, 0.2,
                                        0.2, 0.05, 0.7, False)
            return r, ri.numel()

        for i in range(3):
            r, n = filtergs(i)
        ms, _ = timed(filtergs, steps)
        out["filtergs"] = {"value": steps / (ms / 1000.0), "selected": int(n), "pairs_K": int(r[0])}
    del scene
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------- training step (loss, backward, Adam)
def measure_train(args, dev):
    """ms per training iteration: 4M Gaussians (the urban generator on 2 km x 2 km with 1,200 buildings),
    4 views 1600x900 (altitude 80-300 m, pitch 30-75 deg), targets = renders of a perturbed copy (means
    + N(0, 0.05 m), SH DC + N(0, 0.1)), loss 0.8 L1 + 0.2 (1 - SSIM), backward, FP32 Adam on the visible
    Gaussians, densification statistics.  Batched (one CUDA graph per iteration) vs plain (one view per
    call)."""
    from filtergs_b200 import synthetic as S, train as TR
    from filtergs_b200.batched import Camera
    from filtergs_b200._C import rasterize_gaussians
    P = args.train_gaussians
    sc = S.urban_scene(P=P, seed=1004, half_extent=1000.0, buildings=1200)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    state_args = (t(sc["means3D"]), torch.log(t(sc["scales"])), t(sc["rotations"]),
                  torch.logit(t(sc["opacities"]).clamp(1e-6, 1 - 1e-6)), t(sc["shs"]))
    del sc
    rng = np.random.default_rng(5004)
    cams = []
    for _ in range(4):
        c = S.aerial_camera(rng, W=1600, H=900, fx=1600.0 * 1600 / 1920, altitude=float(rng.uniform(80, 300)),
                            pitch_deg=float(rng.uniform(30, 75)), xy_range=600.0)
        cams.append(Camera(c.W, c.H, c.tanfovx, c.tanfovy, t(c.viewmatrix), t(c.projmatrix), t(c.campos)))
    g = torch.Generator(device=dev).manual_seed(6004)
    pert = TR.TrainState(state_args[0] + 0.05 * torch.randn(P, 3, device=dev, generator=g), *state_args[1:4],
                         state_args[4] + torch.cat([0.1 * torch.randn(P, 1, 3, device=dev, generator=g),
                                                    torch.zeros(P, state_args[4].shape[1] - 1, 3, device=dev)], 1))
    e = torch.empty(0, device=dev)
    bg = torch.zeros(3, device=dev)
    targets = [rasterize_gaussians(bg, pert.xyz, e, pert.opac, pert.scale, pert.rot, 1.0, e, c.viewmatrix,
                                   c.projmatrix, c.tanfovx, c.tanfovy, c.H, c.W, pert.shs, 3, c.campos, False, True,
                                   False, 0.2, 0.2, 0.05, 0.7, False)[1].clone() for c in cams]
    del pert
    out = {"gaussians": P, "views_per_step": 4, "width": 1600, "height": 900, "unit": "ms/iteration",
           "loss": "0.8 L1 + 0.2 (1 - SSIM 11x11, sigma 1.5)", "optimizer": "FP32 Adam on visible Gaussians"}
    # the compositing launch shape for these views, tuned on a throwaway copy of the state (eager steps)
    st = TR.TrainState(*state_args)
    tune = TR.BatchedTrainer(st, cams, targets, bg=bg, graph=False)
    out["render_config"] = autotune(args, lambda i: tune.step(), ("train", P), 0)
    del tune, st
    torch.cuda.empty_cache()
    for name in ("batched", "plain"):
        st = TR.TrainState(*state_args)
        tr = TR.BatchedTrainer(st, cams, targets, bg=bg) if name == "batched" else TR.PlainTrainer(st, cams, targets,
                                                                                                     bg=bg)
        for _ in range(max(3, args.warmup)):
            tr.step()
        first = tr.loss.value()
        ms, _ = timed(lambda i: tr.step(), args.steps)
        if name == "batched":
            tr.check()
        out[name] = {"ms_per_iteration": ms / args.steps, "loss_after_warmup": first, "loss_last": tr.loss.value()}
        del tr, st
        torch.cuda.empty_cache()
    return out


def fp64_image_error(mod, dev):
    """Part of the CPU-baseline leg: the FP32 CUDA image of the CPU-runnable scene (10,000 Gaussians,
    256x256, SH 3, identity camera) against an FP64 evaluation of the same splat equations by the CPU
    port (it differs from the CUDA path only in precision)."""
    from oracle import oracle as O
    from filtergs_b200 import synthetic as S
    sc, cam = S.small_scene(P=10000, seed=1000)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    bg = torch.zeros(3, device=dev)
    e = torch.empty(0, device=dev)
    out = mod.rasterize_gaussians(bg, t(sc["means3D"]), e, t(sc["opacities"]), t(sc["scales"]), t(sc["rotations"]),
                                  1.0, e, t(cam.viewmatrix), t(cam.projmatrix), cam.tanfovx, cam.tanfovy, cam.H, cam.W,
                                  t(sc["shs"]), 3, t(cam.campos), False, True, False, 0.2, 0.2, 0.05, 0.7, False)
    img = out[1].cpu().numpy().astype(np.float64)
    f64 = lambda a: np.asarray(a, np.float64)  # noqa: E731
    s64 = O.Scene(f64(sc["means3D"]), f64(sc["opacities"]), cam.W, cam.H, cam.tanfovx, cam.tanfovy,
                  f64(cam.viewmatrix).reshape(-1), f64(cam.projmatrix).reshape(-1), f64(cam.campos),
                  shs=f64(sc["shs"]), sh_degree=3, scales=f64(sc["scales"]), rotations=f64(sc["rotations"]))
    ref = O.forward(s64, dtype=np.float64)["color"]
    d = np.abs(img - ref)
    return {"max_abs": float(d.max()), "mean_abs": float(d.mean()),
            "workload": "10,000 Gaussians SH3, 256x256 (CPU-runnable scene), FP32 CUDA vs FP64 CPU port"}


def main():
    args = parse()
    if args.only:
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        res = measure_lod(args, dev, args.impl) if args.only == "lod" else measure_train(args, dev)
        print(json.dumps({"workload": args.only, "impl": args.impl, **res}))
        return
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
    dev = torch.device("cuda", local)
    ref_dist = dist and args.impl != "reference"

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

    sc, scene = make_scene(args.P, dev)
    views = make_views(args.views, dev, rank, args.width, args.height)
    bg = torch.zeros(3, device=dev)
    nv = len(views)
    n_ranks = world if args.impl == "ours" else 1
    clocks = ClockSampler(local) if rank == 0 else None
    if clocks:
        clocks.start()
        clocks.wait_first()

    plain = mixed = None
    if args.impl == "reference":
        head = measure_plain(args, mod, scene, views, bg, dev, False, rank, ours=False, clocks=clocks)
        path = "plain"
    elif args.path == "batched":
        head = measure_batched(args, scene, views, bg, dev, ref_dist, rank, clocks=clocks)
        path = "batched"
    else:
        head = measure_plain(args, mod, scene, views, bg, dev, ref_dist, rank, clocks=clocks, profile=True)
        path = "plain"
    value = aggregate_views_per_s(n_ranks, nv, args.steps, head["ms"])

    e2e = None
    if not args.no_e2e:
        if path == "batched":
            e2e = e2e_batched(args, head["br"], views, dev, ref_dist, n_ranks)
        else:
            e2e = e2e_plain(args, mod, scene, views, bg, dev, ref_dist if args.impl == "ours" else False, n_ranks)
    if "br" in head:
        del head["br"]
        torch.cuda.empty_cache()
    if args.impl == "ours" and path == "batched" and not args.no_plain:
        plain = measure_plain(args, mod, scene, views, bg, dev, ref_dist, rank, clocks=clocks)
    if args.impl == "ours" and path == "batched" and not args.no_mixed:
        mv = make_views(args.views, dev, rank, mixed=True)
        mb = measure_batched(args, scene, mv, bg, dev, ref_dist, rank, clocks=clocks, profile=False)
        del mb["br"]
        torch.cuda.empty_cache()
        mp = measure_plain(args, mod, scene, mv, bg, dev, ref_dist, rank, clocks=clocks)
        mixed = {"resolutions": [f"{v['cam'].W}x{v['cam'].H}" for v in mv],
                 "batched_value": n_ranks * nv * args.steps / (mb["ms"] / 1000.0),
                 "plain_value": n_ranks * nv * args.steps / (mp["ms"] / 1000.0),
                 "unit": "views/s", "batched_render_config": mb["tuned"], "plain_render_config": mp["tuned"],
                 "batched_clocks": mb["clocks"], "plain_clocks": mp["clocks"],
                 "pairs_K": mb["K"], "visible_V": mb["vis"], "altitude_m": "80-300", "pitch_deg": "30-75"}
    lod_res = train_res = None
    if not args.no_lod and rank == 0:
        lod_res = measure_lod(args, dev, args.impl)
    if not args.no_train and rank == 0 and args.impl == "ours":
        train_res = measure_train(args, dev)
    if clocks:
        clocks.stop()

    if rank == 0:
        cfg = {"workload": f"urban-aerial {args.P / 1e6:g}M Gaussians SH3, {nv} cameras {args.width}x{args.height} "
                           f"per step, fwd+bwd, {path} path",
               "gaussians": args.P, "width": args.width, "height": args.height, "sh_degree": 3,
               "views_per_step": nv, "path": path,
               "l2": "inputs larger than L2 (472 MB Gaussian parameters read per view)",
               "pairs_K": head["K"], "visible_V": head["vis"], "mean_pairs_K": float(np.mean(head["K"])),
               "mean_visible_V": float(np.mean(head["vis"]))}
        if path == "plain":
            cfg["ogfs_enable_stats"] = bool(args.stats)
        res = {"metric": METRIC, "value": value, "unit": "views/s", "n_gpus": n_ranks, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": head["ms"] / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic (seeded urban-aerial scene and cameras)", "config": cfg}
        if args.impl == "reference":
            res["impl"] = "reference"
            res["cpu_baseline"] = {"value": value, "unit": "views/s", "cores": 1, "kind": "reference",
                                   "sample": "the reference's own rasterizer (CUDA sources compiled unmodified, "
                                             "oracle/_ref) on this GPU, one view per call; it has no CPU "
                                             "implementation of the path"}
            res["e2e"] = e2e or {"value": value, "unit": "views/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
        else:
            cfg["render_config"] = head["tuned"]
            res["roofline"] = roofline(head["prof"], args.P, views, head["K"], head["vis"], path == "batched")
            res["stages"] = stages_of(head["prof"])
            res["gpu_launches"] = int(head["launches"])
            if plain:
                res["plain"] = {"value": n_ranks * nv * args.steps / (plain["ms"] / 1000.0), "unit": "views/s",
                                "ms_per_step": plain["ms"] / args.steps, "render_config": plain["tuned"],
                                "clocks": plain["clocks"]}
                res["batched_over_plain"] = value / res["plain"]["value"]
            if mixed:
                res["mixed_resolution"] = mixed
            if e2e:
                res["e2e"] = e2e
            if not args.no_cpu_baseline:
                res["cpu_baseline"] = torch_cpu_baseline(sc, views[0]["cam"], os.cpu_count() or 1)
                res["cpu_baseline"]["c_port"] = cpu_baseline(sc, views[0]["cam"], os.cpu_count() or 1)
                res["cpu_baseline"]["fp64_image_error"] = fp64_image_error(mod, dev)
        if lod_res:
            res["lod_tree"] = lod_res
        if train_res:
            res["train_step"] = train_res
        if head["clocks"]:
            res["clocks"] = head["clocks"]
        print(json.dumps(res), flush=True)
    if dist:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


# ---------------------------------------------------------------- end to end through the public API
def e2e_plain(args, mod, scene, views, bg, dev, dist, n_ranks):
    """Plain path through the public API: per view, H2D of its camera and upstream gradient from
    pinned host memory, forward + backward, D2H of the rendered image.  The copies run on a side
    stream (view j+1's inputs upload while view j computes, view j's image downloads while its
    backward runs), as a pipelined caller would do; every view still moves its own bytes."""
    nv = len(views)
    host_cam = [torch.from_numpy(np.concatenate([v["cam"].viewmatrix.reshape(-1), v["cam"].projmatrix.reshape(-1),
                                                 v["cam"].campos]).astype(np.float32)).pin_memory() for v in views]
    out_host = [[torch.empty(3, v["cam"].H, v["cam"].W).pin_memory() for v in views] for _ in range(2)]
    dev_cam = [torch.empty(35, device=dev) for _ in range(2)]
    dev_dL = [[torch.empty(3, v["cam"].H, v["cam"].W, device=dev) for v in views] for _ in range(2)]
    copy = torch.cuda.Stream(device=dev)
    main = torch.cuda.current_stream(dev)
    ours = args.impl == "ours"
    if ours:
        from filtergs_b200.rasterization import GaussianRasterizationSettings, GaussianRasterizer
        params = [scene[k].clone().requires_grad_(True) for k in ("means3D", "shs", "opacities", "scales",
                                                                  "rotations")]
        m2 = torch.zeros_like(params[0], requires_grad=True)
    ready = [torch.cuda.Event() for _ in range(2)]
    freed = [torch.cuda.Event() for _ in range(2)]
    total = [0]

    def upload(j):
        b, v = j & 1, j % nv
        with torch.cuda.stream(copy):
            copy.wait_event(freed[b])
            dev_cam[b].copy_(host_cam[v], non_blocking=True)
            dev_dL[b][v].copy_(views[v]["dL_host"], non_blocking=True)
            ready[b].record(copy)

    def one(j):
        b, v = j & 1, j % nv
        c = views[v]["cam"]
        main.wait_event(ready[b])
        if j + 1 < total[0]:
            upload(j + 1)
        view, proj, cpos = dev_cam[b][:16].view(4, 4), dev_cam[b][16:32].view(4, 4), dev_cam[b][32:35]
        if ours:
            rs = GaussianRasterizationSettings(c.H, c.W, c.tanfovx, c.tanfovy, bg, 1.0, view, proj, 3, cpos, False,
                                               False, ogfs_enable_stats=bool(args.stats))
            for t in params + [m2]:
                t.grad = None
            means, shs, op, scl, rot = params
            color = GaussianRasterizer(rs)(means, m2, op, shs=shs, scales=scl, rotations=rot)[0]
        else:
            e = torch.empty(0, device=dev)
            out = mod.rasterize_gaussians(bg, scene["means3D"], e, scene["opacities"], scene["scales"],
                                          scene["rotations"], 1.0, e, view, proj, c.tanfovx, c.tanfovy, c.H, c.W,
                                          scene["shs"], 3, cpos, False, True, False, 0.2, 0.2, 0.05, 0.7, args.stats)
            K, color, pid, pwp, pw, radii, geom, binning, img, st = out
        img_done = torch.cuda.Event()
        img_done.record(main)
        with torch.cuda.stream(copy):
            copy.wait_event(img_done)
            out_host[b][v].copy_(color.detach(), non_blocking=True)
        if ours:
            color.backward(dev_dL[b][v])
        else:
            mod.rasterize_gaussians_backward(bg, scene["means3D"], radii, e, scene["scales"], scene["rotations"], 1.0,
                                             e, view, proj, c.tanfovx, c.tanfovy, dev_dL[b][v], scene["shs"], 3, cpos,
                                             geom, K, binning, img, False)
        freed[b].record(main)

    def run(nviews):
        total[0] = nviews
        upload(0)
        for j in range(nviews):
            one(j)

    run(args.warmup * nv)
    torch.cuda.synchronize()
    _barrier(dist)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    copy.wait_event(start)
    run(args.steps * nv)
    main.wait_stream(copy)      # the last image download is inside the timed region
    end.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(start.elapsed_time(end), dev, dist)
    px = sum(v["cam"].W * v["cam"].H for v in views)
    return {"value": n_ranks * args.steps * nv / (ms / 1000.0), "unit": "views/s",
            "h2d_bytes_per_step": int(nv * 35 * 4 + 3 * px * 4), "d2h_bytes_per_step": int(3 * px * 4),
            "api": "GaussianRasterizer (autograd)" if ours else "reference _C rasterize_gaussians(+_backward)",
            "d2h": "every rendered image; the Gaussian gradients stay on the device for the optimizer step"}


def e2e_batched(args, br, views, dev, dist, n_ranks):
    """Batched path through its public API (BatchedRasterizer): per step, H2D of all cameras and all
    upstream gradients from pinned host memory, the forward and backward graph replays, D2H of every
    rendered image.  Images and gradients are double-buffered (set_io_many re-targets the captured
    graphs) and copied on two copy streams: a step's images download while its backward runs, the
    next step's gradients upload while this step computes."""
    nv = len(views)
    cam_host = torch.from_numpy(np.stack([np.concatenate([v["cam"].viewmatrix.reshape(-1),
                                                          v["cam"].projmatrix.reshape(-1), v["cam"].campos])
                                          for v in views]).astype(np.float32)).pin_memory()
    cam_stage = [torch.empty(nv, 35, device=dev) for _ in range(2)]
    imgs = [[torch.empty(3, v["cam"].H, v["cam"].W, device=dev) for v in views] for _ in range(2)]
    dls = [[torch.empty(3, v["cam"].H, v["cam"].W, device=dev) for v in views] for _ in range(2)]
    out_host = [[torch.empty(3, v["cam"].H, v["cam"].W).pin_memory() for v in views] for _ in range(2)]
    h2d, d2h = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    main = torch.cuda.current_stream(dev)
    cam_ready = [torch.cuda.Event() for _ in range(2)]
    ready = [torch.cuda.Event() for _ in range(2)]
    freed = [torch.cuda.Event() for _ in range(2)]
    rendered = [torch.cuda.Event() for _ in range(2)]
    downloaded = [torch.cuda.Event() for _ in range(2)]
    ids = list(range(nv))
    total = [0]

    def upload(i):
        b = i & 1
        with torch.cuda.stream(h2d):
            h2d.wait_event(freed[b])
            cam_stage[b].copy_(cam_host, non_blocking=True)
            cam_ready[b].record(h2d)
            for v in range(nv):
                dls[b][v].copy_(views[v]["dL_host"], non_blocking=True)
            ready[b].record(h2d)

    def one(i):
        # the forward needs only the cameras; the upstream gradients' upload overlaps it and
        # the backward waits for it; the images download while the backward runs
        b = i & 1
        main.wait_event(cam_ready[b])
        main.wait_event(downloaded[b])
        br.cam_dev.copy_(cam_stage[b])      # the captured kernels read the cameras from these rows
        br.set_io_many(ids, imgs[b], dls[b])
        br.step(forward_done=rendered[b], backward_ready=ready[b])
        freed[b].record(main)
        if i + 1 < total[0]:
            upload(i + 1)
        with torch.cuda.stream(d2h):
            d2h.wait_event(rendered[b])
            for v in range(nv):
                out_host[b][v].copy_(imgs[b][v], non_blocking=True)
            downloaded[b].record(d2h)

    def run(n):
        total[0] = n
        upload(0)
        for i in range(n):
            one(i)

    run(args.warmup)
    torch.cuda.synchronize()
    _barrier(dist)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    h2d.wait_event(start)
    d2h.wait_event(start)
    run(args.steps)
    main.wait_stream(d2h)       # the last downloads are inside the timed region
    end.record()
    torch.cuda.synchronize()
    br.check()
    ms = max_over_ranks(start.elapsed_time(end), dev, dist)
    px = sum(v["cam"].W * v["cam"].H for v in views)
    return {"value": n_ranks * args.steps * nv / (ms / 1000.0), "unit": "views/s",
            "h2d_bytes_per_step": int(nv * 35 * 4 + 3 * px * 4), "d2h_bytes_per_step": int(3 * px * 4),
            "api": "BatchedRasterizer.step (forward and backward graph replays)",
            "overlap": "per step 16 camera rows and 16 upstream gradients uploaded and 16 images downloaded "
                       "(the bytes above), on two copy streams: a step's images download while its backward "
                       "runs, the next step's uploads run during this step; the last step's downloads end "
                       "inside the timed region",
            "d2h": "every rendered image; the summed Gaussian gradients stay on the device for the optimizer "
                   "step (as in the reference's training loop), as they do in the reference arm"}


if __name__ == "__main__":
    main()
