"""Benchmark: primary-ray throughput of the Gaussian ray tracer.

Workload (default): 1,000,000 Gaussians in 64 clusters, one 1920x1080 view,
k = 16, alpha_min = 0.01, T_min = 0.01, SH degree 3, camera at radius 12 (the
configuration the headline metric is quoted on).  A step is one render of
that view.  Scene data lives in HBM (~360 MB, larger than the 126 MB L2, so
no explicit L2 flush is done between steps).

Our arm prints one JSON line with
  value          Mrays/s of the trace kernel launches, inputs resident on the
                 device, timed with CUDA events on the library's stream
  e2e            Mrays/s through gt_render with a host (pinned) output buffer,
                 the device-to-host copy of every image inside the wall-clock
                 timed region
  roofline       algorithmic bytes per launch (16 B per pixel + 44 B per
                 composited entry + 192 B of SH per contributing entry) over
                 the average trace-kernel time, against the measured HBM peak
  cpu_baseline   the CPU restatement of the reference algorithm (oracle,
                 per-round k-buffer traversal), all host threads, on a
                 stratified pixel subset

``--impl reference`` times only that CPU restatement (the reference itself is
a browser WebGPU application and cannot run here).

Multi-GPU: ``torchrun --nproc-per-node N bench.py --gpus N``; every rank
renders the same workload on its own GPU (replicas; the path has no
exchange), value = total rays of all ranks over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "webgpu-gaussiantracer_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "Mrays/s at 1080p/1M Gaussians, batched vs plain; fwd+bwd ms/view; HBM GB/s"


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def init_ranks():
    """One process per GPU (torchrun): rank, world size, local rank and the
    gloo process group used for the barrier and the max over ranks (the path
    has no data exchange).  The short timeout ends a run whose ranks wait on a
    rank that never arrives."""
    import datetime
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    return rank, world, local, dist


def max_over_ranks(dist, x: float) -> float:
    """The largest value of x over all ranks (x itself without a process group)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_mrays(world: int, rays_per_rank: int, slowest_s: float) -> float:
    """Mrays/s of the whole job: every rank traces the same view (replicas),
    the job takes as long as its slowest rank."""
    return world * rays_per_rank / slowest_s / 1e6


def make_workload(name: str):
    from gtrace import synth
    if name == "clusters-1m-1080p":
        pg, amin, v = synth.clusters_1m_config()
        desc = "1M Gaussians (64 clusters), 1920x1080, k=16, alpha_min=0.01, T_min=0.01, SH3, camera radius 12"
    elif name == "clusters-1m-480x270":
        pg, amin, v = synth.clusters_1m_config()
        v = synth.view(480, 270, (0.0, 0.0, 12.0), k=16)
        desc = "1M Gaussians (64 clusters), 480x270 (profiling size), k=16, alpha_min=0.01, T_min=0.01, SH3"
    elif name == "clusters-1m-960x540":
        pg, amin, v = synth.clusters_1m_config()
        v = synth.view(960, 540, (0.0, 0.0, 12.0), k=16)
        desc = ("1M Gaussians (64 clusters), 960x540 (profiling size of the tile-packet kernel), k=16, "
                "alpha_min=0.01, T_min=0.01, SH3")
    elif name == "small-256":
        pg, amin, v = synth.small_config()
        desc = "16,384 Gaussians (uniform), 256x256, k=6, alpha_min=0.01, T_min=0.01, SH3, camera at distance 4"
    elif name == "clusters-200k-800":
        raw, amin, v = synth.clusters_200k_config()
        pg = synth.pack(raw)
        desc = "200k Gaussians (64 clusters), 800x800, k=8, alpha_min=0.01, T_min=0.01, SH3, camera radius 12"
    else:
        raise SystemExit(f"unknown workload {name}")
    return pg, amin, v, desc


def cpu_port_throughput(pg, amin, v, budget_s: float, threads: int = 0, scene=None):
    """Times the CPU restatement of the reference algorithm (oracle, per-round
    k-buffer traversal) on stratified pixel subsets; returns Mrays/s and the
    sample description.  Scene preparation (skipped when `scene` is given) is
    not timed."""
    from oracle import oracle
    t0 = time.perf_counter()
    s = scene if scene is not None else oracle.Scene(pg.gaussiansBuffer, amin, "f32")
    prep = time.perf_counter() - t0
    w, h = v.width, v.height
    stride = 8
    while True:
        xs = np.arange(stride // 2, w, stride)
        ys = np.arange(stride // 2, h, stride)
        pix = (ys[:, None] * w + xs[None, :]).reshape(-1).astype(np.uint32)
        t = time.perf_counter()
        s.render(v.uniforms, w, h, pixels=pix, algo=1, threads=threads)
        dt = time.perf_counter() - t
        if dt >= 0.5 * budget_s or stride <= 1:
            break
        stride = max(1, int(stride / math.sqrt(max(2.0, 0.6 * budget_s / max(dt, 1e-3)))))
    return len(pix) / dt / 1e6, len(pix), stride, dt, prep


def _time_device(ctx, fn, reps: int):
    """Device time (CUDA events on the library stream) of reps calls of fn."""
    ctx.synchronize()
    ctx.timer_start()
    for _ in range(reps):
        fn()
    return ctx.timer_stop() / reps


def _time_device_median(ctx, fn, reps: int):
    """Median over reps calls of fn of each call's device time (CUDA events on
    the library stream around the call): a step of host-synchronous calls
    (forward, loss, adjoint) is timed one at a time, so that one slow host
    turn-around does not stand for the rest."""
    ts = []
    for _ in range(reps):
        ctx.synchronize()
        ctx.timer_start()
        fn()
        ts.append(ctx.timer_stop())
    return statistics.median(ts)


def extra_batched(ctx, reps: int = 2):
    """8 scenes (100k-1M Gaussians, log-uniform), 64 views of uneven size: one
    batched launch against the 64 views rendered one by one."""
    from gtrace import synth
    from gtrace.tracer import Scene
    raw_scenes, views = synth.batched_scenes_config()
    scenes = [Scene(ctx, synth.pack(raw).gaussiansBuffer, amin) for raw, amin in raw_scenes]
    amins = [amin for _, amin in raw_scenes]
    items, bufs = [], []
    rays = 0
    for s, w, h, pos in views:
        v = synth.view(w, h, pos, k=16, alpha_min=amins[s])
        ptr = ctx.device_alloc(w * h * 16)
        bufs.append(ptr)
        items.append((scenes[s], v.uniforms, w, h, ptr))
        rays += w * h
    batched = lambda: ctx.render_batch(items, device_outputs=True, asynchronous=True)  # noqa: E731
    def plain():
        for sc, u, w, h, ptr in items:
            ctx.render_device(sc, u, w, h, ptr, asynchronous=True)
    batched()
    plain()
    tdef = _time_device(ctx, batched, reps)  # the default shape
    # the batch tuner picks k-buffer, hand-off and kernel for this batch shape;
    # render_batch then uses its choice
    tune = ctx.autotune_batch([(sc, u, w, h) for sc, u, w, h, _ in items])
    batched()
    tb = _time_device(ctx, batched, reps)
    tp = _time_device(ctx, plain, reps)
    for ptr in bufs:
        ctx.device_free(ptr)
    n_total = sum(s.n for s in scenes)
    for s in scenes:
        s.close()
    return {"workload": f"8 scenes ({n_total} Gaussians in all, 100k-1M each, 64 clusters), 64 views 320-1920 x "
                        "240-1080, k=16, alpha_min per scene in {0.01, 0.05, 0.1}, camera radius 8-14",
            "rays": rays, "batched_ms": tb, "plain_ms": tp, "batched_mrays": rays / tb / 1e3,
            "plain_mrays": rays / tp / 1e3, "default_shape_ms": tdef,
            "shape": {"kernel": "tile packets" if tune["block_threads"] == 32 else "warp per ray",
                      "kbuf": tune["kbuf"], "handoff_after": tune["handoff_after"],
                      "blocks_per_sm": tune["blocks_per_sm"], "tile": "8x4", "stack": 256},
            "tuner_default_ms": tune["default_ms"], "tuner_best_ms": tune["best_ms"]}


def _train_step_single(ctx, scene, v, img, tgt, dl, gout):
    ctx.render_device(scene, v.uniforms, v.width, v.height, img, checkpoint=True)
    ctx.l2_loss(img, tgt, v.width * v.height, dl)
    return ctx.backward_device(scene, v.uniforms, v.width, v.height, dl, gout, reuse_checkpoint=True)


def extra_fwd_bwd(ctx, reps: int = 9):
    """200k Gaussians, 800x800, k=8, L2 loss against a render of the perturbed
    scene: plain forward vs forward + loss + backward."""
    from gtrace import synth
    from gtrace.tracer import Scene
    raw, amin, v = synth.clusters_200k_config()
    scene = Scene(ctx, synth.pack(raw).gaussiansBuffer, amin)
    target = Scene(ctx, synth.pack(synth.perturb(raw, synth.SEED_BASE + 33)).gaussiansBuffer, amin)
    px = v.width * v.height
    img, tgt, dl = ctx.device_alloc(px * 16), ctx.device_alloc(px * 16), ctx.device_alloc(px * 16)
    gout = ctx.device_alloc(59 * scene.n * 4)
    ctx.render_device(target, v.uniforms, v.width, v.height, tgt)
    fwd = lambda: ctx.render_device(scene, v.uniforms, v.width, v.height, img, asynchronous=True)  # noqa: E731
    info = {}
    def step():
        info.update(_train_step_single(ctx, scene, v, img, tgt, dl, gout))
    ckpt = lambda: ctx.render_device(scene, v.uniforms, v.width, v.height, img, checkpoint=True)  # noqa: E731
    fwd()
    step()
    tf = _time_device_median(ctx, fwd, reps)
    tfb = _time_device_median(ctx, step, reps)
    tck = _time_device_median(ctx, ckpt, reps)
    for p in (img, tgt, dl, gout):
        ctx.device_free(p)
    scene.close()
    target.close()
    return {"workload": "200k Gaussians (64 clusters), 800x800, k=8, alpha_min=0.01, L2 loss vs perturbed scene",
            "fwd_ms": tf, "fwd_bwd_ms": tfb, "ratio": tfb / tf, "adjoint_ms": info.get("bwd_ms"),
            "checkpoint_fwd_ms": tck, "mode": "checkpoint" if info.get("used_mode") == 1 else "replay"}


def extra_batched_fwd_bwd(ctx, pg, amin, reps: int = 1, n_views: int = 32):
    """32 views (640x480 - 1920x1080) of the 1M scene: batched forward with
    checkpoint + per-view L2 loss + one batched adjoint accumulating all views,
    against 32 plain forwards one by one (n_views: the first n of the 32)."""
    import ctypes as C
    from gtrace import _lib as L
    from gtrace import synth
    from gtrace.tracer import Scene, _uniforms
    scene = Scene(ctx, pg.gaussiansBuffer, amin)
    target_raw = synth.perturb(synth.raw_clusters(1_000_000, synth.SEED_BASE + 1), synth.SEED_BASE + 44)
    target = Scene(ctx, synth.pack(target_raw).gaussiansBuffer, amin)
    views = synth.batched_fwd_bwd_views(n_views)
    imgs = [ctx.device_alloc(v.width * v.height * 16) for v in views]
    tgts = [ctx.device_alloc(v.width * v.height * 16) for v in views]
    dls = [ctx.device_alloc(v.width * v.height * 16) for v in views]
    gout = ctx.device_alloc(59 * scene.n * 4)
    for v, t in zip(views, tgts):
        ctx.render_device(target, v.uniforms, v.width, v.height, t)
    items = [(scene, v.uniforms, v.width, v.height, p) for v, p in zip(views, imgs)]
    lib = ctx._lib
    bitems = (L.BatchItem * len(views))()
    for i, v in enumerate(views):
        bitems[i].scene = scene.handle
        bitems[i].u = _uniforms(v.uniforms)
        bitems[i].w, bitems[i].h = v.width, v.height
        bitems[i].out_rgba = None
        bitems[i].dL_drgba = dls[i]
    sc = (C.c_void_p * 1)(scene.handle.value)
    op = (C.c_void_p * 1)(gout)
    rays = sum(v.width * v.height for v in views)
    its = (L.BatchItem * len(views))()
    for i, (s_, u_, w_, h_, p_) in enumerate(items):
        its[i].scene = s_.handle
        its[i].u = _uniforms(u_)
        its[i].w, its[i].h = w_, h_
        its[i].out_rgba = p_

    info = {}

    def step():
        flags = L.GT_FLAG_OUTPUT_DEVICE | L.GT_FLAG_CHECKPOINT
        ctx.check(lib.gt_render_batch(ctx.handle, its, len(views), flags, None))
        for v, i_, t_, d_ in zip(views, imgs, tgts, dls):
            ctx.l2_loss(i_, t_, v.width * v.height, d_)
        opts = L.BwdOpts(0, 0, 0, 0, 0, 0.0, 0.0)
        ctx.check(lib.gt_backward_batch(ctx.handle, bitems, len(views), sc, op, 1,
                                        L.GT_FLAG_INPUT_DEVICE | L.GT_FLAG_OUTPUT_DEVICE | L.GT_FLAG_CHECKPOINT,
                                        C.byref(opts), None))
        info.update(used_mode=opts.used_mode, bwd_ms=opts.bwd_ms)

    def fwd_ckpt():
        flags = L.GT_FLAG_OUTPUT_DEVICE | L.GT_FLAG_CHECKPOINT
        ctx.check(lib.gt_render_batch(ctx.handle, its, len(views), flags, None))
    def plain():
        for s_, u_, w_, h_, p_ in items:
            ctx.render_device(s_, u_, w_, h_, p_, asynchronous=True)
    tune = ctx.autotune_batch([(s_, u_, w_, h_) for s_, u_, w_, h_, _ in items])
    step()
    step()  # the second call sizes the checkpoint pool from the first one's count
    plain()
    tfb = _time_device(ctx, step, reps)
    tp = _time_device(ctx, plain, reps)
    tfc = _time_device(ctx, fwd_ckpt, reps)
    for p in imgs + tgts + dls + [gout]:
        ctx.device_free(p)
    scene.close()
    target.close()
    return {"workload": f"1M Gaussians (64 clusters), {len(views)} views 640x480-1920x1080, k=16, "
                        "L2 loss vs perturbed scene",
            "rays": rays, "batched_fwd_bwd_ms": tfb, "plain_fwd_ms": tp, "ratio": tfb / tp,
            "checkpoint_fwd_ms": tfc, "adjoint_ms": info.get("bwd_ms"),
            "shape": {"kernel": "tile packets" if tune["block_threads"] == 32 else "warp per ray",
                      "kbuf": tune["kbuf"], "handoff_after": tune["handoff_after"]},
            "mode": "checkpoint" if info.get("used_mode") == 1 else "replay"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="clusters-1m-1080p")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU baseline work")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-step-budget", type=float, default=0.0,
                    help="--impl reference: seconds of CPU work per step (0: 60 s spread over the steps)")
    ap.add_argument("--shape", default=None,
                    help="packets:KBUF:HANDOFF_AFTER or warp:KBUF: this launch shape instead of the tuner's")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched and forward+backward measurements")
    ap.add_argument("--extra", choices=["fwd_bwd", "batched", "batched_fwd_bwd"], default=None,
                    help="run only this extra measurement (one GPU) and print its result as the line")
    ap.add_argument("--views", type=int, default=32, help="--extra batched_fwd_bwd: views of the batch")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank, world, local, dist = init_ranks()

    pg, amin, v, desc = make_workload(args.workload)
    w, h = v.width, v.height
    rays = w * h
    threads = os.cpu_count() or 1

    if args.extra:
        # one extra measurement on its own (the profiling runs); rank 0 only
        if rank == 0:
            from gtrace.tracer import Context
            ctx = Context(local)
            fn = {"fwd_bwd": lambda: extra_fwd_bwd(ctx), "batched": lambda: extra_batched(ctx),
                  "batched_fwd_bwd": lambda: extra_batched_fwd_bwd(ctx, pg, amin, n_views=args.views)}[args.extra]
            with ClockSampler(local) as eclk:
                res = fn()
            res["clocks"] = eclk.summary()
            print(json.dumps({"extra": args.extra, **res}), flush=True)
        if dist:
            dist.destroy_process_group()
        return

    if args.impl == "reference":
        if rank != 0:
            if dist:
                dist.destroy_process_group()
            return
        from oracle import oracle
        ref_scene = oracle.Scene(pg.gaussiansBuffer, amin, "f32")
        # the pixel sample is sized once (about `budget` seconds of CPU work);
        # every warm-up and timed step then traces that same sample
        budget = args.ref_step_budget if args.ref_step_budget > 0 else max(2.0, 60.0 / (args.steps + 3))
        _, n_px, stride, _, _ = cpu_port_throughput(pg, amin, v, budget_s=budget, scene=ref_scene)
        xs = np.arange(stride // 2, w, stride)
        ys = np.arange(stride // 2, h, stride)
        pix = (ys[:, None] * w + xs[None, :]).reshape(-1).astype(np.uint32)
        sample = f"{n_px} pixels (every {stride}th pixel in x and y) of the {w}x{h} view"
        vals, step_s = [], []
        for i in range(args.warmup + args.steps):
            t = time.perf_counter()
            ref_scene.render(v.uniforms, w, h, pixels=pix, algo=1)
            dt = time.perf_counter() - t
            if i >= args.warmup:
                vals.append(n_px / dt / 1e6)
                step_s.append(dt)
        val = statistics.median(vals)
        # a step is the timed pixel sample (wall clock); the full frame at that
        # rate is reported beside it, not as the step time
        line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "Mrays/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.median(step_s) * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded)",
                "config": {"workload": desc, "width": w, "height": h,
                           "step": f"{n_px} rays of the view (a stratified pixel sample), timed on the host cores",
                           "rays_per_step": n_px,
                           "full_frame_ms_at_this_rate": rays / (val * 1e6) * 1e3},
                "cpu_baseline": {"value": val, "unit": "Mrays/s", "cores": threads, "kind": "port",
                                 "sample": sample + "; CPU restatement of the reference traversal (oracle algo 1); "
                                           "the reference runs only as a browser WebGPU app"},
                "e2e": {"value": val, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        if dist:
            dist.destroy_process_group()
        return

    from gtrace.tracer import Context, Scene
    ctx = Context(local)
    t_sc = time.perf_counter()
    scene = Scene(ctx, pg.gaussiansBuffer, amin)
    scene_wall_ms = (time.perf_counter() - t_sc) * 1e3
    info = scene.info()
    # the scene built again in its place (as a training loop rebuilds it): the
    # steady cost once the context holds its kernels, memory pool and pinned
    # upload chunks; this copy is the one rendered
    scene.close()
    t_sc = time.perf_counter()
    scene = Scene(ctx, pg.gaussiansBuffer, amin)
    warm_wall_ms = (time.perf_counter() - t_sc) * 1e3
    warm_info = scene.info()
    out_dev = ctx.device_alloc(rays * 16)
    # the launch shape for this view from the library's tuner (gt_autotune:
    # k-buffer size and hand-off point of the tile packets, blocks, k-buffer
    # and leaf batch of the warp-per-ray kernel), cached by the context and
    # used by every render below
    # (--shape installs a given shape instead, without the tuner's launches:
    # the profiling commands use it so that their launch lists hold renders)
    if args.shape:
        kind, kb, ha = (args.shape.split(":") + ["0", "0"])[:3]
        bt = 32 if kind == "packets" else 128
        ctx.set_tune(scene, v.uniforms, w, h, block_threads=bt, kbuf=int(kb) or (32 if bt == 32 else 64),
                     handoff_after=int(ha), blocks_per_sm=8)
        tune = {"block_threads": bt, "kbuf": int(kb), "handoff_after": int(ha), "blocks_per_sm": 8,
                "best_ms": None, "default_ms": None}
    else:
        tune = ctx.autotune(scene, v.uniforms, w, h)
    shape = {"kernel": "tile packets" if tune["block_threads"] == 32 else "warp per ray", "kbuf": tune["kbuf"],
             "handoff_after": tune["handoff_after"] if tune["block_threads"] == 32 else None,
             "blocks_per_sm": tune["blocks_per_sm"] if tune["block_threads"] == 128 else None,
             "tuned_ms": tune["best_ms"], "default_shape_ms": tune["default_ms"],
             "source": "--shape " + args.shape if args.shape else "gt_autotune"}
    # one synchronous render: counters for the algorithmic byte count
    st0 = ctx.render_device(scene, v.uniforms, w, h, out_dev)
    alg_bytes = 16 * st0["rays"] + 44 * st0["entries"] + 192 * st0["contributing"]
    for _ in range(args.warmup):
        ctx.render_device(scene, v.uniforms, w, h, out_dev, asynchronous=True)
    ctx.synchronize()
    ctx.kernel_times()
    if dist:
        dist.barrier()
    n_launch0 = ctx.launch_count()
    with ClockSampler(local) as clk:
        ctx.synchronize()
        ctx.timer_start()
        for _ in range(args.steps):
            ctx.render_device(scene, v.uniforms, w, h, out_dev, asynchronous=True)
        ms = ctx.timer_stop()
    n_launch = ctx.launch_count() - n_launch0
    ktimes = ctx.kernel_times()
    ms_step = max_over_ranks(dist, ms / args.steps)
    value = whole_job_mrays(world, rays, ms_step * 1e-3)

    # end to end: host output buffer (pinned), copy inside the timed region
    host = ctx.host_alloc(rays * 16, np.float32, (h, w, 4))
    for _ in range(2):
        ctx.render(scene, v.uniforms, w, h, out=host)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ctx.render(scene, v.uniforms, w, h, out=host)
    e2e_s = max_over_ranks(dist, (time.perf_counter() - t0) / args.steps)
    e2e = whole_job_mrays(world, rays, e2e_s)
    checksum = float(np.float64(host[..., :3]).sum())
    ctx.host_free(host)
    ctx.device_free(out_dev)

    peak, peak_kind = load_peaks()
    clocks = clk_summary = clk.summary()
    k_ms = statistics.mean(ktimes) if ktimes else ms_step
    achieved = alg_bytes / (k_ms * 1e-3) / 1e9
    # per-render DRAM traffic, warp instructions and L2 hit rate of the trace
    # launches from the committed ncu summary of this workload
    prof = {}
    tpath = os.path.join(ROOT, "profiles", "trace_profile.json")
    if os.path.exists(tpath):
        try:
            prof = json.load(open(tpath)).get(args.workload, {}) or {}
        except Exception:
            prof = {}
    traffic = prof.get("dram_bytes_per_render")
    issue = None
    dev = ctx.device_attributes()
    if prof.get("warp_inst_per_render"):
        mhz = clk_summary["sm_mhz"] or dev["max_sm_mhz"]
        slots = dev["sm_count"] * 4 * mhz * 1e6 * k_ms * 1e-3  # 4 schedulers an SM, one issue a clock each
        issue = {"bound": "issue", "achieved_warp_inst": prof["warp_inst_per_render"], "slots": slots,
                 "frac": prof["warp_inst_per_render"] / slots, "sm_count": dev["sm_count"], "sm_mhz": mhz,
                 "source": prof.get("source")}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        mr, n, stride, dt, prep = cpu_port_throughput(pg, amin, v, budget_s=args.cpu_budget)
        cpu = {"value": mr, "unit": "Mrays/s", "cores": threads, "kind": "port",
               "sample": f"{n} pixels (every {stride}th pixel in x and y) of the {w}x{h} view, {dt:.1f} s; "
                         f"CPU restatement of the reference traversal"}
    extras = None
    if rank == 0 and world == 1 and not args.no_extras and args.workload == "clusters-1m-1080p":
        extras = {}
        for name, fn in (("fwd_bwd", lambda: extra_fwd_bwd(ctx)), ("batched", lambda: extra_batched(ctx)),
                         ("batched_fwd_bwd", lambda: extra_batched_fwd_bwd(ctx, pg, amin))):
            with ClockSampler(local) as eclk:
                extras[name] = fn()
            extras[name]["clocks"] = eclk.summary()
    line = {"metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, no dataset)",
            "config": {"workload": desc, "width": w, "height": h, "n_gaussians": int(info["n_particles"]),
                       "n_proxies": int(info["n_kept"]), "k": 16 if "1m" in args.workload else None,
                       # a scene created on a context that has built one before (kernels
                       # loaded, memory pool and pinned upload chunks in place); the
                       # process's first creation beside it
                       "scene_build_ms": warm_info["build_ms"], "scene_upload_ms": warm_info["upload_ms"],
                       "scene_create_wall_ms": warm_wall_ms,
                       "scene_first_create": {"build_ms": info["build_ms"], "upload_ms": info["upload_ms"],
                                              "create_wall_ms": scene_wall_ms},
                       "bvh_depth": info["bvh_depth"], "shape": shape,
                       "l2": "inputs larger than L2 (scene %.0f MB > 126 MB), no flush" % (info["device_bytes"] / 1e6),
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "alg_bytes_per_launch": alg_bytes, "kernel_ms": k_ms,
                         "l2_hit_pct": prof.get("l2_hit_pct"), "l2_hit_source": prof.get("l2_hit_source"),
                         "issue": issue,
                         # warp execution efficiency: active lanes per warp instruction of the
                         # tile-packet kernel (a full ncu capture of the 960x540 case)
                         "warp_exec_eff": ({"lanes_per_inst": prof["lanes_per_inst"],
                                            "frac": prof["lanes_per_inst"] / 32.0,
                                            "source": prof.get("lanes_source")}
                                           if prof.get("lanes_per_inst") else None),
                         "timed": "a render's trace launches (large views: the tile-packet kernel and the "
                                  "warp-per-ray launch that finishes the rays it hands over)"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "Mrays/s", "h2d_bytes_per_step": 112 + 256,
                    "d2h_bytes_per_step": rays * 16},
            "gpu_launches": n_launch, "clocks": clocks,
            "counters": {k2: st0[k2] for k2 in ("rounds", "entries", "contributing", "proxy_tests", "node_visits",
                                                 "anyhits")},
            "image_checksum": checksum, "extras": extras}
    if rank == 0:
        print(json.dumps(line), flush=True)
    scene.close()
    ctx.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
