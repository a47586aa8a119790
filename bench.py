"""Benchmark: one frame of the surfel-radiosity path on the product-scale scene.

A step is one frame on fixed surfels: transfer build (clusters, candidate
pairs, visibility, closure, CSR) -> direct light on surfels -> Jacobi solve
-> gather grid -> per-pixel shade with the sRGB encode, i.e. the stages the
reference runs after surfel generation (main.rs:448-475 and 522-534). Surfel
generation runs once before timing and is reported separately.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2_product|c2_product_strict|c1_cornell|c3_stress|c4_batch|
                                c4_multi|c5_diff|solve_hbm|pathtrace]
                    [--no-cpu-baseline] [--film WxH] [--surfels N]

`c2_product` (the default) times one `ifx_frame` call per step; `--film` and
`--surfels` shrink a workload for profiling or for a CPU comparison the
oracle can finish.

N > 1 runs under torchrun as N independent replicas (one process per GPU,
each rendering its own frame; the path has no cross-GPU exchange), timed on
the device and reduced as the max over ranks. `--impl reference` times the
reference algorithm's CPU implementation (the oracle restatement in oracle/,
since the Rust reference cannot be built here) on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (scene file, description)
    "c2_product": ("interflect_b200/scenes/c2_product.rad",
                   "product scale: 5 objects + floor plane, quad + sphere light, 1920x1080, 200k surfels requested, "
                   "16 bounces"),
    "c2_product_strict": ("interflect_b200/scenes/c2_product_strict.rad",
                          "product scale, reference features only"),
    "c1_cornell": ("interflect_b200/scenes/c1_cornell.rad", "Cornell box 260x260, 20k surfels, 12 bounces"),
    "c3_stress": ("interflect_b200/scenes/c3_stress.rad",
                  "512 primitives, 3840x2160, 1M surfels requested, 24 bounces"),
    "c4_batch": ("interflect_b200/scenes/c1_cornell.rad",
                 "256 relighting right-hand sides (1-4 surfels-as-lights, intensity U[1,50]) on the Cornell "
                 "transfer, one CSR SpMM solve, 12 bounces max"),
    "c4_multi": ("interflect_b200/scenes/gen_scenes.py:packed_scenes",
                 "64 stress-style scenes (8-128 primitives, 2k-50k surfels, 256^2-1024^2 films, 24 bounces max) "
                 "solved and shaded in one persistent cooperative launch replayed from a CUDA graph"),
    "solve_hbm": ("interflect_b200/scenes/c3_stress.rad",
                  "Jacobi solve alone on a stress-sized transfer: the stress scene's 1M surfels and clusters with "
                  "a synthetic CSR of 109 links per row (109M links), 24 bounces max; the HBM-bound stage"),
    "pathtrace": ("tests/golden/scenes/bench_cornell.rad",
                  "the path-traced ground truth of the accuracy benchmark: Lambertian Cornell box, 300x300, 512 "
                  "samples per pixel (bench.sh defaults)"),
    "c5_diff": ("interflect_b200/scenes/c5_cornell_fill.rad",
                "Cornell box 512x512 with a second (fill) light, 20k surfels, 12 fixed bounces; L2 loss against a "
                "target rendered from per-surfel albedo + N(0,0.05) clamped to [0.05,0.95]; gradient w.r.t. "
                "per-surfel albedo and both light emissions"),
}
PT_METRIC = "path-traced samples per second (--mode reference, 12-vertex paths with next-event estimation)"
PT_FILM, PT_SPP, PT_CPU_ROWS = 300, 512, 16
DIFF_METRIC = "albedo+emission gradient ms (differentiable forward + adjoint) vs one forward frame"
BATCH_METRIC = "relighting solves per second (256 right-hand sides on one transfer matrix)"
METRIC = "SDF evaluations per second, one full frame (transfer + light + solve + grid + shade)"
# Kernels with per-launch CUDA-event times and work counters (the ray-marching
# kernels, plus the shade stage's setup/compose kernels as one group).
KERNEL_NAMES = ("visibility", "closure", "light", "primary", "shadow", "reflect", "shadow2", "shade_other")
UNIT = "evals/s"
FP32_LANES_PER_SM = 128
N_SMS = 148


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


def fp32_peak_tflops(peaks: dict) -> tuple[float, str]:
    """Non-tensor FP32 peak: 148 SMs x 128 lanes x 2 FLOP (FMA) x max SM clock."""
    mhz = peaks.get("sm_max_mhz")
    src = "MEASURED_PEAKS.json sm_max_mhz"
    if not mhz:
        mhz, src = 1965.0, "nominal 1965 MHz"
    return N_SMS * FP32_LANES_PER_SM * 2 * mhz * 1e6 / 1e12, src


class ClockSampler:
    """nvidia-smi samples during the timed region (clocks and throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return world, rank, local


def allreduce_max_sum(vals_max: list[float], vals_sum: list[float], world: int):
    if world <= 1:
        return vals_max, vals_sum
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    tm = torch.tensor(vals_max, dtype=torch.float64, device=dev)
    ts = torch.tensor(vals_sum, dtype=torch.float64, device=dev)
    dist.all_reduce(tm, op=dist.ReduceOp.MAX)
    dist.all_reduce(ts, op=dist.ReduceOp.SUM)
    return tm.tolist(), ts.tolist()


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


class L2Flusher:
    """Writes a buffer larger than the 126 MB L2 between timed steps."""

    def __init__(self, device: int):
        import torch
        self.torch = torch
        self.buf = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{device}")

    def flush(self):
        self.buf.fill_(1)
        self.torch.cuda.synchronize()


L2_NOTE = ("GPU arm: L2 flushed (256 MB write) before every timed step; CPU arm: the oracle on the host cores, "
           "no flush")
SURFEL_NOTE = {
    "c2_product": "200k surfels requested, 55,003 placed: the reference's generator draws min(24 x target, 6M) "
                  "Halton seeds (surfel.rs:183) and keeps those that pass its Poisson-disc spacing for the "
                  "requested density, which this scene's surface area allows 55,003 times; links follow "
                  "(772,534), so the ~2M links a 200k-surfel scene would have are unreachable under the "
                  "reference algorithm",
}


def workload_config(workload, scene_path, desc, cfg, placed, world) -> dict:
    """The workload's identity, the same keys and values in both arms."""
    return {"workload": workload, "scene": scene_path, "description": desc, "film": f"{cfg.width}x{cfg.height}",
            "surfels_requested": cfg.surfels, "surfels_placed": placed, "max_bounces": cfg.bounces,
            "cluster_res": 8, "l2": L2_NOTE, "parallelism": f"replicas x{world}"}


def fused_frame(ctx, cfg, srgb, cluster_res=8, out_srgb=None):
    return ctx.frame(cfg.width, cfg.height, "beauty", cluster_res=cluster_res, max_bounces=cfg.bounces,
                     linear=False, srgb=srgb, out_srgb=out_srgb)


def frame(ctx, cfg, cluster_res=8):
    info = ctx.build(cluster_res)
    le = ctx.light_surfels()
    st = ctx.solve(cfg.bounces)
    ctx.grid_build()
    _, _, se = ctx.render_frame(cfg.width, cfg.height, linear=False, srgb=False)
    return info, le, st, se


def run_ours(args, world, rank, local) -> dict | None:
    import numpy as np
    import interflect_b200 as ifx

    scene_path, desc = WORKLOADS[args.workload]
    with open(os.path.join(ROOT, scene_path)) as f:
        src = f.read()
    scene = ifx.parse(src)
    if args.film:
        fw, fh = (int(v) for v in args.film.lower().split("x"))
        scene.set_cfg(width=fw, height=fh)
    if args.surfels:
        scene.set_cfg(surfels=args.surfels)
    cfg = scene.cfg
    ctx = ifx.Context(local)
    ctx.upload(scene)
    t0 = time.time()
    placed = ctx.generate(cfg.surfels)
    gen_s = time.time() - t0
    surf = ctx.surfels()

    # Work accounting (instrumented kernels, outside any timed region).
    ctx.set_work_counting(True)
    ctx.reset_work()
    frame(ctx, cfg)
    work = {k: ctx.work(k) for k in KERNEL_NAMES}
    ctx.set_work_counting(False)

    flusher = L2Flusher(local)
    for _ in range(args.warmup):
        fused_frame(ctx, cfg, srgb=False)
    barrier(world)
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    launches0 = ctx.stats()["kernel_launches"]
    total_ms, evals_total = 0.0, 0
    f = None
    for _ in range(args.steps):
        flusher.flush()
        ctx.timer_start()
        f = fused_frame(ctx, cfg, srgb=False)
        total_ms += ctx.timer_stop()
        evals_total += f["transfer"].evals + f["light_evals"] + f["shade_evals"]
    launches = ctx.stats()["kernel_launches"] - launches0
    clocks = sampler.stop() if sampler else None
    info, st = f["transfer"], f["solve"]
    barrier(world)

    # Per-stage and per-kernel times (and the roofline's kernel duration) come
    # from frames made of the stage calls, where no kernel shares the GPU with
    # another stream.
    staged_ms = 0.0
    kms = {k: [] for k in KERNEL_NAMES}
    stage = {"transfer": [], "light": [], "solve": [], "grid": [], "shade": []}
    n_staged = min(args.steps, 10)
    for _ in range(n_staged):
        flusher.flush()
        ctx.timer_start()
        frame(ctx, cfg)
        staged_ms += ctx.timer_stop()
        s_ = ctx.stats()
        for k in KERNEL_NAMES:
            kms[k].append(s_["ms_" + k])
        for k in stage:
            stage[k].append(s_["ms_" + k])
    barrier(world)

    # End to end through the C ABI with host buffers: scene + surfels in,
    # encoded image out, every step. The image lands in one page-locked host
    # array the caller reuses (surfels are staged through the library's own
    # page-locked buffer).
    e2e_ms, e2e_evals = 0.0, 0
    import torch
    img = torch.zeros((cfg.height, cfg.width, 3), dtype=torch.uint8, pin_memory=True).numpy()
    h2d = None
    for i in range(args.warmup + args.steps):
        flusher.flush()
        ctx.timer_start()
        ctx.upload(scene)
        ctx.upload_surfels(surf["p"], surf["n"], surf["albedo"], surf["area"])
        f2 = fused_frame(ctx, cfg, srgb=True, out_srgb=img)
        ms = ctx.timer_stop()
        if i >= args.warmup:
            e2e_ms += ms
            e2e_evals += f2["transfer"].evals + f2["light_evals"] + f2["shade_evals"]
            img = f2["srgb"]
    h2d = placed * 16 * 3 + len(src)  # surfel p+area, n, albedo as float4; scene text
    d2h = int(img.nbytes)

    (t_max, e2e_max), (ev_sum, e2e_ev_sum) = allreduce_max_sum([total_ms, e2e_ms], [evals_total, e2e_evals], world)
    if rank != 0:
        return None

    sec = t_max / 1e3
    value = ev_sum / sec
    # Dominant kernel: the single kernel with the largest share of the frame.
    avg = {k: statistics.mean(v) for k, v in kms.items()}
    dom = max((k for k in avg if k != "shade_other"), key=avg.get)
    flops = work[dom][1]
    peaks = measured_peaks()
    peak, peak_src = fp32_peak_tflops(peaks)
    achieved = flops / (avg[dom] / 1e3) / 1e12
    traffic = None
    tj = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    traffic_src = None
    if os.path.exists(tj) and not args.film and not args.surfels:
        with open(tj) as f:
            tw = json.load(f).get(args.workload, {})
        traffic, traffic_src = tw.get(dom), tw.get("_source")

    # Issue-slot roofline of the same kernel: its warp instructions per launch
    # (ncu, the same workload) over the live duration, against 148 SMs x 4
    # schedulers x the SM clock sampled during the timed region.
    issue = None
    ij = os.path.join(ROOT, "profiles", "ncu_issue.json")
    if os.path.exists(ij) and not args.film and not args.surfels:
        with open(ij) as f:
            iw = json.load(f).get(args.workload, {})
        inst = iw.get(dom)
        mhz = (clocks or {}).get("sm_mhz") or peaks.get("sm_max_mhz") or 1965.0
        if inst:
            slots = N_SMS * 4 * mhz * 1e6 * (avg[dom] / 1e3)
            issue = {"warp_inst_per_launch": inst, "issue_slots_per_launch": slots, "frac": inst / slots,
                     "sm_mhz": mhz, "source": "profiles/ncu_issue.json (ncu smsp__inst_executed.sum): "
                                              + str(iw.get("_source", ""))}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.workload, scene_path, desc, cfg, placed, world),
        "workload_stats": {"clusters": info.clusters, "candidates": info.candidates, "links": info.links,
                           "bounces_run": st.iterations, "evals_per_frame": evals_total // max(args.steps, 1),
                           "note": SURFEL_NOTE.get(args.workload, "")},
        "frame": "ifx_frame: GI stages on one stream, GI-free shading passes overlapped on a second",
        "frame_ms": t_max / args.steps,
        "staged_frame_ms": staged_ms / n_staged,
        "stage_ms": {k: statistics.mean(v) for k, v in stage.items()},
        "solve_gbs": solve_bytes(info.links, placed, info.clusters) * st.iterations
        / (statistics.mean(stage["solve"]) / 1e3) / 1e9,
        "links_per_s": info.links / (statistics.mean(stage["transfer"]) / 1e3),
        "kernel_ms": avg,
        "surfel_generation_s": gen_s,
        "roofline": {"kernel": dom, "bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_src,
                     "flops_per_launch": flops, "peak_source": f"fp32 CUDA-core peak from {peak_src}",
                     "work": {k: float(v[1]) for k, v in work.items()}, "issue": issue},
        "e2e": {"value": e2e_ev_sum / (e2e_max / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_max / args.steps,
                "host_buffers": "scene text and surfel arrays from host memory (surfels staged through the "
                                "library's page-locked buffer); sRGB frame into a page-locked array reused "
                                "every step"},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if not args.no_cpu_baseline and world == 1:
        threads = os.cpu_count() or 1
        stride, rows_frac = cpu_sample_plan(placed, cfg.width, cfg.height, args)
        c = cpu_frame(src, surf, cfg, threads, stride=stride, rows_frac=rows_frac)
        line["cpu_baseline"] = cpu_baseline(c, cfg, threads)
        line["parity"] = frame_parity(ctx, cfg, c)
    return line


def relight_rhs(n: int, R: int, seed: int = 7):
    """R emission vectors, each 1-4 surfels-as-lights of intensity U[1, 50]."""
    import numpy as np
    rng = np.random.default_rng(seed)
    E = np.zeros((R, n, 3), np.float32)
    for r in range(R):
        k = rng.integers(1, 5)
        idx = rng.choice(n, size=k, replace=False)
        E[r, idx, :] = rng.uniform(1.0, 50.0, size=(k, 1)).astype(np.float32)
    return E


def run_batch(args, world, rank, local) -> dict | None:
    """Batched relighting: solves/s of the SpMM path against a plain loop of
    single-RHS solves through the same API, both on this GPU."""
    import interflect_b200 as ifx
    scene_path, desc = WORKLOADS[args.workload]
    with open(os.path.join(ROOT, scene_path)) as f:
        src = f.read()
    scene = ifx.parse(src)
    ctx = ifx.Context(local)
    ctx.upload(scene)
    placed = ctx.generate(scene.cfg.surfels)
    info = ctx.build(8)
    R, bounces = 256, scene.cfg.bounces
    E = relight_rhs(placed, R)
    tuned = ctx.autotune_batched(E)
    ctx.solve_batched(E, bounces, outputs=False)  # leaves E resident
    for _ in range(args.warmup):
        ctx.solve_batched(None, bounces, outputs=False, R=R)
    flusher = L2Flusher(local)
    barrier(world)
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    launches0 = ctx.stats()["kernel_launches"]
    total_ms = 0.0
    for _ in range(args.steps):
        flusher.flush()
        ctx.timer_start()
        _, _, its, _ = ctx.solve_batched(None, bounces, outputs=False, R=R)
        total_ms += ctx.timer_stop()
    launches = ctx.stats()["kernel_launches"] - launches0
    clocks = sampler.stop() if sampler else None
    # End to end: right-hand sides from host memory, radiosity back to host.
    e2e_ms = 0.0
    for _ in range(args.steps):
        flusher.flush()
        ctx.timer_start()
        ctx.solve_batched(E, bounces, outputs=True)
        e2e_ms += ctx.timer_stop()
    # Baseline: the plain loop of single-RHS solves through the public API.
    loop_n = min(R, 32)
    ctx.timer_start()
    for r in range(loop_n):
        ctx.set_emission(E[r])
        ctx.solve(bounces)
    loop_ms = ctx.timer_stop()
    (t_max, e2e_max), _ = allreduce_max_sum([total_ms, e2e_ms], [0.0], world)
    if rank != 0:
        return None
    value = R * args.steps * world / (t_max / 1e3)
    loop_rate = loop_n / (loop_ms / 1e3)
    # HBM roofline of the SpMM solve: algorithmic bytes of one step (every
    # right-hand side's own bounce count) over the step's device time.
    nbytes = spmm_bytes(info.links, placed, info.clusters, [int(x) for x in its])
    peak, peak_src = hbm_peak(measured_peaks())
    gbs = nbytes / (t_max / args.steps / 1e3) / 1e9
    return {
        "metric": BATCH_METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "scene": scene_path, "description": desc, "surfels_placed": placed,
                   "clusters": info.clusters, "links": info.links, "rhs": R, "max_bounces": bounces,
                   "bounces_run_max": int(max(its)), "spmm_warps_per_block": tuned,
                   "l2": "flushed (256 MB write) before every timed step"},
        "plain_loop": {"value": loop_rate, "unit": "solves/s", "rhs_timed": loop_n,
                       "speedup": value / loop_rate,
                       "contains": "per right-hand side: ifx_surfels_set_emission (E uploaded from host memory, "
                                   "direct = rad = E, irr = 0) then ifx_solve (one cooperative launch, its stop "
                                   "rule read back by the host), i.e. the single-RHS API a caller would loop over"},
        "roofline": {"kernel": "k_agg_batched + k_spmm + k_bounce_end_batched", "bound": "hbm", "achieved": gbs,
                     "peak": peak, "unit": "GB/s", "frac": gbs / peak, "traffic": None,
                     "bytes_per_step": nbytes, "peak_source": peak_src,
                     "bytes_model": "per bounce: 8 B/link + 4 B/row start + 20 B/surfel (albedo, area) shared by "
                                    "all right-hand sides, plus 80 B/surfel + 32 B/cluster per right-hand side "
                                    "still iterating (E, rad read twice, irr and rad written; cluster values "
                                    "written and read)"},
        "e2e": {"value": R * args.steps / (e2e_max / 1e3), "unit": "solves/s",
                "h2d_bytes_per_step": int(E.nbytes), "d2h_bytes_per_step": int(2 * E.nbytes)},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }


def run_multi(args, world, rank, local) -> dict | None:
    """Packed multi-scene frame: scenes/s of one graph launch over all 64
    scenes against (a) the same scenes one packed launch each and (b) the
    plain per-scene pipeline (light + solve + grid + render) in a loop."""
    import interflect_b200 as ifx
    from interflect_b200.scenes.gen_scenes import packed_scenes
    srcs = packed_scenes(64)
    t0 = time.time()
    members = []
    for src in srcs:
        sc = ifx.parse(src)
        ctx = ifx.Context(local)
        ctx.upload(sc)
        n = ctx.generate(sc.cfg.surfels)
        info = ctx.build(8)
        members.append((ctx, sc.cfg, n, info))
    prep_s = time.time() - t0
    ms = ifx.MultiScene(local)
    for ctx, cfg, _, _ in members:
        ms.add(ctx, cfg.width, cfg.height, cfg.bounces)
    grid, block = ms.build(autotune=True)
    flusher = L2Flusher(local)
    for _ in range(args.warmup):
        ms.run()
    barrier(world)
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    packed = []
    for _ in range(args.steps):
        flusher.flush()
        packed.append(ms.run())
    clocks = sampler.stop() if sampler else None
    iters = [ms.download(i, linear=False, srgb=False)[2].iterations for i in range(len(members))]
    # (a) One packed launch per scene (the unbatched form of the same work).
    singles = []
    for ctx, cfg, _, _ in members:
        one = ifx.MultiScene(local)
        one.add(ctx, cfg.width, cfg.height, cfg.bounces)
        one.build(autotune=False)
        singles.append(one)
    for one in singles:
        one.run()
    loop_a = []
    for _ in range(max(1, args.steps // 3)):
        flusher.flush()
        loop_a.append(sum(one.run() for one in singles))
    for one in singles:
        one.close()
    # (b) The plain pipeline per scene.
    loop_b = []
    for _ in range(max(1, args.steps // 10)):
        tot = 0.0
        for ctx, cfg, _, _ in members:
            ctx.timer_start()
            ctx.light_surfels()
            ctx.solve(cfg.bounces)
            ctx.grid_build()
            ctx.render_frame(cfg.width, cfg.height, linear=False, srgb=False)
            tot += ctx.timer_stop()
        loop_b.append(tot)
    # End to end: one replay plus every scene's encoded frame to the host.
    ms = ifx.MultiScene(local)
    for ctx, cfg, _, _ in members:
        ms.add(ctx, cfg.width, cfg.height, cfg.bounces)
    ms.build(autotune=False)
    d2h = sum(cfg.width * cfg.height * 3 for _, cfg, _, _ in members)
    e2e = []
    for _ in range(max(1, args.steps // 3)):
        flusher.flush()
        t = time.perf_counter()
        ms.run()
        for i in range(len(members)):
            ms.download(i, linear=False, srgb=True)
        e2e.append((time.perf_counter() - t) * 1e3)
    S = len(members)
    (t_max, a_max, b_max, e_max), _ = allreduce_max_sum(
        [statistics.median(packed), statistics.median(loop_a), statistics.median(loop_b), statistics.median(e2e)],
        [0.0], world)
    if rank != 0:
        return None
    return {
        "metric": "packed multi-scene frames per second (solve + shade of 64 scenes in one launch)",
        "value": S * world / (t_max / 1e3), "unit": "scenes/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "scenes": S, "description": WORKLOADS[args.workload][1],
                   "surfels_placed_total": sum(m[2] for m in members),
                   "links_total": sum(m[3].links for m in members),
                   "pixels_total": sum(m[1].width * m[1].height for m in members),
                   "bounces_run": [int(min(iters)), int(max(iters))], "launch": {"grid": grid, "block": block},
                   "l2": "flushed (256 MB write) before every timed step"},
        "one_launch_per_scene": {"value": S / (a_max / 1e3), "unit": "scenes/s", "speedup": a_max / t_max,
                                 "note": "the like-for-like baseline: the same packed kernel launched once per "
                                         "scene; both re-compose stored hits (geometry, camera and visibility "
                                         "were traced once at preparation)"},
        "plain_pipeline_loop": {"value": S / (b_max / 1e3), "unit": "scenes/s", "speedup": b_max / t_max,
                                "note": "ifx_light_surfels + ifx_solve + ifx_grid_build + ifx_render_frame per "
                                        "scene (re-traces every ray)"},
        "scene_preparation_s": prep_s,
        "e2e": {"value": S / (e_max / 1e3), "unit": "scenes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": d2h,
                "includes": "graph replay and every scene's sRGB frame downloaded to host"},
        "gpu_launches": args.steps,
        "clocks": clocks,
    }


def spmm_bytes(links: int, n: int, nc: int, its: list[int]) -> int:
    """Algorithmic bytes of one batched solve: the matrix, row starts, albedo
    and area once per bounce (the most any right-hand side runs), and per
    right-hand side per bounce its E, rad (read by the rows and by the
    cluster means), irr and rad writes and its cluster values."""
    return (8 * links + 4 * (n + 1) + 20 * n) * max(its) + (80 * n + 32 * nc) * sum(its)


def hbm_peak(peaks: dict) -> tuple[float, str]:
    for k in ("hbm_gbs", "hbm_copy_gbs", "copy_gbs"):
        if peaks.get(k):
            return float(peaks[k]), f"MEASURED_PEAKS.json {k} (measured copy bandwidth)"
    return 6650.0, "fallback 6.65 TB/s (earlier measurement on this pool; MEASURED_PEAKS.json absent)"


def solve_bytes(links: int, n: int, nc: int) -> int:
    """Algorithmic bytes of one bounce: link index + weight, row starts, the
    row's direct/albedo/rad read and irr/rad written (16 B each), the
    members' rad + area read by the cluster means, the cluster values."""
    return 8 * links + 4 * (n + 1) + 64 * n + 24 * nc


def run_solve_hbm(args, world, rank, local) -> dict | None:
    """The solve alone on a stress-sized transfer: the stress scene's 1M
    surfels and clusters with a synthetic CSR of 109 links per row (sorted
    cluster indices, seeded weights), installed with ifx_transfer_upload and
    solved by ifx_solve (the sliced-ELL kernel). The same matrix is also
    solved through ifx_solve_noalloc (the CSR kernel) for comparison, and the
    two results must agree bit for bit."""
    import numpy as np
    import torch
    import interflect_b200 as ifx
    with open(os.path.join(ROOT, "interflect_b200/scenes/c3_stress.rad")) as f:
        scene = ifx.parse(f.read())
    ctx = ifx.Context(local)
    ctx.upload(scene)
    n = ctx.generate(1_000_000)
    nc = ctx.build_clusters(8)
    per_row, bounces = 109, 24
    L = n * per_row
    rng = np.random.default_rng(11)
    idx = np.sort(rng.integers(0, nc, size=(n, per_row), dtype=np.uint32), axis=1).reshape(-1)
    w = (rng.random(L, dtype=np.float32) * np.float32(0.98 / per_row * 2)).astype(np.float32)
    starts = (np.arange(n + 1, dtype=np.uint64) * per_row).astype(np.uint32)
    ctx.upload_transfer(starts, idx, w)
    E = (rng.random((n, 3), dtype=np.float32) * np.float32(0.1)).astype(np.float32)
    flusher = L2Flusher(local)

    def once():
        ctx.set_emission(E)
        flusher.flush()
        st = ctx.solve(bounces)
        return st, ctx.stats()["ms_solve"]

    for _ in range(args.warmup):
        once()
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    times, st = [], None
    launches0 = ctx.stats()["kernel_launches"]
    for _ in range(args.steps):
        st, ms = once()
        times.append(ms)
    launches = ctx.stats()["kernel_launches"] - launches0
    clocks = sampler.stop() if sampler else None
    rad_sell = ctx.surfels()["rad"]
    # The CSR kernel on the same matrix (caller-owned device copies).
    dev = torch.device(f"cuda:{local}")
    s = ctx.surfels()
    cl = ctx.clusters(nc)
    t = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)
    p_area = t(np.concatenate([s["p"], s["area"][:, None]], 1))
    f4 = lambda a: t(np.concatenate([a, np.zeros((len(a), 1), np.float32)], 1))
    direct, albedo, irr = f4(E), f4(s["albedo"]), torch.zeros(n, 4, device=dev)
    rad = direct.clone()
    cp = t(np.concatenate([cl["p"], cl["area"][:, None]], 1))
    ranges = t(np.stack([cl["offsets"][:-1], cl["offsets"][1:]], 1).astype(np.int32), torch.int32)
    members = t(cl["members"].astype(np.int32), torch.int32)
    d_starts, d_idx, d_w = t(starts.astype(np.int32), torch.int32), t(idx.astype(np.int32), torch.int32), t(w)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    csr = []
    for i in range(args.warmup + args.steps):
        rad.copy_(direct)
        flusher.flush()
        e0.record(stream)
        st2 = ifx.solve_noalloc(local, stream.cuda_stream, n, nc, p_area.data_ptr(), direct.data_ptr(),
                                albedo.data_ptr(), irr.data_ptr(), rad.data_ptr(), cp.data_ptr(), ranges.data_ptr(),
                                members.data_ptr(), d_starts.data_ptr(), d_idx.data_ptr(), d_w.data_ptr(), bounces)
        e1.record(stream)
        e1.synchronize()
        if i >= args.warmup:
            csr.append(e0.elapsed_time(e1))
    same = bool(np.array_equal(rad[:, :3].cpu().numpy().view(np.uint32), rad_sell.view(np.uint32))) and \
        st2.iterations == st.iterations
    (t_max, csr_max), _ = allreduce_max_sum([statistics.median(times), statistics.median(csr)], [0.0], world)
    if rank != 0:
        return None
    bpb = solve_bytes(L, n, nc)
    gbs = bpb * st.iterations / (t_max / 1e3) / 1e9
    mp = measured_peaks()
    peak = mp.get("hbm_gbs", 6650.0)
    peak_src = ("MEASURED_PEAKS.json hbm_gbs (copy bandwidth)" if "hbm_gbs" in mp
                else "fallback 6650 GB/s (an earlier copy-bandwidth measurement on this pool)")
    traffic = None
    tj = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tj):
        with open(tj) as f:
            traffic = json.load(f).get(args.workload, {}).get("jacobi_sell")
    return {
        "metric": "Jacobi solve bandwidth (algorithmic bytes per bounce x bounces / time)", "value": gbs * world,
        "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "surfels": n, "clusters": nc, "links": L, "bounces_run": st.iterations,
                   "bytes_per_bounce": bpb, "l2": "flushed before each solve; working set 7x the 126 MB L2"},
        "roofline": {"kernel": "k_jacobi_sell + k_cluster_agg", "bound": "hbm", "achieved": gbs, "peak": peak,
                     "unit": "GB/s", "frac": gbs / peak, "traffic": traffic,
                     "peak_source": peak_src},
        "csr_kernel": {"value": bpb * st.iterations / (csr_max / 1e3) / 1e9, "unit": "GB/s",
                       "ms": csr_max, "bit_identical_to_sliced_ell": same},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }


def run_diff(args, world, rank, local) -> dict | None:
    """Differentiation: one gradient step (the frame for the current albedo
    and emission, the loss gradient on the host, the adjoint) against one
    forward frame of the same scene through the plain pipeline."""
    import numpy as np
    import interflect_b200 as ifx
    scene_path, desc = WORKLOADS[args.workload]
    with open(os.path.join(ROOT, scene_path)) as f:
        src = f.read()
    scene = ifx.parse(src)
    cfg = scene.cfg
    ctx = ifx.Context(local)
    ctx.upload(scene)
    placed = ctx.generate(cfg.surfels)
    flusher = L2Flusher(local)
    # One forward frame as the renderer makes it (transfer + light + solve +
    # grid + shade), CUDA-event timed.
    for _ in range(args.warmup):
        frame(ctx, cfg)
    fwd = []
    for _ in range(args.steps):
        flusher.flush()
        ctx.timer_start()
        info, _, _, _ = frame(ctx, cfg)
        fwd.append(ctx.timer_stop())
    # Differentiable frame: geometry, visibility and the transposes once.
    K = cfg.bounces
    dinfo = ctx.diff_setup(cfg.width, cfg.height, K)
    surf = ctx.surfels()
    rng = np.random.default_rng(2026)
    rho0 = surf["albedo"]
    rho_t = np.clip(rho0 + rng.normal(0.0, 0.05, rho0.shape), 0.05, 0.95).astype(np.float32)
    emit0 = ctx.light_emission()
    target = ctx.diff_forward(rho_t, emit0)
    for _ in range(args.warmup):
        img = ctx.diff_forward(rho0, emit0)
        ctx.diff_backward(2.0 * (img - target))
    barrier(world)
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    launches0 = ctx.stats()["kernel_launches"]
    dev_f, dev_b, e2e = [], [], []
    for _ in range(args.steps):
        flusher.flush()
        ctx.timer_start()
        img = ctx.diff_forward(rho0, emit0)
        g_img = 2.0 * (img - target)
        g_rho, g_e = ctx.diff_backward(g_img)
        e2e.append(ctx.timer_stop())
        st = ctx.stats()
        dev_f.append(st["ms_diff_forward"])
        dev_b.append(st["ms_diff_backward"])
    launches = ctx.stats()["kernel_launches"] - launches0
    clocks = sampler.stop() if sampler else None
    (grad_max, fwd_max, e2e_max), _ = allreduce_max_sum(
        [statistics.median([f + b for f, b in zip(dev_f, dev_b)]), statistics.median(fwd), statistics.median(e2e)],
        [0.0], world)
    if rank != 0:
        return None
    loss = float(((img - target) ** 2).sum())
    return {
        "metric": DIFF_METRIC, "value": grad_max, "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": grad_max, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "scene": scene_path, "description": desc, "film": [cfg.width, cfg.height],
                   "surfels_placed": placed, "clusters": info.clusters, "links": info.links, "bounces": K,
                   "gather_entries": dinfo["gather_entries"], "lights": dinfo["lights"],
                   "l2": "flushed (256 MB write) before every timed step"},
        "forward_frame_ms": fwd_max,
        "gradient_over_forward": grad_max / fwd_max,
        "gradient_device_ms": {"forward": statistics.median(dev_f), "adjoint": statistics.median(dev_b)},
        "setup_ms": dinfo["ms_setup"],
        "loss": loss, "grad_rho_norm": float(np.linalg.norm(g_rho)), "grad_emit": g_e.tolist(),
        "e2e": {"value": e2e_max, "unit": "ms", "h2d_bytes_per_step": int(rho0.nbytes + emit0.nbytes + g_img.nbytes),
                "d2h_bytes_per_step": int(img.nbytes + g_rho.nbytes + g_e.nbytes),
                "includes": "albedo+emission upload, frame download, host loss gradient, adjoint, gradient download"},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }


def cpu_sample_plan(placed: int, width: int, height: int, args) -> tuple[int, float]:
    """(row stride of the transfer and light stages, fraction of film rows
    shaded) for the CPU legs: every row up to 100k surfels and 1080p, else a
    bounded sample (about 10k surfel rows, about 330k pixels) so that one CPU
    frame stays within tens of seconds."""
    stride = args.cpu_stride if args.cpu_stride else max(1, -(-placed // 10000)) if placed > 100000 else 1
    if args.cpu_rows:
        rows_frac = args.cpu_rows
    else:
        rows_frac = 1.0 if width * height <= 1920 * 1080 else min(1.0, 330000 / (width * height))
    return stride, rows_frac


def cpu_frame(src, surf, cfg, threads, stride=1, rows_frac=1.0):
    """One frame of the oracle (the reference algorithm on the CPU) on the
    given surfels, stage by stage. With stride > 1 only every stride-th
    transfer row and surfel light is computed, and with rows_frac < 1 only
    the first rows of the film are shaded: the sample the rate is taken on.
    Returns the evaluation counts, the per-stage seconds, the film and the
    oracle itself (for the parity comparison)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import Oracle
    o = Oracle(src, threads=threads)
    o.set_surfels(surf["p"], surf["n"], surf["albedo"], surf["area"])
    t = {}
    t0 = time.perf_counter()
    o.build_clusters(8)
    info = o.build_transfer(stride)
    t["transfer"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    le = o.light_surfels(stride)
    t["light"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    it, _ = o.solve(cfg.bounces)
    t["solve"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    o.build_grid()
    t["grid"] = time.perf_counter() - t0
    rows = max(1, int(cfg.height * rows_frac))
    t0 = time.perf_counter()
    film, se = o.render(cfg.width, cfg.height, "beauty", rows=(0, rows))
    t["shade"] = time.perf_counter() - t0
    return dict(evals=info["evals"] + le + se, transfer_evals=info["evals"], light_evals=le, shade_evals=se,
                stage_s=t, dt=sum(t.values()), rows=rows, stride=stride, film=film, info=info, iterations=it,
                oracle=o)


def cpu_baseline(c: dict, cfg, threads: int) -> dict:
    """The CPU leg's line: SDF evaluations per second of the oracle on the
    host cores over the sample `c` (cpu_frame's result)."""
    full = c["stride"] == 1 and c["rows"] == cfg.height
    if full:
        value = c["evals"] / c["dt"]
        sample = (f"one frame of the same workload on the same surfels, every transfer row and film row; "
                  f"{c['evals'] / 1e6:.1f}M SDF evals in {c['dt']:.2f} s")
    else:
        # The ray stages' rate on the sample; the solve and grid run in full
        # on the sampled matrix and are not part of the rate.
        st = c["stage_s"]
        ray_s = st["transfer"] + st["light"] + st["shade"]
        value = c["evals"] / ray_s
        est = (st["transfer"] + st["light"]) * c["stride"] + st["shade"] * cfg.height / c["rows"]
        sample = (f"transfer rows and surfel lights i % {c['stride']} == 0 and film rows 0..{c['rows']} of "
                  f"{cfg.height}: {c['evals'] / 1e6:.1f}M SDF evals in {ray_s:.2f} s of ray stages "
                  f"(transfer {st['transfer']:.2f} s, light {st['light']:.2f} s, shade {st['shade']:.2f} s); "
                  f"a whole frame at these rates is about {est:.0f} s")
    return {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample, "cpu": cpu_model(),
            "stage_s": c["stage_s"]}


def frame_parity(ctx, cfg, c: dict) -> dict:
    """The GPU's frame against the oracle's on the same surfels: link rows of
    the sampled transfer rows (column indices exact, weights and per-row
    evaluation counts), direct light of the sampled surfels, and, where the
    CPU ran the whole frame, the bounce count and every shaded film row."""
    import numpy as np
    o = c["oracle"]
    n = ctx.n_surfels
    f = ctx.frame(cfg.width, cfg.height, "beauty", cluster_res=8, max_bounces=cfg.bounces, linear=True, srgb=False)
    gt = ctx.transfer()
    ot = o.transfer(n, c["info"]["links"])
    rows = np.arange(0, n, c["stride"])
    gs, os_ = gt["starts"].astype(np.int64), ot["starts"].astype(np.int64)
    mism, wmax = 0, 0.0
    for i in rows:
        gi_, oi_ = gt["idx"][gs[i]:gs[i + 1]], ot["idx"][os_[i]:os_[i + 1]]
        if not np.array_equal(gi_, oi_):
            mism += 1
            continue
        if len(gi_):
            a = gt["w"][gs[i]:gs[i + 1]].astype(np.float64)
            b = ot["w"][os_[i]:os_[i + 1]].astype(np.float64)
            wmax = max(wmax, float((np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-6)).max()))
    gd = ctx.row_diag()
    evals_equal = bool(np.array_equal(gd["row_evals"][rows], ot["row_evals"][rows]))
    out = {"rows_compared": int(len(rows)), "link_row_mismatches": int(mism), "link_weight_max_rel": wmax,
           "row_evals_equal": evals_equal}
    full = c["stride"] == 1 and c["rows"] == cfg.height
    if c["stride"] == 1:
        g, r = ctx.surfels(), o.surfels()
        e = np.abs(g["direct"].astype(np.float64) - r["direct"]) / np.maximum(
            np.maximum(np.abs(g["direct"]), np.abs(r["direct"])), 1e-6)
        out["direct_max_rel"] = float(e.max()) if e.size else 0.0
        out["bounces_equal"] = f["solve"].iterations == c["iterations"]
    if full:
        lin, film = f["linear"].astype(np.float64), c["film"].astype(np.float64)
        e = np.abs(lin - film) / np.maximum(np.maximum(np.abs(lin), np.abs(film)), 1e-6)
        out.update({"film_rows_compared": c["rows"], "max_rel": float(e.max()), "rms": float(np.sqrt(np.mean(e ** 2))),
                    "bit_identical_frac": float(np.mean(f["linear"] == c["film"])),
                    "evals_equal": f["transfer"].evals + f["light_evals"] + f["shade_evals"] == c["evals"]})
    else:
        out["film"] = "not compared: the sampled transfer leaves the CPU solve incomplete"
    out["tolerance"] = "integers exact, floats within 1e-4 relative"
    out["ok"] = bool(mism == 0 and wmax <= 1e-4 and evals_equal and out.get("max_rel", 0.0) <= 1e-4
                     and out.get("direct_max_rel", 0.0) <= 1e-4 and out.get("bounces_equal", True)
                     and out.get("evals_equal", True))
    return out


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_pathtrace(args, world, rank, local) -> dict | None:
    """The path tracer of `--mode reference` (reference.rs:61-137): one step
    is one full film at 512 samples per pixel."""
    import interflect_b200 as ifx
    scene_path, desc = WORKLOADS[args.workload]
    with open(os.path.join(ROOT, scene_path)) as f:
        src = f.read()
    scene = ifx.parse(src)
    W = H = PT_FILM
    if args.film:
        W, H = (int(v) for v in args.film.lower().split("x"))
    spp = PT_SPP
    ctx = ifx.Context(local)
    ctx.upload(scene)
    ctx.set_work_counting(True)
    ctx.reset_work()
    ctx.render_reference(W, H, spp, linear=False, srgb=False)
    counts, flops = ctx.work("path")
    ctx.set_work_counting(False)
    for _ in range(args.warmup):
        ctx.render_reference(W, H, spp, linear=False, srgb=False)
    flusher = L2Flusher(local)
    barrier(world)
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    launches0 = ctx.stats()["kernel_launches"]
    total_ms, kms = 0.0, []
    for _ in range(args.steps):
        flusher.flush()
        ctx.timer_start()
        ctx.render_reference(W, H, spp, linear=False, srgb=False)
        total_ms += ctx.timer_stop()
        kms.append(ctx.stats()["ms_shade"])
    launches = ctx.stats()["kernel_launches"] - launches0
    clocks = sampler.stop() if sampler else None
    barrier(world)
    # End to end: the scene uploaded from host memory and the encoded image
    # read back, every step.
    e2e_ms, out8 = 0.0, None
    for i in range(args.warmup + args.steps):
        flusher.flush()
        ctx.timer_start()
        ctx.upload(scene)
        _, out8 = ctx.render_reference(W, H, spp, linear=False, srgb=True)
        ms = ctx.timer_stop()
        if i >= args.warmup:
            e2e_ms += ms
    (t_max, e2e_max), _ = allreduce_max_sum([total_ms, e2e_ms], [0.0], world)
    if rank != 0:
        return None
    samples = W * H * spp
    value = samples * args.steps * world / (t_max / 1e3)
    kavg = statistics.mean(kms)
    peak, peak_src = fp32_peak_tflops(measured_peaks())
    achieved = flops / (kavg / 1e3) / 1e12
    line = {
        "metric": PT_METRIC, "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "scene": scene_path, "description": desc, "film": [W, H],
                   "spp": spp, "max_depth": 12, "l2": "flushed (256 MB write) before every timed step",
                   "parallelism": f"replicas x{world}"},
        "kernel_ms": {"path": kavg},
        "roofline": {"kernel": "path", "bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None, "flops_per_launch": flops,
                     "peak_source": f"fp32 CUDA-core peak from {peak_src}",
                     "sdf_queries_per_launch": int(counts[11]), "march_steps_per_launch": int(counts[12])},
        "e2e": {"value": samples * args.steps / (e2e_max / 1e3), "unit": "samples/s",
                "h2d_bytes_per_step": len(src), "d2h_bytes_per_step": int(out8.nbytes),
                "ms_per_step": e2e_max / args.steps},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = pathtrace_cpu(src, W, H, spp)
    return line


def pathtrace_cpu(src, W, H, spp, rows=PT_CPU_ROWS) -> dict:
    """The oracle's path tracer on all host cores over the first `rows` rows."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import Oracle
    threads = os.cpu_count() or 1
    o = Oracle(src, threads=threads)
    rows = min(rows, H)
    t0 = time.perf_counter()
    o.render(W, H, "reference", rows=(0, rows), spp=spp)
    dt = time.perf_counter() - t0
    n = W * rows * spp
    return {"value": n / dt, "unit": "samples/s", "cores": threads, "kind": "port",
            "sample": f"rows 0..{rows} of the {W}x{H} film at {spp} spp ({n / 1e6:.2f}M samples in {dt:.2f} s)",
            "cpu": cpu_model()}


def run_reference(args, world, rank) -> dict | None:
    if rank != 0:
        return None
    if args.workload == "pathtrace":
        return run_reference_pathtrace(args, world)
    if args.workload in ("c4_batch", "c4_multi", "c5_diff", "solve_hbm"):
        # Batched relighting, packed scenes, gradients and the solve alone have
        # no CPU entry point in the reference; these lines carry their own
        # baselines (plain per-RHS / per-scene loops, the forward frame, the
        # CSR kernel).
        return {"impl": "reference", "unavailable": f"the reference has no CPU counterpart of the {args.workload} "
                                                    "workload; its line reports its own baseline"}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import Oracle
    scene_path, desc = WORKLOADS[args.workload]
    with open(os.path.join(ROOT, scene_path)) as f:
        src = f.read()
    threads = os.cpu_count() or 1
    o = Oracle(src, threads=threads)
    cfg_i = o.info()

    class Cfg:
        width, height, bounces, surfels = cfg_i["width"], cfg_i["height"], cfg_i["bounces"], cfg_i["surfels"]
    if args.film:
        Cfg.width, Cfg.height = (int(v) for v in args.film.lower().split("x"))
    if args.surfels:
        Cfg.surfels = args.surfels
    t0 = time.time()
    placed = o.generate(Cfg.surfels)
    gen_s = time.time() - t0
    surf = o.surfels()
    stride, rows_frac = cpu_sample_plan(placed, Cfg.width, Cfg.height, args)
    total_t, total_ev, last = 0.0, 0, None
    for i in range(args.warmup + args.steps):
        c = cpu_frame(src, surf, Cfg, threads, stride=stride, rows_frac=rows_frac)
        b = cpu_baseline(c, Cfg, threads)
        if i >= args.warmup:
            total_t += c["evals"] / b["value"]
            total_ev += c["evals"]
        last = (c, b)
    value = total_ev / total_t
    c, b = last
    b["value"] = value
    b["sample"] = f"{args.steps} timed steps, each " + b["sample"]
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_t / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.workload, scene_path, desc, Cfg, placed, world),
            "workload_stats": {"clusters": c["info"]["clusters"], "links": c["info"]["links"],
                               "bounces_run": c["iterations"], "evals_per_step": c["evals"],
                               "note": SURFEL_NOTE.get(args.workload, "")},
            "surfel_generation_s": gen_s,
            "cpu_baseline": b,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the Rust reference cannot be built in this image (no rustc/cargo); this arm times the "
                    "oracle, a line-by-line C++ restatement of the reference's CPU path, on all host threads"}


def run_reference_pathtrace(args, world) -> dict:
    scene_path, desc = WORKLOADS[args.workload]
    with open(os.path.join(ROOT, scene_path)) as f:
        src = f.read()
    W = H = PT_FILM
    vals = []
    for i in range(args.warmup + args.steps):
        b = pathtrace_cpu(src, W, H, PT_SPP)
        if i >= args.warmup:
            vals.append(b)
    value = statistics.mean(v["value"] for v in vals)
    rows = min(PT_CPU_ROWS, H)
    return {"impl": "reference", "metric": PT_METRIC, "value": value, "unit": "samples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": W * H * PT_SPP / value * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "scene": scene_path, "description": desc, "film": [W, H],
                       "spp": PT_SPP},
            "cpu_baseline": {"value": value, "unit": "samples/s", "cores": vals[0]["cores"], "kind": "port",
                             "sample": f"each step shades rows 0..{rows} of the film; ms_per_step is the "
                                       "whole film at that rate", "cpu": vals[0]["cpu"]},
            "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the Rust reference cannot be built in this image (no rustc/cargo); this arm times the "
                    "oracle's restatement of reference.rs on all host threads"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2_product", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-rows", type=float, default=None,
                    help="fraction of film rows the CPU legs shade (default: all up to 1080p, else about 330k pixels)")
    ap.add_argument("--cpu-stride", type=int, default=None,
                    help="CPU legs compute transfer rows and surfel lights i %% stride == 0 (default: 1 up to "
                         "100k surfels, else about 10k rows)")
    ap.add_argument("--film", default=None, help="WxH film override for small profiling cases (e.g. 640x360)")
    ap.add_argument("--surfels", type=int, default=None, help="surfel target override for small profiling cases")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            line = run_reference(args, world, rank)
        elif args.workload == "c4_batch":
            line = run_batch(args, world, rank, local)
        elif args.workload == "c5_diff":
            line = run_diff(args, world, rank, local)
        elif args.workload == "solve_hbm":
            line = run_solve_hbm(args, world, rank, local)
        elif args.workload == "c4_multi":
            line = run_multi(args, world, rank, local)
        elif args.workload == "pathtrace":
            line = run_pathtrace(args, world, rank, local)
        else:
            line = run_ours(args, world, rank, local)
        if line is not None:
            print(json.dumps(line), flush=True)
            if not line.get("parity", {}).get("ok", True):
                # A fast frame that differs from the reference algorithm's is
                # not a result: say so and fail the run.
                print(f"bench: the GPU frame differs from the oracle's: {line['parity']}", file=sys.stderr)
                sys.exit(3)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
