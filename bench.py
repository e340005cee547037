#!/usr/bin/env python
"""Benchmark of the fused GRRT ray kernel on the plain-method scale workload.

Workload (one "step" = one full image): 1024 x 1024 rays from r_obs = 1000 M,
inclination 17 deg, field of view +-20 M, Kerr spin a = 0.9375, fixed-step RK2
with h = 0.02 r clamped to [1e-3, 1] and at most 4096 steps, through a
256 x 128 x 256 x 11 float32 synthetic torus brick (seeded).  The metric is
ray-steps/s: RK2 geodesic steps executed by live rays (counted on the device)
divided by the device time of the timed steps, summed over all GPUs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference algorithm's CPU restatement (the float64
oracle, OpenMP over every host core) on a bounded sample of the same workload.

Other workloads (--workload): views (256 uneven views in one launch),
precompute (coefficient bricks from a 256 x 128 x 256 seeded snapshot, cells/s)
and grrt (the physical polarized renderer's default 160 x 90 image, pixels/s),
whose lines carry an FP64 exp() roofline measured in the same run; learned
(time to an image at 1e-3 Stokes-I error: the learned step size against plain
RK2 and the step-doubling controller); bricks (the reference's own fixed-step
RK4 brick renderer, its default 160 x 90 image, pixels/s, FP64 roofline);
micro (the plugin's sample_and_step_stokes on 16.8M points, points/s, HBM
roofline).
For N > 1 the job runs as torchrun ranks, one full image per rank (replicas:
rays are independent and the path has no exchange step).
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
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "blackhole-sim_b200"))

METRIC = "ray-steps/s"
UNIT = "ray-steps/s"
WORKLOAD = dict(width=1024, height=1024, spin_a=0.9375, r_obs=1000.0, inclination_deg=17.0, max_steps=4096,
                h_scale=0.02, h_min=1e-3, h_max=1.0, escape_radius=220.0)
BRICK = dict(nr=256, ntheta=128, nphi=256, seed=0)
FOV_Y_DEG = 2.0 * math.degrees(math.atan(20.0 / 1000.0))  # +-20 M at r_obs = 1000 M (the View default)
# Algorithmic work of the implemented method (counted from the kernel's
# arithmetic, one FMA = 2 FLOP, a divide / sqrt = 1): a geodesic RK2 step
# (two Hamiltonian right-hand sides with their pole sin/cos, the FP64 state
# update, the termination tests, the drift bookkeeping) and the extra work of a
# step whose midpoint lies in the brick (cell location, 8-corner x 11-channel
# trilinear gather, Stokes RK2, optical depth).
FLOP_PER_STEP = 213
FLOP_PER_BRICK_STEP = 305
BYTES_PER_BRICK_STEP = 8 * 11 * 4     # 8 corners x 11 float32 channels
BYTES_PER_RAY = 16                    # float4 Stokes written once per ray
MEASURED_PEAKS = REPO / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
PROFILE_SUMMARY = REPO / "profiles" / "render_kernel_fp32_image1024.md"


# ------------------------------------------------------------------ helpers
def dist_env() -> tuple[int, int, int]:
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def init_dist(world: int, backend: str):
    import torch.distributed as td

    if world > 1 and not td.is_initialized():
        import datetime

        td.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
    return td


def max_over_ranks(value: float, world: int, device) -> float:
    """Largest value over all ranks (the timing rule: max over ranks)."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as td

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, world: int, device) -> float:
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as td

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    td.all_reduce(t, op=td.ReduceOp.SUM)
    return float(t.item())


def barrier(world: int) -> None:
    if world > 1:
        import torch
        import torch.distributed as td

        if td.get_backend() == "nccl":  # name this rank's GPU: NCCL would otherwise guess one
            td.barrier(device_ids=[torch.cuda.current_device()])
        else:
            td.barrier()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms in the background."""

    QUERY = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.lines: list[str] = []
        self._t = None

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.uuid:
            cmd.insert(1, f"--id={self.uuid}")
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 10:
                continue
            try:
                sm.append(float(f[2]))
                smax.append(float(f[3]))
                power.append(float(f[4]))
            except ValueError:
                continue
            for n, v in zip(names, f[6:10]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


def load_peaks() -> dict:
    if MEASURED_PEAKS.exists():
        d = json.loads(MEASURED_PEAKS.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": FALLBACK_HBM_GBS, "source": "fallback"}


def profiled_traffic(summary: Path = PROFILE_SUMMARY) -> float | None:
    """DRAM bytes per launch of a kernel from its committed ncu summary."""
    if not summary.exists():
        return None
    for line in summary.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def _bricks_module():
    """blackhole_native/bricks.py loaded by its path: it needs numpy only, and
    importing the package would load the CUDA library (the reference arm must
    run without it)."""
    import importlib.util

    name = "_bhn_bricks_numpy"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, REPO / "blackhole-sim_b200" / "blackhole_native" / "bricks.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def make_brick():
    return _bricks_module().torus_brick(BRICK["nr"], BRICK["ntheta"], BRICK["nphi"], spin_a=WORKLOAD["spin_a"],
                                        seed=BRICK["seed"], dtype=np.float32)


def run_oracle(brick, n: int, threads: int = 0) -> tuple[int, float]:
    """The float64 oracle on an n x n image of the workload's field of view.
    Returns (ray_steps, seconds)."""
    sys.path.insert(0, str(REPO))
    from oracle import oracle as O

    w = WORKLOAD
    ov = O.make_view(spin_a=w["spin_a"], r_obs=w["r_obs"], theta_obs=math.radians(w["inclination_deg"]), phi_obs=0.0,
                     fov_y_deg=FOV_Y_DEG, roll_deg=0.0, h_scale=w["h_scale"], h_min=w["h_min"], h_max=w["h_max"],
                     escape_radius=w["escape_radius"], affine_to_length_cm=1.0, max_optical_depth=30.0, width=n,
                     height=n, x0=0, y0=0, crop_w=n, crop_h=n, max_steps=w["max_steps"])
    t0 = time.perf_counter()
    _, steps, _, _ = O.render(ov, brick.coeffs, brick.r, brick.theta, brick.phi, stop_at_tau=True, threads=threads)
    return int(steps.sum()), time.perf_counter() - t0


def calibrated_oracle_size(brick, target_s: float) -> int:
    """Side n of the n x n oracle sample that takes about target_s seconds
    (two rounds: the first, tiny sample under-uses the threads)."""
    n = 48
    for _ in range(2):
        steps, dt = run_oracle(brick, n)
        n = int(n * math.sqrt(max(target_s, 0.1) / max(dt, 1e-3)) * (0.5 if n == 48 else 1.0))
        n = max(32, min(1024, n))
    return n


def cpu_baseline(brick, target_s: float = 12.0) -> dict:
    from oracle import oracle as O

    n = calibrated_oracle_size(brick, target_s)
    steps, dt = run_oracle(brick, n)
    return {"value": steps / dt, "unit": UNIT, "cores": O.max_threads(), "kind": "port",
            "sample": f"float64 oracle (C, OpenMP), {n}x{n} rays over the full field of view, {steps} ray-steps "
                      f"in {dt:.2f} s"}


def fp32_peak(device, stream) -> float:
    """FP32 FMA peak of this GPU in TFLOP/s (the denominator of the FP32
    roofline), measured with the library's FMA-chain probe."""
    import ctypes

    import torch

    from blackhole_native import _lib

    probe = torch.empty(1 << 20, dtype=torch.float32, device=device)
    flops = ctypes.c_int64()
    L = _lib.lib()
    for _ in range(2):
        _lib.check(L.bhn_fp32_peak_probe(probe.data_ptr(), 4096, 8, ctypes.byref(flops), stream.cuda_stream))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    _lib.check(L.bhn_fp32_peak_probe(probe.data_ptr(), 4096, 8, ctypes.byref(flops), stream.cuda_stream))
    e1.record(stream)
    torch.cuda.synchronize(device)
    return flops.value / (e0.elapsed_time(e1) * 1e-3) / 1e12


def render_rooflines(steps: int, brick_steps: int, rays: int, kernel_s: float, fp32_peak_tflops: float,
                     traffic: float | None, traffic_source: str | None) -> tuple[dict, dict]:
    """HBM roofline (algorithmic gather bytes) and FP32 roofline (algorithmic
    FLOP) of one render launch."""
    peaks = load_peaks()
    alg_bytes = brick_steps * BYTES_PER_BRICK_STEP + rays * BYTES_PER_RAY
    alg_flops = steps * FLOP_PER_STEP + brick_steps * FLOP_PER_BRICK_STEP
    achieved_gbs = alg_bytes / kernel_s / 1e9
    roofline = {"bound": "hbm", "achieved": round(achieved_gbs, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": round(achieved_gbs / peaks["hbm_gbs"], 4), "traffic": traffic,
                "traffic_source": traffic_source,
                "peak_source": f"{peaks['source']} (MEASURED_PEAKS.json hbm_gbs)" if peaks["source"] == "measured"
                else "fallback 6.65 TB/s",
                "kernel": "render_kernel<Tracer32>", "algorithmic_bytes_per_launch": int(alg_bytes)}
    achieved_tf = alg_flops / kernel_s / 1e12
    roofline_fp32 = {"bound": "fp32", "achieved": round(achieved_tf, 2), "peak": round(fp32_peak_tflops, 2),
                     "unit": "TFLOP/s", "frac": round(achieved_tf / fp32_peak_tflops, 4),
                     "peak_source": "measured in this run (bhn_fp32_peak_probe FMA loop)",
                     "algorithmic_flops_per_launch": int(alg_flops)}
    return roofline, roofline_fp32


# ------------------------------------------------------------------ arms
def bench_ours(args) -> dict | None:
    import torch

    import blackhole_native as bn
    from blackhole_native import _lib

    rank, world, local_rank = dist_env()
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    init_dist(world, "nccl")

    brick_h = make_brick()
    db = bn.DeviceBrick(brick_h, device=device, precisions=("fp32",))
    wl = dict(WORKLOAD)
    if args.side:  # a smaller image of the same scene (profiling runs)
        wl.update(width=args.side, height=args.side)
    view = bn.View(**wl)
    if args.tune:
        from blackhole_native import autotune

        best = autotune.tune(db, [view], "image1024", log=lambda m: print(m, file=sys.stderr, flush=True))
        print(json.dumps({"autotune": "image1024", "best": best.__dict__, "cache": str(autotune.CACHE)}), flush=True)
        return None
    cfg = bn.RenderConfig(**args.config) if args.config else None
    if cfg is None:
        from blackhole_native import autotune

        cfg = autotune.cached_config("image1024", device) or bn.RenderConfig()
    rnd = bn.Renderer(db, [view], config=cfg, precision="fp32")
    stream = torch.cuda.current_stream(device)

    fp32_peak_tflops = fp32_peak(device, stream)

    rnd.capture()
    for _ in range(args.warmup):
        rnd.graph_launch()
    torch.cuda.synchronize(device)
    st = rnd.result().stats()
    steps_per_launch, brick_steps, rays = st.ray_steps, st.brick_steps, st.rays

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(device).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid).start()
    time.sleep(0.3)
    K = args.steps
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(K + 1)]
    barrier(world)
    torch.cuda.synchronize(device)
    evs[0].record(stream)
    for i in range(K):
        rnd.graph_launch()
        evs[i + 1].record(stream)
    torch.cuda.synchronize(device)
    barrier(world)
    clk = clocks.stop()
    per_launch_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(K)]
    total_ms = evs[0].elapsed_time(evs[K])
    st2 = rnd.result().stats()
    assert st2.ray_steps == steps_per_launch, "ray-step count changed between launches"
    t_max = max_over_ranks(total_ms, world, device)
    all_steps = sum_over_ranks(steps_per_launch * K, world, device)
    value = all_steps / (t_max * 1e-3)

    # end to end through the public API with host buffers, every step: pinned
    # brick values -> device (copy + repack) -> render -> Stokes image back to
    # pinned host, with PipelinedRenderer overlapping step k's render with
    # step k + 1's upload and step k - 1's download
    e2e = None
    if not args.no_e2e:
        pinned = torch.from_numpy(brick_h.coeffs.reshape(-1)).pin_memory()
        pipe = bn.PipelinedRenderer(db, [view], config=cfg, precision="fp32")
        host_outs = [torch.empty(pipe.out_shape, dtype=pipe.out_dtype).pin_memory() for _ in range(2)]
        pipe.run([pinned] * 3, host_outs)
        torch.cuda.synchronize(device)
        ke = max(3, min(K, 10))
        barrier(world)
        torch.cuda.synchronize(device)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        pipe.run([pinned] * ke, host_outs)
        a1.record(stream)
        torch.cuda.synchronize(device)
        barrier(world)
        te = max_over_ranks(a0.elapsed_time(a1), world, device)
        ref_img = rnd.out.cpu()
        assert all(torch.equal(h, ref_img) for h in host_outs), "pipelined images differ from the device render"
        e2e = {"value": sum_over_ranks(steps_per_launch * ke, world, device) / (te * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": int(pinned.numel() * pinned.element_size()),
               "d2h_bytes_per_step": int(host_outs[0].numel() * host_outs[0].element_size()),
               "ms_per_step": te / ke, "pipelined": True}
        pipe.release()
        del pinned, host_outs, pipe

    kernel_s = statistics.mean(per_launch_ms) * 1e-3
    traffic = profiled_traffic()
    roofline, roofline_fp32 = render_rooflines(
        steps_per_launch, brick_steps, rays, kernel_s, fp32_peak_tflops,
        traffic if view.width == 1024 else None,
        f"not measured in this run: dram__bytes_read.sum + dram__bytes_write.sum of one timed launch of this "
        f"workload from the ncu capture summarised in {PROFILE_SUMMARY.relative_to(REPO)}" if traffic else None)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(brick_h, args.cpu_seconds)

    # accuracy of the timed method (outside the timed region): a quarter-size
    # crop from just outside the shadow through the torus image (3.75 M to
    # 13.75 M right of centre) against the FP64 kernel at h/4, and the FP32
    # Hamiltonian drift there
    accuracy = None
    if rank == 0 and not args.no_accuracy:
        from blackhole_native import studies

        db64 = bn.DeviceBrick(brick_h, device=device, precisions=("fp32", "fp64"))
        crop = (view.width // 2 + view.width * 3 // 32, view.height // 2 - view.height // 8, view.width // 4,
                view.height // 4)
        accuracy = studies.fine_step_check(db64, view, crop, config=cfg)
        del db64

    # the second half of the metric (outside the timed region, rank 0 of a 1-GPU run):
    # time to a 2048^2 image at <= 1e-3 Stokes-I rel L1, learned step size
    # against the step-doubling controller and the fastest plain step
    tti = None
    if rank == 0 and world == 1 and not args.no_time_to_image:
        tti = time_to_image(device, 2048, 3)
    # the batched-views workload in brief (the full record is `--workload views`): the
    # 256 seeded uneven views in one CUDA-graph launch, aggregate rate
    views_block = None
    if rank == 0 and world == 1 and not args.no_views:
        views_block = views_summary(device, K=3)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": t_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"plain fused kernel at scale: {view.width}x{view.height} rays, r_obs=1000M, "
                               "i=17deg, FOV +-20M, a=0.9375, RK2 h=0.02r in [1e-3,1], max_steps=4096, "
                               "256x128x256x11 float32 seeded torus brick",
                   "rays_per_step": rays, "ray_steps_per_step": steps_per_launch,
                   "brick_steps_per_step": brick_steps, "l2": "inputs larger than L2 (403 MB brick records)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "launch": {"block_threads": cfg.block_threads, "blocks_per_sm": cfg.blocks_per_sm,
                              "tile": [cfg.tile_w, cfg.tile_h], "refill_min": cfg.refill_min,
                              "cuda_graph": True}},
        "e2e": e2e, "gpu_launches": K, "clocks": clk, "roofline": roofline, "roofline_fp32": roofline_fp32,
        "cpu_baseline": cpu,
        "kernel_ms": {"mean": statistics.mean(per_launch_ms), "min": min(per_launch_ms), "max": max(per_launch_ms)},
        "status_counts": st2.status,
        "h_drift": {"max_all_rays": st2.max_h_drift, "max_escaped_rays": st2.max_h_drift_escaped},
        "accuracy": accuracy,
        "time_to_image": tti,
        "views": views_block,
    }
    rnd.release_graph()
    if world > 1:
        import torch.distributed as td

        td.destroy_process_group()
    return line if rank == 0 else None


def views_summary(device, K: int = 3) -> dict:
    """The 256-view batched launch (scenes.uneven_views(256, seed=0) through the
    shared 128x64x128x11 brick, autotuned shape, CUDA graph): ray-steps/s over
    K timed launches after 3 warm-up launches, with its own clock record."""
    import torch

    import blackhole_native as bn
    from blackhole_native import autotune, scenes

    db = bn.DeviceBrick(scenes.shared_brick(), device=device, precisions=("fp32",))
    views = scenes.uneven_views(256, seed=0)
    cfg = autotune.cached_config("views256", device) or bn.RenderConfig()
    rnd = bn.Renderer(db, views, config=cfg, precision="fp32")
    stream = torch.cuda.current_stream(device)
    rnd.capture()
    for _ in range(3):
        rnd.graph_launch()
    torch.cuda.synchronize(device)
    st = rnd.result().stats()
    clocks = ClockSampler(_uuid(device)).start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(K):
        rnd.graph_launch()
    e1.record(stream)
    torch.cuda.synchronize(device)
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / K
    rnd.release_graph()
    return {"workload": "256 seeded uneven views (side 64-1024, a~U(0,0.998), incl~U(5,85)deg, "
                        "max_steps~U{512..8192}), shared 128x64x128x11 float32 brick, one CUDA-graph launch",
            "value": st.ray_steps / (ms * 1e-3), "unit": UNIT, "ms_per_launch": ms, "launches": K,
            "ray_steps_per_launch": st.ray_steps, "rays": st.rays, "status_counts": st.status, "clocks": clk}


def bench_views(args) -> dict | None:
    """Many uneven views (seeded: side 64..1024, a ~ U(0, 0.998), inclination
    ~ U(5, 85) deg, max_steps ~ U{512..8192}) through one shared 128x64x128x11
    float32 brick, all in one persistent CUDA-graph launch."""
    import torch

    import blackhole_native as bn
    from blackhole_native import autotune, scenes

    rank, world, local_rank = dist_env()
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    init_dist(world, "nccl")
    db = bn.DeviceBrick(scenes.shared_brick(), device=device, precisions=("fp32",))
    views = scenes.uneven_views(args.n_views, seed=0)
    key = f"views{args.n_views}"
    if args.tune:
        space = dict(autotune.DEFAULT_SPACE, block_threads=(128, 256), blocks_per_sm=(2, 4))
        best = autotune.tune(db, views[:48], key, space=space, repeats=2,
                             log=lambda m: print(m, file=sys.stderr, flush=True))
        print(json.dumps({"autotune": key, "best": best.__dict__, "cache": str(autotune.CACHE)}), flush=True)
        return None
    cfg = bn.RenderConfig(**args.config) if args.config else (autotune.cached_config(key, device) or bn.RenderConfig())
    rnd = bn.Renderer(db, views, config=cfg, precision="fp32")
    stream = torch.cuda.current_stream(device)
    fp32_peak_tflops = fp32_peak(device, stream)
    rnd.capture()
    for _ in range(args.warmup):
        rnd.graph_launch()
    torch.cuda.synchronize(device)
    st = rnd.result().stats()
    K = args.steps
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(K + 1)]
    clocks = ClockSampler(_uuid(device)).start()
    time.sleep(0.3)
    barrier(world)
    torch.cuda.synchronize(device)
    evs[0].record(stream)
    for i in range(K):
        rnd.graph_launch()
        evs[i + 1].record(stream)
    torch.cuda.synchronize(device)
    barrier(world)
    clk = clocks.stop()
    total_ms = evs[0].elapsed_time(evs[K])
    t_max = max_over_ranks(total_ms, world, device)
    value = sum_over_ranks(st.ray_steps * K, world, device) / (t_max * 1e-3)
    rnd.release_graph()
    roofline, roofline_fp32 = render_rooflines(st.ray_steps, st.brick_steps, st.rays, total_ms / K * 1e-3,
                                               fp32_peak_tflops, None, None)
    # per view, each rendered alone (same launch shape)
    per_view = []
    for v in views:
        r1 = bn.Renderer(db, [v], config=cfg, precision="fp32")
        r1.launch()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        r1.launch()
        b.record(stream)
        b.synchronize()
        s1 = r1.result().stats()
        per_view.append(s1.ray_steps / (a.elapsed_time(b) * 1e-3))
    pv = np.asarray(per_view)
    h_drift = accuracy = cpu = None
    if rank == 0:
        from blackhole_native import studies

        # Hamiltonian drift of every ray of the batch (one untimed launch with per-ray outputs)
        rr = bn.Renderer(db, views, config=cfg, precision="fp32", ray_outputs=True).launch()
        torch.cuda.synchronize(device)
        h_drift = studies._drift_summary(rr.h_drift.cpu().numpy().astype(np.float64), rr.status.cpu().numpy())
        del rr
        if not args.no_accuracy:
            # Stokes error against the FP64 kernel at h/4 on a crop through the torus
            # image (right of the shadow, at most 128^2: the image workload's crop) of four views
            db64 = bn.DeviceBrick(scenes.shared_brick(), device=device, precisions=("fp32", "fp64"))
            per = []
            for v in views[:4]:
                w, h = min(max(v.width // 4, 16), 128), min(max(v.height // 4, 16), 128)
                x0 = min(v.width // 2 + v.width * 3 // 32, v.width - w)
                y0 = max(v.height // 2 - v.height // 8, 0)
                per.append(studies.fine_step_check(db64, v, (x0, y0, w, h), config=cfg))
            keys = ("rel_l1_I", "rel_l1_Q", "rel_l1_U", "rel_l1_V", "flux_weighted_dm")
            accuracy = {"views": [{"side": [v.width, v.height], "spin_a": v.spin_a, "inclination_deg": v.inclination_deg,
                                   "crop": a["crop"], "mask_fraction": a["mask_fraction"]["fine_step"],
                                   **a["fp32_vs_fp64_fine"]} for v, a in zip(views[:4], per)],
                        "max": {k: max(a["fp32_vs_fp64_fine"][k] for a in per) for k in keys},
                        "fine_step_factor": 0.25}
            del db64
        if world == 1 and not args.no_cpu_baseline:
            cpu = views_cpu_baseline(scenes.shared_brick(), views, args.cpu_seconds)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": t_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"batched persistent launch: {len(views)} seeded views (side 64-1024, a~U(0,0.998), "
                               "incl~U(5,85)deg, max_steps~U{512..8192}), shared 128x64x128x11 float32 brick, "
                               "one CUDA-graph launch",
                   "rays_per_step": st.rays, "ray_steps_per_step": st.ray_steps,
                   "brick_steps_per_step": st.brick_steps,
                   "l2": "brick records (18 MB) fit in L2; the 1.03e8 rays' Stokes outputs (1.6 GB) do not",
                   "autotune": {"block_threads": cfg.block_threads, "blocks_per_sm": cfg.blocks_per_sm,
                                "tile": [cfg.tile_w, cfg.tile_h], "refill_min": cfg.refill_min,
                                "reg_cap": cfg.reg_cap}},
        "per_view_ray_steps_per_s": {"min": float(pv.min()), "median": float(np.median(pv)),
                                     "max": float(pv.max()), "views": len(pv)},
        "status_counts": st.status, "gpu_launches": K, "clocks": clk, "roofline": roofline,
        "roofline_fp32": roofline_fp32, "cpu_baseline": cpu, "h_drift": h_drift, "accuracy": accuracy,
        "e2e": None,
    }
    if world > 1:
        import torch.distributed as td

        td.destroy_process_group()
    return line if rank == 0 else None


def views_cpu_baseline(brick, views, target_s: float) -> dict:
    """The FP64 oracle (C, OpenMP over every host core) on centred crops of the
    batch's views, as many views as fit in about target_s seconds."""
    sys.path.insert(0, str(REPO))
    from oracle import oracle as O

    steps, spent, used = 0, 0.0, 0
    for v in views:
        n = min(24, v.width, v.height)
        ov = O.make_view(spin_a=v.spin_a, r_obs=v.r_obs, theta_obs=math.radians(v.inclination_deg), phi_obs=0.0,
                         fov_y_deg=v.fov_y_deg, roll_deg=0.0, h_scale=v.h_scale, h_min=v.h_min, h_max=v.h_max,
                         escape_radius=v.escape_radius, affine_to_length_cm=1.0, max_optical_depth=30.0,
                         width=v.width, height=v.height, x0=(v.width - n) // 2, y0=(v.height - n) // 2, crop_w=n,
                         crop_h=n, max_steps=v.max_steps)
        t0 = time.perf_counter()
        _, st, _, _ = O.render(ov, brick.coeffs, brick.r, brick.theta, brick.phi, stop_at_tau=True)
        spent += time.perf_counter() - t0
        steps += int(st.sum())
        used += 1
        if spent >= target_s:
            break
    return {"value": steps / spent, "unit": UNIT, "cores": O.max_threads(), "kind": "port",
            "sample": f"float64 oracle (C, OpenMP): centred 24x24 crops of the first {used} views, {steps} "
                      f"ray-steps in {spent:.2f} s"}


# ------------------------------------------------------------------ synchrotron workloads
PRECOMPUTE = dict(nr=256, ntheta=128, nphi=256, spin_a=0.9375, seed=5, nu_hz=230e9)
PRECOMPUTE_PROFILE = REPO / "profiles" / "precompute_kernel_snapshot_2M_cells.md"
PRECOMPUTE_PROFILE_CELLS = 64 * 128 * 256   # the captured case; its traffic scales with the cells
GRRT_SNAPSHOT = dict(nr=64, ntheta=32, nphi=64, spin_a=0.9375, seed=0)
GRRT_PROFILE = REPO / "profiles" / "grrt_kernel_default_image.md"   # the snapshot is read once per launch
# calibration.PhysicalScaling of a 4.3e6 solar-mass hole at 8.3 kpc with code units rho 3e-18 g/cm^3, B 25 G
SCALING = dict(mass_bh_g=8.54e39, distance_cm=2.57e22, rho_cgs_per_code=3.0e-18, b_gauss_per_code=25.0)


def fp64_peaks(device, stream) -> dict:
    """FP64 FMA TFLOP/s and double exp() evaluations/s of this GPU (bhn_fp64_peak_probe)."""
    import ctypes

    import torch

    from blackhole_native import _lib

    L = _lib.lib()
    probe = torch.empty(1 << 20, dtype=torch.float64, device=device)
    out = {}
    for mode, iters, key in ((0, 2048, "fma_tflops"), (1, 512, "exp_per_s")):
        ops = ctypes.c_int64()
        for _ in range(2):
            _lib.check(L.bhn_fp64_peak_probe(probe.data_ptr(), iters, 8, mode, ctypes.byref(ops), stream.cuda_stream))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _lib.check(L.bhn_fp64_peak_probe(probe.data_ptr(), iters, 8, mode, ctypes.byref(ops), stream.cuda_stream))
        e1.record(stream)
        torch.cuda.synchronize(device)
        rate = ops.value / (e0.elapsed_time(e1) * 1e-3)
        out[key] = rate / 1e12 if mode == 0 else rate
    return out


def exps_per_evaluation(model_struct) -> int:
    """Double exp() calls of the kernel-table lookups one coefficient
    evaluation needs: F and G at every Lorentz-factor node and distinct pitch
    angle of each component (the Gauss-Legendre nodes +-mu share sin(alpha),
    so an n-node rule has (n + 1) // 2 distinct angles)."""
    m = model_struct
    n = 0
    if m.thermal:
        n += m.thermal_gamma_n * ((m.thermal_pitch_n + 1) // 2)
    if m.nonthermal:
        n += m.nonthermal_gamma_n * ((m.nonthermal_pitch_n + 1) // 2)
    return 2 * n


def exp_roofline(evals: float, seconds: float, peaks: dict, per_eval: int, kernel: str) -> dict:
    achieved = evals * per_eval / seconds
    return {"bound": "fp64-exp", "achieved": round(achieved / 1e9, 2), "peak": round(peaks["exp_per_s"] / 1e9, 2),
            "unit": "Gexp/s", "frac": round(achieved / peaks["exp_per_s"], 4), "traffic": None,
            "peak_source": "measured in this run (bhn_fp64_peak_probe, 8 chains of x <- exp(-x) per thread)",
            "kernel": kernel, "exp_per_unit": per_eval,
            "fp64_fma_tflops_measured": round(peaks["fma_tflops"], 2)}


def timed_launches(fn, k: int, stream, device) -> list[float]:
    import torch

    evs = [torch.cuda.Event(enable_timing=True) for _ in range(k + 1)]
    torch.cuda.synchronize(device)
    evs[0].record(stream)
    for i in range(k):
        fn()
        evs[i + 1].record(stream)
    torch.cuda.synchronize(device)
    return [evs[i].elapsed_time(evs[i + 1]) for i in range(k)]


def bench_precompute(args) -> dict | None:
    """Coefficient-brick precompute (coefficient_bricks.py:119-152, Hybrid
    model): one step = every cell of a 256 x 128 x 256 seeded snapshot to an
    [nr][nt][np][11] float32 brick."""
    import ctypes

    import torch

    from blackhole_native import _device as dev
    from blackhole_native import grrt, synchrotron as syn

    rank, world, local_rank = dist_env()
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    init_dist(world, "nccl")
    stream = torch.cuda.current_stream(device)
    P = dict(PRECOMPUTE)
    if args.side:  # fewer r shells of the same snapshot layout (profiling runs)
        P["nr"] = args.side
    snap = grrt.seeded_snapshot(P["nr"], P["ntheta"], P["nphi"], P["spin_a"], P["seed"])
    scaling = grrt.PhysicalScaling(**SCALING)
    cells = P["nr"] * P["ntheta"] * P["nphi"]
    L = syn._declare()
    m = syn.model_struct(syn.HybridSynchrotronCoefficients(), P["nu_hz"], scaling)
    d_rho = torch.from_numpy(np.ascontiguousarray(snap.rho)).to(device)
    d_te = torch.from_numpy(np.ascontiguousarray(snap.theta_e)).to(device)
    d_b = torch.from_numpy(np.ascontiguousarray(snap.b_con)).to(device)
    out = torch.empty((P["nr"], P["ntheta"], P["nphi"], 11), dtype=torch.float32, device=device)

    def launch():
        _lib_check(L.bhn_brick_precompute(dev.ptr(d_rho), dev.ptr(d_te), dev.ptr(d_b), cells, ctypes.byref(m),
                                          dev.ptr(out), 4, stream.cuda_stream))

    peaks = fp64_peaks(device, stream)
    for _ in range(args.warmup):
        launch()
    torch.cuda.synchronize(device)
    assert bool(torch.isfinite(out).all()), "non-finite coefficients"
    clocks = ClockSampler(_uuid(device)).start()
    time.sleep(0.3)
    barrier(world)
    per = timed_launches(launch, args.steps, stream, device)
    barrier(world)
    clk = clocks.stop()
    t_max = max_over_ranks(sum(per), world, device)
    value = sum_over_ranks(cells * args.steps, world, device) / (t_max * 1e-3)

    e2e = None
    if not args.no_e2e:  # public API with host arrays: fields up, brick back to host
        ke = max(1, min(args.steps, 3))
        ref = out.cpu().numpy()
        syn.precompute_coefficient_bricks(snap, scaling, P["nu_hz"])
        barrier(world)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        a0.record(stream)
        for _ in range(ke):
            brick = syn.precompute_coefficient_bricks(snap, scaling, P["nu_hz"])
        a1.record(stream)
        torch.cuda.synchronize(device)
        barrier(world)
        te = max_over_ranks(a0.elapsed_time(a1), world, device)
        assert np.array_equal(brick.coeffs, ref), "public-API brick differs from the device launch"
        e2e = {"value": sum_over_ranks(cells * ke, world, device) / (te * 1e-3), "unit": "cells/s",
               "h2d_bytes_per_step": int(cells * 6 * 8), "d2h_bytes_per_step": int(cells * 11 * 4),
               "ms_per_step": te / ke, "api": "precompute_coefficient_bricks"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = precompute_cpu_baseline(snap, scaling, args.cpu_seconds)
    per_mean = statistics.mean(per)
    line = {
        "metric": "cells/s", "value": value, "unit": "cells/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"coefficient-brick precompute, Hybrid synchrotron model at 230 GHz: "
                               f"{P['nr']}x{P['ntheta']}x{P['nphi']} seeded GRMHD-like snapshot -> float32 "
                               "[nr][nt][np][11] brick",
                   "cells_per_step": cells, "l2": f"inputs larger than L2 ({cells * 48 / 1e6:.0f} MB of float64 fields)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "e2e": e2e, "gpu_launches": args.steps, "clocks": clk,
        "roofline": dict(exp_roofline(cells, per_mean * 1e-3, peaks, exps_per_evaluation(m), "precompute_kernel"),
                         traffic=_scaled_traffic(PRECOMPUTE_PROFILE, cells / PRECOMPUTE_PROFILE_CELLS)),
        "cpu_baseline": cpu,
        "kernel_ms": {"mean": per_mean, "min": min(per), "max": max(per)},
    }
    if world > 1:
        import torch.distributed as td

        td.destroy_process_group()
    return line if rank == 0 else None


def precompute_cpu_baseline(snap, scaling, target_s: float) -> dict:
    """The float64 oracle (per-cell numpy loop, one core) on a run of cells."""
    sys.path.insert(0, str(REPO))
    from oracle import synchrotron as S

    rho = snap.rho.reshape(-1)
    te = snap.theta_e.reshape(-1)
    b = snap.b_con.reshape(-1, 4)
    start = rho.size // 2

    def run(n):
        sl = slice(start, start + n)
        t0 = time.perf_counter()
        S.precompute(rho[sl].reshape(1, 1, n), te[sl].reshape(1, 1, n), b[sl].reshape(1, 1, n, 4),
                     PRECOMPUTE["nu_hz"], scaling.rho_cgs_per_code, scaling.b_gauss_per_code)
        return time.perf_counter() - t0

    dt = run(4)
    n = max(4, min(20000, int(4 * max(target_s, 0.5) / max(dt, 1e-4))))
    dt = run(n)
    return {"value": n / dt, "unit": "cells/s", "cores": 1, "kind": "port",
            "sample": f"float64 oracle (oracle/synchrotron.py, numpy per cell, one core): {n} cells of the same "
                      f"snapshot in {dt:.2f} s"}


def bench_grrt(args) -> dict | None:
    """Physical polarized GRRT (polarized_renderer.render_stokes_image): one
    step = the reference's default 160 x 90 image (camera r = 55 M, i = 65 deg,
    FOV 32 deg, RK4 step 0.06, 5000 steps, RK2 Stokes steps) of a seeded
    64 x 32 x 64 snapshot."""
    import torch

    from blackhole_native import grrt

    rank, world, local_rank = dist_env()
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    init_dist(world, "nccl")
    stream = torch.cuda.current_stream(device)
    G = GRRT_SNAPSHOT
    snap = grrt.seeded_snapshot(G["nr"], G["ntheta"], G["nphi"], G["spin_a"], G["seed"])
    scaling = grrt.PhysicalScaling(**SCALING)
    cfg = grrt.PolarizedRenderConfig()
    if args.side:  # a smaller image of the same scene (profiling runs)
        cfg = grrt.PolarizedRenderConfig(width=args.side, height=max(1, round(args.side * 9 / 16)))
    ds = grrt.DeviceSnapshot(snap, device)
    pixels = cfg.width * cfg.height
    img, diag = grrt.render_stokes_image_device(cfg, ds, scaling, diagnostics=True)
    torch.cuda.synchronize(device)
    d = diag.cpu().numpy()
    segments, steps = float(d[..., 1].sum()), float(d[..., 6].sum())
    out = torch.empty_like(img)
    peaks = fp64_peaks(device, stream)
    for _ in range(args.warmup):
        grrt.render_stokes_image_device(cfg, ds, scaling, out=out)
    clocks = ClockSampler(_uuid(device)).start()
    time.sleep(0.3)
    barrier(world)
    per = timed_launches(lambda: grrt.render_stokes_image_device(cfg, ds, scaling, out=out), args.steps, stream,
                         device)
    barrier(world)
    clk = clocks.stop()
    assert torch.equal(out, img), "images differ between launches"
    t_max = max_over_ranks(sum(per), world, device)
    value = sum_over_ranks(pixels * args.steps, world, device) / (t_max * 1e-3)

    e2e = None
    if not args.no_e2e:  # public API: host snapshot in, host image out
        ke = max(1, min(args.steps, 3))
        barrier(world)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        a0.record(stream)
        for _ in range(ke):
            host = grrt.render_stokes_image(cfg, snap, scaling)
        a1.record(stream)
        torch.cuda.synchronize(device)
        barrier(world)
        te = max_over_ranks(a0.elapsed_time(a1), world, device)
        assert np.array_equal(host, img.cpu().numpy()), "public-API image differs from the device launch"
        e2e = {"value": sum_over_ranks(pixels * ke, world, device) / (te * 1e-3), "unit": "pixels/s",
               "h2d_bytes_per_step": ds.upload_bytes, "d2h_bytes_per_step": int(pixels * 4 * 8),
               "ms_per_step": te / ke, "api": "render_stokes_image"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = grrt_cpu_baseline(snap, scaling, cfg, args.cpu_seconds)
    m = grrt.model_struct(grrt.HybridSynchrotronCoefficients(), cfg.transfer.observing_frequency_hz, scaling)
    chunk = grrt.default_chunk(pixels)
    launches_per_image = 1 + 3 * (cfg.max_steps // chunk + 2)  # init, then trace / coefficient / transfer rounds
    per_mean = statistics.mean(per)
    line = {
        "metric": "pixels/s", "value": value, "unit": "pixels/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"physical polarized GRRT, default render config: {cfg.width}x{cfg.height} pixels, "
                               "camera r=55M i=65deg FOV 32deg, RK4 step 0.06, 5000 steps, RK2 Stokes steps, "
                               f"Hybrid synchrotron at 230 GHz, seeded {G['nr']}x{G['ntheta']}x{G['nphi']} snapshot",
                   "pixels_per_step": pixels, "emitting_segments_per_step": segments, "rk4_steps_per_step": steps,
                   "segments_per_ray_and_round": chunk,
                   "l2": "snapshot (11.5 MB) resident in L2; the work is per-segment arithmetic",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "e2e": e2e, "gpu_launches": args.steps * launches_per_image, "clocks": clk,
        "roofline": dict(exp_roofline(segments, per_mean * 1e-3, peaks, exps_per_evaluation(m),
                                      "grrt_coef_kernel (timed: the whole render, all rounds of the trace, "
                                      "coefficient and transfer kernels)"),
                         traffic=profiled_traffic(GRRT_PROFILE)),
        "cpu_baseline": cpu,
        "kernel_ms": {"mean": per_mean, "min": min(per), "max": max(per)},
    }
    if world > 1:
        import torch.distributed as td

        td.destroy_process_group()
    return line if rank == 0 else None


def grrt_cpu_baseline(snap, scaling, cfg, target_s: float) -> dict:
    """The float64 oracle (oracle/grrt.py, one core) on pixels of the image's middle row."""
    sys.path.insert(0, str(REPO))
    from blackhole_native import grrt
    from oracle import grrt as OG
    from oracle import oracle as O

    cam = cfg.camera
    v = O.View()
    v.spin_a, v.r_obs, v.theta_obs, v.phi_obs = snap.spin_a, cam.r, cam.theta, cam.phi
    v.fov_y_deg, v.roll_deg, v.width, v.height = cam.fov_y_degrees, cam.roll_degrees, cfg.width, cfg.height
    fields = grrt.snapshot_fields(snap)
    sc = {"rho_cgs_per_code": scaling.rho_cgs_per_code, "b_gauss_per_code": scaling.b_gauss_per_code}
    t0 = time.perf_counter()
    n = segs = 0
    py = cfg.height // 2
    while n < cfg.width and (n == 0 or time.perf_counter() - t0 < target_s):
        px = (cfg.width // 2 + n) % cfg.width
        _, (_, emit, _) = OG.trace_pixel(v, fields, snap.r, snap.theta, snap.phi, sc,
                                         cfg.transfer.observing_frequency_hz, cfg.step, cfg.max_steps,
                                         cfg.escape_radius, length_cm=scaling.rg_cm, px=px, py=py)
        n += 1
        segs += emit
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "pixels/s", "cores": 1, "kind": "port",
            "sample": f"float64 oracle (oracle/grrt.py, one core): {n} pixels of the middle row "
                      f"({segs} emitting segments) in {dt:.2f} s"}


# The reference's own brick renderer (accelerated_renderer.render_stokes_image_bricks)
BRICKS_BRICK = dict(nr=128, ntheta=64, nphi=128, spin_a=0.9375, seed=0)
BRICKS_PROFILE = REPO / "profiles" / "brick_trace_kernel_default_image.md"
# FP64 FLOP of the fixed-step method (a multiply or add = 1, an FMA = 2, a
# divide / sqrt / sincos = 1): an RK4 step is four right-hand sides of 129
# (metric, three reciprocals, both quotient-rule derivatives) plus the stage
# arguments and the update; a sampled segment adds the midpoint, the weights,
# the 11-channel trilinear sample (7 lerps x 11 x 3), ds, the Stokes RK2 step
# and the optical depth.
FP64_FLOP_PER_RK4_STEP = 577
FP64_FLOP_PER_SEGMENT = 336


def bench_bricks(args) -> dict | None:
    """The reference's brick renderer (accelerated_renderer.py:100-158): one
    step = its default 160 x 90 image (camera r = 55 M, i = 65 deg, FOV 32
    deg, RK4 step 0.06, 5000 steps, RK2 Stokes steps) of a seeded
    128 x 64 x 128 x 11 float32 torus brick, FP64, one thread per ray."""
    from types import SimpleNamespace

    import torch

    from blackhole_native import accelerated as acc
    from blackhole_native import bricks

    rank, world, local_rank = dist_env()
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    init_dist(world, "nccl")
    stream = torch.cuda.current_stream(device)
    B = BRICKS_BRICK
    b = bricks.torus_brick(B["nr"], B["ntheta"], B["nphi"], spin_a=B["spin_a"], seed=B["seed"], dtype=np.float32)
    grid = SimpleNamespace(r=b.r, theta=b.theta, phi=b.phi, coeffs=b.coeffs)
    snap = SimpleNamespace(spin_a=B["spin_a"])
    cfg = acc.AcceleratedRenderConfig()
    if args.side:  # a larger or smaller image of the same scene
        cfg = acc.AcceleratedRenderConfig(width=args.side, height=max(1, round(args.side * 9 / 16)))
    db = acc.DeviceBricks(grid, device)
    pixels = cfg.width * cfg.height
    img, diag = acc.render_stokes_image_bricks_device(cfg, snap, db, diagnostics=True)
    full_img, full_diag = acc.render_stokes_image_bricks_device(cfg, snap, db, diagnostics=True, full_trace=True)
    torch.cuda.synchronize(device)
    assert torch.equal(full_img, img), "the outbound exit changed the image"
    d, fd = diag.cpu().numpy(), full_diag.cpu().numpy()
    steps, segments = float(d[..., 2].sum()), float(d[..., 1].sum())
    peaks = fp64_peaks(device, stream)
    for _ in range(args.warmup):
        acc.render_stokes_image_bricks_device(cfg, snap, db)
    clocks = ClockSampler(_uuid(device)).start()
    time.sleep(0.3)
    barrier(world)
    outs = []
    # unchecked launches (no read-back inside the timed region); every image is compared with the checked one below
    per = timed_launches(lambda: outs.append(acc.render_stokes_image_bricks_device(cfg, snap, db, check=False)),
                         args.steps, stream, device)
    barrier(world)
    clk = clocks.stop()
    assert all(torch.equal(o, img) for o in outs), "images differ between launches"
    t_max = max_over_ranks(sum(per), world, device)
    value = sum_over_ranks(pixels * args.steps, world, device) / (t_max * 1e-3)
    # the same image with every ray traced to the reference's own end (escape radius 220, capture, max_steps)
    full_outs = []
    per_full = timed_launches(lambda: full_outs.append(acc.render_stokes_image_bricks_device(
        cfg, snap, db, full_trace=True, check=False)), args.steps, stream, device)
    assert all(torch.equal(o, img) for o in full_outs), "full-trace images differ"
    full_trace = {"ms_per_step": statistics.mean(per_full), "pixels_per_s": pixels / (statistics.mean(per_full) * 1e-3),
                  "rk4_steps_per_step": float(fd[..., 2].sum()), "longest_ray_steps": int(fd[..., 2].max()),
                  "note": "full_trace=True: rays also traced past the brick to the escape radius; same image"}

    e2e = None
    if not args.no_e2e:  # public API: host brick in (float32, uploaded and widened on the device), host image out
        ke = max(1, min(args.steps, 3))
        acc.render_stokes_image_bricks(cfg, snap, grid)  # untimed warm-up call of the public path
        barrier(world)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        a0.record(stream)
        for _ in range(ke):
            host = acc.render_stokes_image_bricks(cfg, snap, grid)
        a1.record(stream)
        torch.cuda.synchronize(device)
        barrier(world)
        te = max_over_ranks(a0.elapsed_time(a1), world, device)
        assert np.array_equal(host, img.cpu().numpy()), "public-API image differs from the device launch"
        h2d = int(b.coeffs.nbytes + (b.r.size + b.theta.size + b.phi.size) * 8)  # the brick in its own dtype
        e2e = {"value": sum_over_ranks(pixels * ke, world, device) / (te * 1e-3), "unit": "pixels/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(pixels * 4 * 8), "ms_per_step": te / ke,
               "api": "render_stokes_image_bricks"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = bricks_cpu_baseline(grid, snap, cfg, args.cpu_seconds)
    per_mean = statistics.mean(per)
    flops = FP64_FLOP_PER_RK4_STEP * steps + FP64_FLOP_PER_SEGMENT * segments
    achieved = flops / (per_mean * 1e-3) / 1e12
    line = {
        "metric": "pixels/s", "value": value, "unit": "pixels/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"reference brick renderer (render_stokes_image_bricks), {cfg.width}x{cfg.height} "
                               "pixels, camera r=55M i=65deg FOV 32deg, RK4 step 0.06, 5000 steps, RK2 Stokes "
                               f"steps, seeded {B['nr']}x{B['ntheta']}x{B['nphi']}x11 float32 torus brick",
                   "pixels_per_step": pixels, "rk4_steps_per_step": steps, "sampled_segments_per_step": segments,
                   "longest_ray_steps": int(d[..., 2].max()),
                   "outbound_exit": "a ray past the brick's outer radius moving out with no radial turning point "
                                    "ahead ends there (nothing later is sampled; image bit-identical to full traces)",
                   "l2": "brick (92 MB of float64 coefficients) resident in L2 between launches; the rays read "
                         "at most a few cells per step",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "e2e": e2e, "gpu_launches": args.steps * 2,  # setup_views_kernel + brick_trace_kernel
        "clocks": clk,
        "roofline": {"bound": "fp64", "achieved": round(achieved, 3), "peak": round(peaks["fma_tflops"], 2),
                     "unit": "TFLOP/s", "frac": round(achieved / peaks["fma_tflops"], 4),
                     "traffic": profiled_traffic(BRICKS_PROFILE),
                     "traffic_source": f"ncu capture of the same workload ({BRICKS_PROFILE.relative_to(REPO)})",
                     "peak_source": "measured in this run (bhn_fp64_peak_probe FMA chains)",
                     "kernel": ("brick_trace_pair_kernel" if (pixels + 31) // 32 <= 4 * torch.cuda.get_device_properties(
                         device).multi_processor_count else "brick_trace_kernel"),
                     "algorithmic_flops_per_launch": flops,
                     "flop_per_rk4_step": FP64_FLOP_PER_RK4_STEP, "flop_per_segment": FP64_FLOP_PER_SEGMENT},
        "cpu_baseline": cpu,
        "kernel_ms": {"mean": per_mean, "min": min(per), "max": max(per), "all": [round(x, 3) for x in per]},
        "full_trace": full_trace,
    }
    if world > 1:
        import torch.distributed as td

        td.destroy_process_group()
    return line if rank == 0 else None


def bricks_cpu_baseline(grid, snap, cfg, target_s: float) -> dict:
    """The float64 oracle (oracle/bricktrace.py, one core) on pixels of the image's middle row."""
    sys.path.insert(0, str(REPO))
    from oracle import bricktrace as OB
    from oracle import oracle as O

    cam = cfg.camera
    v = O.View()
    v.spin_a, v.r_obs, v.theta_obs, v.phi_obs = snap.spin_a, cam.r, cam.theta, cam.phi
    v.fov_y_deg, v.roll_deg, v.width, v.height = cam.fov_y_degrees, cam.roll_degrees, cfg.width, cfg.height
    rg, tg, pg = (np.asarray(g, dtype=np.float32).astype(np.float64) for g in (grid.r, grid.theta, grid.phi))
    coeffs = np.asarray(grid.coeffs, dtype=np.float64)
    t0 = time.perf_counter()
    n = segs = 0
    py = cfg.height // 2
    while n < cfg.width and (n == 0 or time.perf_counter() - t0 < target_s):
        px = (cfg.width // 2 + n) % cfg.width
        _, (_, k) = OB.trace_pixel_bricks(v, coeffs, rg, tg, pg, cfg.step, cfg.max_steps, cfg.escape_radius,
                                          length_cm=1.0, px=px, py=py)
        n += 1
        segs += k
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "pixels/s", "cores": 1, "kind": "port",
            "sample": f"float64 oracle (oracle/bricktrace.py, one core): {n} pixels of the middle row "
                      f"({segs} sampled segments) in {dt:.2f} s"}


# The plugin's sample_and_step_stokes (native_kernels.py:325-407, lib.rs:308-366)
MICRO = dict(nr=256, ntheta=128, nphi=256, points=1 << 24, seed=0, ds_cm=0.05, e2e_points=1 << 20)
MICRO_PROFILE = REPO / "profiles" / "sample_and_step_kernel_16M_points.md"
# Algorithmic bytes per point: the (r, theta, phi) triple, the 8 corner cells'
# 11 float64 coefficients, the 4 float64 Stokes values written (the initial
# vector is broadcast).
MICRO_BYTES_PER_POINT = 3 * 8 + 8 * 11 * 8 + 4 * 8


def bench_micro(args) -> dict | None:
    """The plugin micro-kernel sample_and_step_stokes at scale: one step =
    16.8M seeded points inside a 256 x 128 x 256 x 11 float64 torus brick
    (738 MB, larger than L2), each sampled trilinearly and advanced by one
    Stokes RK2 step, FP64, on device tensors; e2e through the reference-facing
    call (host arrays in, the brick passed every call, a flat list out)."""
    import torch

    from blackhole_native import bricks, kernels

    rank, world, local_rank = dist_env()
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    init_dist(world, "nccl")
    stream = torch.cuda.current_stream(device)
    M = MICRO
    b = bricks.torus_brick(M["nr"], M["ntheta"], M["nphi"], spin_a=0.9375, seed=M["seed"], dtype=np.float64)
    n = int(args.side) * 1024 if args.side else M["points"]
    rng = np.random.default_rng(M["seed"] + 1)
    pts = np.empty((n, 3))
    pts[:, 0] = rng.uniform(b.r[0], b.r[-1], n)
    pts[:, 1] = rng.uniform(b.theta[0], b.theta[-1], n)
    pts[:, 2] = rng.uniform(0.0, 2.0 * math.pi, n)
    c = torch.as_tensor(b.coeffs.reshape(-1), device=device)
    rg, tg, pg = (torch.as_tensor(g, device=device) for g in (b.r, b.theta, b.phi))
    dp = torch.as_tensor(pts, device=device)
    ini = torch.zeros(4, dtype=torch.float64, device=device)
    ref = kernels.sample_and_step_stokes(c, rg, tg, pg, dp, M["ds_cm"], ini)  # the checked public tensor call
    out = torch.empty_like(ref)
    def launch():  # the public call's launch path (cell-ordered for large point sets), without its input checks
        kernels._launch_sample_and_step(c, rg, tg, pg, dp, n, M["ds_cm"], ini, 0, out)

    for _ in range(args.warmup):
        launch()
    clocks = ClockSampler(_uuid(device)).start()
    time.sleep(0.3)
    barrier(world)
    per = timed_launches(launch, args.steps, stream, device)
    barrier(world)
    clk = clocks.stop()
    assert torch.equal(out, ref), "outputs differ between launches"
    t_max = max_over_ranks(sum(per), world, device)
    value = sum_over_ranks(n * args.steps, world, device) / (t_max * 1e-3)

    e2e = None
    if not args.no_e2e:  # host numpy in, flat list out, the brick passed with every call (the reference's call)
        ne = min(n, M["e2e_points"])
        host = [b.coeffs.reshape(-1), b.r, b.theta, b.phi, pts[:ne]]
        ke = max(1, min(args.steps, 3))
        barrier(world)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        a0.record(stream)
        for _ in range(ke):
            lst = kernels.sample_and_step_stokes(*host, M["ds_cm"], [0.0, 0.0, 0.0, 0.0])
        a1.record(stream)
        torch.cuda.synchronize(device)
        barrier(world)
        te = max_over_ranks(a0.elapsed_time(a1), world, device)
        assert np.array_equal(np.asarray(lst), ref[: 4 * ne].cpu().numpy()), "list API differs from the tensor call"
        e2e = {"value": sum_over_ranks(ne * ke, world, device) / (te * 1e-3), "unit": "points/s",
               "h2d_bytes_per_step": int(sum(x.nbytes for x in host) + 32), "d2h_bytes_per_step": int(ne * 32),
               "ms_per_step": te / ke, "api": "sample_and_step_stokes (numpy in, list out)",
               "points_per_step": ne}

    # stokes_rk2_brick (lib.rs:210-279) over the whole brick: a streaming kernel,
    # 88 B of coefficients in and 32 B of Stokes out per cell
    from blackhole_native import _device as dev
    from blackhole_native import _lib

    cells = int(b.cells)
    rk_out = torch.empty(4 * cells, dtype=torch.float64, device=device)
    rk_ref = kernels.stokes_rk2_brick(c, M["ds_cm"], ini)  # the checked public tensor call

    def rk2():
        _lib.check(_lib.lib().bhn_stokes_rk2_brick(dev.ptr(c), cells, M["ds_cm"], dev.ptr(ini), 4, dev.ptr(rk_out),
                                                   stream.cuda_stream))

    for _ in range(args.warmup):
        rk2()
    rk_per = timed_launches(rk2, args.steps, stream, device)
    assert torch.equal(rk_out, rk_ref)
    rk_ms = statistics.mean(rk_per)
    rk_gbs = 120.0 * cells / (rk_ms * 1e-3) / 1e9
    peaks = load_peaks()
    stokes_rk2 = {"cells_per_step": cells, "ms_per_step": rk_ms, "cells_per_s": cells / (rk_ms * 1e-3),
                  "roofline": {"bound": "hbm", "achieved": round(rk_gbs, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                               "frac": round(rk_gbs / peaks["hbm_gbs"], 4), "kernel": "stokes_rk2_brick_kernel",
                               "algorithmic_bytes_per_cell": 120}}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = micro_cpu_baseline(b, pts, M["ds_cm"], args.cpu_seconds)
    per_mean = statistics.mean(per)
    achieved = MICRO_BYTES_PER_POINT * n / (per_mean * 1e-3) / 1e9
    line = {
        "metric": "points/s", "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"plugin sample_and_step_stokes: {n} seeded points inside a {M['nr']}x{M['ntheta']}x"
                               f"{M['nphi']}x11 float64 torus brick, ds_cm {M['ds_cm']}, broadcast initial",
                   "points_per_step": n, "l2": "brick (738 MB) larger than L2; points uniform over the domain",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "e2e": e2e, "clocks": clk,
        # this package's kernels per step: cell keys + the ordered sampler (the radix sort's are the library's)
        "gpu_launches": args.steps * (2 if n >= kernels.SORT_MIN_POINTS else 1),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": profiled_traffic(MICRO_PROFILE),
                     "peak_source": f"{peaks['source']} (MEASURED_PEAKS.json hbm_gbs)" if peaks["source"] == "measured"
                     else "fallback 6.65 TB/s",
                     "kernel": "sample_and_step_ordered_kernel (timed: cell keys, radix sort and the ordered "
                               "sampler)", "algorithmic_bytes_per_point": MICRO_BYTES_PER_POINT},
        "cpu_baseline": cpu,
        "kernel_ms": {"mean": per_mean, "min": min(per), "max": max(per)},
        "stokes_rk2_brick": stokes_rk2,
    }
    if world > 1:
        import torch.distributed as td

        td.destroy_process_group()
    return line if rank == 0 else None


def micro_cpu_baseline(b, pts, ds_cm: float, target_s: float) -> dict:
    """The float64 oracle (oracle/bhoracle.c bho_sample_and_step_stokes, one core) on a prefix of the points."""
    sys.path.insert(0, str(REPO))
    from oracle import oracle as O

    coeffs = b.coeffs.reshape(-1)
    n = 1 << 16
    t0 = time.perf_counter()
    O.sample_and_step_stokes(coeffs, b.r, b.theta, b.phi, pts[:n], ds_cm, np.zeros(4))
    dt = time.perf_counter() - t0
    if dt < target_s / 4:
        n = min(len(pts), int(n * target_s / max(dt, 1e-3)))
        t0 = time.perf_counter()
        O.sample_and_step_stokes(coeffs, b.r, b.theta, b.phi, pts[:n], ds_cm, np.zeros(4))
        dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "points/s", "cores": 1, "kind": "port",
            "sample": f"float64 oracle (oracle/bhoracle.c, one core): {n} of the points in {dt:.2f} s"}


def _scaled_traffic(summary: Path, scale: float) -> float | None:
    t = profiled_traffic(summary)
    return None if t is None else t * scale


def _uuid(device):
    import torch

    try:
        return "GPU-" + str(torch.cuda.get_device_properties(device).uuid)
    except Exception:
        return None


def _lib_check(rc):
    from blackhole_native import _lib

    _lib.check(rc)


# ------------------------------------------------------------------ learned step size
FLOP_PER_RHS = 60   # one FP32 Hamiltonian right-hand side with its pole sin / cos (half of a plain step's 213
                    # less the state update and tests)


def time_to_image(device, side: int, reps: int, spin: float = 0.9375, incl: float = 30.0,
                  cpu_seconds: float = 0.0) -> dict:
    """Time to an image at <= 1e-3 Stokes-I rel L1 against the FP64 kernel at
    h/16: plain fixed-step RK2 at h, h/2, h/4, h/8 against the learned step
    size and the step-doubling controller, on a side x side view (horizon
    guard on) of a seeded torus brick (seed 1).  The error is taken over
    pixels whose fine-step result is stable and kept the null constraint
    (studies.py).  Each method's time is the fastest of ``reps`` launches
    (CUDA events); GPU clocks are sampled while the methods run."""
    import torch

    from blackhole_native import learned, studies
    from blackhole_native.bricks import torus_brick
    from blackhole_native.render import DeviceBrick, View

    brick = torus_brick(256, 128, 256, spin_a=spin, seed=1)
    db = DeviceBrick(brick, device=device, precisions=("fp32", "fp64"))
    v = View(side, side, spin_a=spin, inclination_deg=incl, max_steps=65536, horizon_guard=True)
    v16 = v.scaled_step(1 / 16)
    ref_res = studies._render(db, v16, "fp64", ray_outputs=True)[0]
    ref = ref_res.image().cpu().numpy()
    drift = ref_res.per_ray("h_drift").cpu().numpy().astype(np.float64)
    del ref_res
    ref8 = studies._render(db, v.scaled_step(1 / 8), "fp64")[0].image().cpu().numpy()
    perts = [studies._render(db, w, "fp64")[0].image().cpu().numpy()
             for w in (v.scaled_step(1 / 16 * (1 + 1e-6)), studies.camera_perturbed(v16))]
    scale = studies.median_lit(ref[..., 0])
    mask = studies.stable_mask(ref, perts, scale) & np.isfinite(ref8[..., 0]) & (
        np.abs(ref8[..., 0] - ref[..., 0]) <= 1e-2 * np.abs(ref[..., 0]) + 1e-4 * scale) & (drift <= studies.MAX_DRIFT)
    net = learned.shipped_weights()
    if net is None:
        raise RuntimeError("the shipped step-size network (weights/step_net.npz) is missing")
    torch.cuda.synchronize(device)
    clocks = ClockSampler(_uuid(device)).start()
    time.sleep(0.3)
    runs = {}
    for f in (1.0, 0.5, 0.25, 0.125):
        runs[f"plain h*{f}"] = learned.render_plain(db, [v.scaled_step(f)], repeats=reps)
    runs["learned"] = learned.render_learned(db, [v], net, learned.AdaptConfig(), repeats=reps)
    for tol in (1e-5, 2e-5, 4e-5):  # the controller at each tolerance; its fastest one under the bar is compared
        runs[f"controller tol {tol:g}"] = learned.render_adaptive(db, [v], learned.AdaptConfig(tol=tol), repeats=reps)
    torch.cuda.synchronize(device)
    clk = clocks.stop()
    table = {}
    for k, r in runs.items():
        e = studies.image_errors(r.image().cpu().numpy(), ref, mask, scale)
        table[k] = {"ms": round(r.ms, 2), "rel_l1_I": e["rel_l1_I"], "capped_rel_l1_I": e["capped_rel_l1_I"],
                    "rel_l1_Q": e["rel_l1_Q"], "rel_l1_U": e["rel_l1_U"], "rel_l1_V": e["rel_l1_V"],
                    "flux_weighted_dm": e["flux_weighted_dm"], "bad_frac": e["bad_frac"],
                    **({"rhs_evals": r.counters["rhs_evals"]} if r.counters else {})}
    ok = {k: t["ms"] for k, t in table.items() if t["rel_l1_I"] <= 1e-3}
    plain_best = min((t for k, t in ok.items() if k.startswith("plain")), default=None)
    plain_key = min((k for k in ok if k.startswith("plain")), key=lambda k: ok[k], default=None)
    ctrl_key = min((k for k in ok if k.startswith("controller")), key=lambda k: ok[k], default=None)
    # Hamiltonian drift of the learned loop's rays: one more launch with per-ray outputs
    lr = learned.render_learned(db, [v], net, learned.AdaptConfig(), repeats=1, ray_outputs=True)
    res = lr.renderer.result()
    h_drift = studies._drift_summary(res.per_ray("h_drift").cpu().numpy().astype(np.float64),
                                     res.per_ray("status").cpu().numpy())
    out = {"workload": f"{side}x{side} rays, a={spin}, i={incl}deg, horizon guard, 256x128x256x11 float32 torus "
                       "brick (seed 1), reference FP64 kernel at h/16",
           "mask_fraction": float(mask.mean()), "timing": f"each method: the fastest of {reps} launches (CUDA events)",
           "learned_ms": ok.get("learned"), "controller_ms": ok.get(ctrl_key) if ctrl_key else None,
           "controller_best": ctrl_key,
           "plain_best_ms": plain_best, "plain_best": plain_key,
           "speedup_learned_vs_plain": (plain_best / ok["learned"]) if plain_best and ok.get("learned") else None,
           "speedup_learned_vs_controller": (ok[ctrl_key] / ok["learned"]) if ctrl_key and ok.get("learned") else None,
           "runs": table, "h_drift_learned": h_drift, "clocks": clk}
    lrun = runs["learned"]
    if lrun.counters:
        tf = lrun.counters["rhs_evals"] * FLOP_PER_RHS / (lrun.ms * 1e-3) / 1e12
        out["roofline_fp32_learned"] = {
            "bound": "fp32", "achieved": round(tf, 2), "unit": "TFLOP/s",
            "note": f"{FLOP_PER_RHS} FP32 FLOP per right-hand-side evaluation x the learned loop's evaluations "
                    "(brick segments and network not counted)",
            "peak": round(fp32_peak(device, torch.cuda.current_stream(device)), 2)}
        out["roofline_fp32_learned"]["frac"] = round(tf / out["roofline_fp32_learned"]["peak"], 4)
    if cpu_seconds > 0 and plain_key is not None:
        out["cpu_baseline"] = plain_cpu_time_to_image(brick, v.scaled_step(float(plain_key.split("*")[1])), side,
                                                      cpu_seconds)
    return out


def plain_cpu_time_to_image(brick, view, side: int, target_s: float) -> dict:
    """The FP64 oracle (C, OpenMP over every host core) with the plain method
    at the step that meets the 1e-3 bar on the GPU, on a centred crop sized to
    about target_s seconds; the time to the full image is extrapolated by the
    pixel count."""
    sys.path.insert(0, str(REPO))
    from oracle import oracle as O

    def run(n):
        x0 = (side - n) // 2
        ov = O.make_view(spin_a=view.spin_a, r_obs=view.r_obs, theta_obs=math.radians(view.inclination_deg),
                         phi_obs=0.0, fov_y_deg=view.fov_y_deg, roll_deg=0.0, h_scale=view.h_scale,
                         h_min=view.h_min, h_max=view.h_max, escape_radius=view.escape_radius,
                         affine_to_length_cm=1.0, max_optical_depth=30.0, width=side, height=side, x0=x0, y0=x0,
                         crop_w=n, crop_h=n, max_steps=view.max_steps, flags=1)  # flags 1: horizon guard
        t0 = time.perf_counter()
        O.render(ov, brick.coeffs, brick.r, brick.theta, brick.phi, stop_at_tau=True)
        return time.perf_counter() - t0

    n = 16
    dt = run(n)
    n = int(max(16, min(side, n * math.sqrt(target_s / max(dt, 1e-3)))))
    dt = run(n)
    ms = dt * (side * side) / (n * n) * 1e3
    return {"value": ms, "unit": "ms", "cores": O.max_threads(), "kind": "port",
            "sample": f"float64 oracle (C, OpenMP), plain RK2 at {view.h_scale:g} r, centred {n}x{n} crop in "
                      f"{dt:.2f} s, extrapolated to {side}x{side} pixels"}


def bench_learned(args) -> dict | None:
    """The metric's second half on its own line: time to an image at <= 1e-3
    Stokes-I rel L1, learned step size against plain RK2 and the controller
    (time_to_image)."""
    import torch

    rank, world, local_rank = dist_env()
    if rank != 0:
        return None
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    side = args.side or 2048
    reps = max(args.steps, 1)
    tti = time_to_image(device, side, reps, cpu_seconds=0.0 if args.no_cpu_baseline else args.cpu_seconds)
    learned_ms = tti["learned_ms"]
    return {
        "metric": "time to an image at <= 1e-3 Stokes-I rel L1 vs the FP64 fine-step kernel (learned step size)",
        "value": learned_ms, "unit": "ms", "n_gpus": 1, "steps": reps, "warmup": None, "ms_per_step": learned_ms,
        "timing": tti["timing"], "higher_is_better": False, "scaling": "none", "vs_baseline": None,
        "dtype": "f32 (BF16 network)", "data": "synthetic",
        "config": {"workload": "learned step size: " + tti["workload"], "mask_fraction": tti["mask_fraction"]},
        "plain_best_ms": tti["plain_best_ms"], "speedup_vs_plain": tti["speedup_learned_vs_plain"],
        "speedup_vs_controller": tti["speedup_learned_vs_controller"], "controller_ms": tti["controller_ms"],
        "controller_best": tti["controller_best"], "runs": tti["runs"], "gpu_launches": len(tti["runs"]) * reps, "clocks": tti["clocks"],
        "roofline": tti.get("roofline_fp32_learned"), "cpu_baseline": tti.get("cpu_baseline"),
        "h_drift": tti["h_drift_learned"],
    }


def bench_reference(args) -> dict | None:
    rank, world, _ = dist_env()
    if rank != 0:
        return None
    sys.path.insert(0, str(REPO))
    from oracle import oracle as O

    brick = make_brick()
    n = calibrated_oracle_size(brick, args.ref_seconds)
    for _ in range(args.warmup):
        run_oracle(brick, max(32, n // 4))
    total_steps, total_s = 0, 0.0
    for _ in range(args.steps):
        s, dt = run_oracle(brick, n)
        total_steps += s
        total_s += dt
    value = total_steps / total_s
    sample = (f"float64 oracle restatement of the reference loop (C, OpenMP, {O.max_threads()} threads); each step "
              f"renders {n}x{n} rays over the full field of view of the workload")
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_s * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "plain fused kernel at scale: 1024x1024 rays, r_obs=1000M, i=17deg, FOV +-20M, "
                               "a=0.9375, RK2 h=0.02r in [1e-3,1], max_steps=4096, 256x128x256x11 float32 "
                               "seeded torus brick (bounded CPU sample per step)",
                   "sample_side": n},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": O.max_threads(), "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-views", action="store_true", help="skip the 256-view block of the default line")
    ap.add_argument("--no-time-to-image", action="store_true",
                    help="skip the learned-vs-controller-vs-plain time to a 2048^2 image at 1e-3")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the crop check against the FP64 kernel at a quarter of the step")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target length of the CPU-baseline sample")
    ap.add_argument("--ref-seconds", type=float, default=4.0, help="target length of one reference-arm step")
    ap.add_argument("--config", type=json.loads, default=None, help="RenderConfig fields as JSON (skips autotune)")
    ap.add_argument("--tune", action="store_true", help="run the launch-shape autotuner on the workload and exit")
    ap.add_argument("--workload", choices=["image", "views", "precompute", "grrt", "learned", "bricks", "micro"],
                    default="image",
                    help="image: the 1024x1024 single view (default); views: many uneven views in one launch; "
                         "precompute: coefficient bricks from a snapshot; grrt: the physical polarized renderer; "
                         "learned: time to an image at 1e-3, learned step size against plain RK2; bricks: the "
                         "reference's own brick renderer (fixed-step RK4); micro: the plugin's "
                         "sample_and_step_stokes at 16.8M points")
    ap.add_argument("--n-views", type=int, default=256)
    ap.add_argument("--side", type=int, default=0,
                    help="profiling only: image workload side x side rays; precompute nr = side; grrt and "
                         "bricks image side x side*9/16; micro side*1024 points")
    args = ap.parse_args(argv)
    args.warmup = max(3, args.warmup)  # at least 3 untimed warm-up steps, whatever is asked
    if args.impl == "reference":
        line = bench_reference(args)
    elif args.workload == "views":
        line = bench_views(args)
    elif args.workload == "precompute":
        line = bench_precompute(args)
    elif args.workload == "grrt":
        line = bench_grrt(args)
    elif args.workload == "learned":
        line = bench_learned(args)
    elif args.workload == "bricks":
        line = bench_bricks(args)
    elif args.workload == "micro":
        line = bench_micro(args)
    else:
        line = bench_ours(args)
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
