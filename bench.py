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
        import torch.distributed as td

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


def profiled_traffic() -> float | None:
    """DRAM bytes per launch of the render kernel from the committed ncu summary."""
    if not PROFILE_SUMMARY.exists():
        return None
    for line in PROFILE_SUMMARY.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def make_brick():
    from blackhole_native import bricks

    return bricks.torus_brick(BRICK["nr"], BRICK["ntheta"], BRICK["nphi"], spin_a=WORKLOAD["spin_a"],
                              seed=BRICK["seed"], dtype=np.float32)


def cpu_sample_view(n: int, **over):
    from blackhole_native import View

    kw = dict(WORKLOAD)
    kw.update(width=n, height=n)
    kw.update(over)
    return View(**kw)


def run_oracle(brick, n: int, threads: int = 0) -> tuple[int, float]:
    """The float64 oracle on an n x n image of the workload's field of view.
    Returns (ray_steps, seconds)."""
    sys.path.insert(0, str(REPO))
    from oracle import oracle as O

    v = cpu_sample_view(n)
    ov = O.make_view(spin_a=v.spin_a, r_obs=v.r_obs, theta_obs=math.radians(v.inclination_deg), phi_obs=0.0,
                     fov_y_deg=v.fov_y_deg, roll_deg=0.0, h_scale=v.h_scale, h_min=v.h_min, h_max=v.h_max,
                     escape_radius=v.escape_radius, affine_to_length_cm=1.0, max_optical_depth=30.0, width=n,
                     height=n, x0=0, y0=0, crop_w=n, crop_h=n, max_steps=v.max_steps)
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

    # FP32 FMA peak on this GPU (denominator of the FP32 roofline)
    probe = torch.empty(1 << 20, dtype=torch.float32, device=device)
    flops = __import__("ctypes").c_int64()
    L = _lib.lib()
    for _ in range(2):
        _lib.check(L.bhn_fp32_peak_probe(probe.data_ptr(), 4096, 8, __import__("ctypes").byref(flops),
                                         stream.cuda_stream))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    _lib.check(L.bhn_fp32_peak_probe(probe.data_ptr(), 4096, 8, __import__("ctypes").byref(flops),
                                     stream.cuda_stream))
    e1.record(stream)
    torch.cuda.synchronize(device)
    fp32_peak_tflops = flops.value / (e0.elapsed_time(e1) * 1e-3) / 1e12

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

    peaks = load_peaks()
    kernel_s = statistics.mean(per_launch_ms) * 1e-3
    alg_bytes = brick_steps * BYTES_PER_BRICK_STEP + rays * BYTES_PER_RAY
    alg_flops = steps_per_launch * FLOP_PER_STEP + brick_steps * FLOP_PER_BRICK_STEP
    achieved_gbs = alg_bytes / kernel_s / 1e9
    traffic = profiled_traffic()
    roofline = {"bound": "hbm", "achieved": round(achieved_gbs, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": round(achieved_gbs / peaks["hbm_gbs"], 4), "traffic": traffic,
                "peak_source": f"{peaks['source']} (MEASURED_PEAKS.json hbm_gbs)" if peaks["source"] == "measured"
                else "fallback 6.65 TB/s",
                "kernel": "render_kernel<Tracer32>", "algorithmic_bytes_per_launch": int(alg_bytes)}
    achieved_tf = alg_flops / kernel_s / 1e12
    roofline_fp32 = {"bound": "fp32", "achieved": round(achieved_tf, 2), "peak": round(fp32_peak_tflops, 2),
                     "unit": "TFLOP/s", "frac": round(achieved_tf / fp32_peak_tflops, 4),
                     "peak_source": "measured in this run (bhn_fp32_peak_probe FMA loop)",
                     "algorithmic_flops_per_launch": int(alg_flops)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(brick_h, args.cpu_seconds)

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
        "status_counts": st2.status, "max_h_drift": st2.max_h_drift,
    }
    rnd.release_graph()
    if world > 1:
        import torch.distributed as td

        td.destroy_process_group()
    return line if rank == 0 else None


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
    rnd.capture()
    for _ in range(args.warmup):
        rnd.graph_launch()
    torch.cuda.synchronize(device)
    st = rnd.result().stats()
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
    total_ms = evs[0].elapsed_time(evs[K])
    t_max = max_over_ranks(total_ms, world, device)
    value = sum_over_ranks(st.ray_steps * K, world, device) / (t_max * 1e-3)
    rnd.release_graph()
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
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": t_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"batched persistent launch: {len(views)} seeded views (side 64-1024, a~U(0,0.998), "
                               "incl~U(5,85)deg, max_steps~U{512..8192}), shared 128x64x128x11 float32 brick, "
                               "one CUDA-graph launch",
                   "rays_per_step": st.rays, "ray_steps_per_step": st.ray_steps,
                   "autotune": {"block_threads": cfg.block_threads, "blocks_per_sm": cfg.blocks_per_sm,
                                "tile": [cfg.tile_w, cfg.tile_h], "refill_min": cfg.refill_min,
                                "reg_cap": cfg.reg_cap}},
        "per_view_ray_steps_per_s": {"min": float(pv.min()), "median": float(np.median(pv)),
                                     "max": float(pv.max()), "views": len(pv)},
        "status_counts": st.status, "gpu_launches": K,
    }
    if world > 1:
        import torch.distributed as td

        td.destroy_process_group()
    return line if rank == 0 else None


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
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target length of the CPU-baseline sample")
    ap.add_argument("--ref-seconds", type=float, default=4.0, help="target length of one reference-arm step")
    ap.add_argument("--config", type=json.loads, default=None, help="RenderConfig fields as JSON (skips autotune)")
    ap.add_argument("--tune", action="store_true", help="run the launch-shape autotuner on the workload and exit")
    ap.add_argument("--workload", choices=["image", "views"], default="image",
                    help="image: the 1024x1024 single view (default); views: many uneven views in one launch")
    ap.add_argument("--n-views", type=int, default=256)
    ap.add_argument("--side", type=int, default=0,
                    help="render side x side rays of the same scene instead of 1024x1024 (profiling only)")
    args = ap.parse_args(argv)
    args.warmup = max(3, args.warmup)  # at least 3 untimed warm-up steps, whatever is asked
    if args.impl == "reference":
        line = bench_reference(args)
    elif args.workload == "views":
        line = bench_views(args)
    else:
        line = bench_ours(args)
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
