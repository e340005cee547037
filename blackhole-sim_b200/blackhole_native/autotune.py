"""Autotuner for the persistent ray kernel's launch shape.

Search space: threads per block, resident blocks per SM (the persistent grid
is SMs x blocks_per_sm), the ray-order tile (rays of one tile are consecutive
in the work queue, so a warp's 32 rays start spatially coherent), and the
warp refill threshold (how many finished lanes a warp collects before it
fetches new rays: 1 = always compact, 32 = never).  Every candidate renders
the same views; the fastest by CUDA-event time wins.  Results are cached per
(GPU name, workload key) in a JSON file next to this module.
"""

from __future__ import annotations

import itertools
import json
import os
from dataclasses import asdict, replace
from pathlib import Path
from typing import Callable, Iterable, Sequence

import torch

from .render import DeviceBrick, RenderConfig, Renderer, View

CACHE = Path(os.environ.get("BHN_AUTOTUNE_CACHE", Path(__file__).resolve().parent / "autotune_cache.json"))

DEFAULT_SPACE = {
    "block_threads": (64, 128, 256),
    "blocks_per_sm": (2, 3, 4, 6, 8),
    "tile": ((8, 4), (4, 8), (16, 2), (32, 1)),
    "refill_min": (1, 8, 16, 32),
    "reg_cap": (0, 80, 64),
}


def _key(workload: str, device: torch.device) -> str:
    return f"{torch.cuda.get_device_name(device)}|{workload}"


def _load() -> dict:
    try:
        return json.loads(CACHE.read_text())
    except (OSError, ValueError):
        return {}


def cached_config(workload: str, device: torch.device | None = None) -> RenderConfig | None:
    """The cached best launch shape for ``workload`` on this GPU, if any."""
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device())
    entry = _load().get(_key(workload, device))
    return RenderConfig(**entry["config"]) if entry else None


def store(workload: str, config: RenderConfig, ms: float, device: torch.device, table: list | None = None) -> None:
    data = _load()
    data[_key(workload, device)] = {"config": asdict(config), "ms": ms, "table": table or []}
    CACHE.write_text(json.dumps(data, indent=1, sort_keys=True) + "\n")


def launch_candidates(space: dict | None = None, base: RenderConfig | None = None) -> Iterable[RenderConfig]:
    """Stage 1: threads per block x resident blocks x register budget, each in
    both loop modes (per-step refill and whole-warp batches), since the best
    shape differs between them."""
    s = space or DEFAULT_SPACE
    b = base or RenderConfig()
    for bt, bps, rc, rm in itertools.product(s["block_threads"], s["blocks_per_sm"], s["reg_cap"],
                                             sorted({min(s["refill_min"]), 32})):
        if bt * bps > 2048:   # more threads than an SM holds
            continue
        yield replace(b, block_threads=bt, blocks_per_sm=bps, reg_cap=rc, refill_min=rm)


def order_candidates(space: dict | None = None, base: RenderConfig | None = None) -> Iterable[RenderConfig]:
    """Stage 2: ray-order tile x warp refill threshold, on the best launch shape."""
    s = space or DEFAULT_SPACE
    b = base or RenderConfig()
    for (tw, th), rm in itertools.product(s["tile"], s["refill_min"]):
        yield replace(b, tile_w=tw, tile_h=th, refill_min=rm)


def candidates(space: dict | None = None) -> Iterable[RenderConfig]:
    """The full product of both stages (for exhaustive sweeps)."""
    for c in launch_candidates(space):
        yield from order_candidates(space, c)


def time_config(brick: DeviceBrick, views: Sequence[View], cfg: RenderConfig, *, precision: str = "fp32",
                repeats: int = 3) -> float:
    """Median CUDA-event milliseconds of one graph-replayed launch."""
    r = Renderer(brick, views, config=cfg, precision=precision)
    r.capture()
    r.graph_launch()
    torch.cuda.synchronize()
    times = []
    s = torch.cuda.current_stream()
    for _ in range(repeats):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        r.graph_launch()
        b.record(s)
        b.synchronize()
        times.append(a.elapsed_time(b))
    r.release_graph()
    times.sort()
    return times[len(times) // 2]


def tune(brick: DeviceBrick, views: Sequence[View], workload: str, *, space: dict | None = None,
         precision: str = "fp32", repeats: int = 3, log: Callable[[str], None] | None = None) -> RenderConfig:
    """Two-stage search (launch shape, then ray order on the winner); caches and
    returns the fastest configuration."""
    device = brick.device
    best, best_ms, table = RenderConfig(), float("inf"), []
    for stage in (launch_candidates, order_candidates):
        for cfg in stage(space, best):
            ms = time_config(brick, views, cfg, precision=precision, repeats=repeats)
            table.append([asdict(cfg), round(ms, 4)])
            if log:
                log(f"{asdict(cfg)} {ms:.3f} ms")
            if ms < best_ms:
                best, best_ms = cfg, ms
    store(workload, best, best_ms, device, table)
    return best
