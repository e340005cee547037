"""Tiled and progressive (coarse-to-fine) rendering.

``generate_tiles`` / ``progressive_levels`` / ``generate_progressive_tiles``
mirror the reference's scheduling helpers (python/blackhole_sim/tiles.py:9-59).
``progressive_render`` is their GPU use: every level of the coarse-to-fine
ladder is one persistent launch on the current stream, queued back to back,
and each level's image is handed out as soon as its own launch has finished
(an event per level), so a viewer shows the coarse image while the finer
levels still render.
"""

from __future__ import annotations

from dataclasses import dataclass, replace
from typing import Iterator, Sequence

import torch

from .render import DeviceBrick, RenderConfig, Renderer, View


@dataclass(frozen=True, order=True)
class RenderTile:
    """tiles.py:9-27."""

    level: int
    y0: int
    x0: int
    x1: int
    y1: int

    @property
    def width(self) -> int:
        return self.x1 - self.x0

    @property
    def height(self) -> int:
        return self.y1 - self.y0

    @property
    def pixels(self) -> int:
        return self.width * self.height


def generate_tiles(width: int, height: int, tile_size: int = 64, level: int = 0) -> list[RenderTile]:
    """tiles.py:30-35: row-major tiles of at most tile_size pixels a side."""
    tiles: list[RenderTile] = []
    for y in range(0, int(height), int(tile_size)):
        for x in range(0, int(width), int(tile_size)):
            tiles.append(RenderTile(level, x0=x, y0=y, x1=min(x + tile_size, width), y1=min(y + tile_size, height)))
    return tiles


def progressive_levels(width: int, height: int, min_width: int = 480) -> list[tuple[int, int, int]]:
    """tiles.py:38-51: (level, width, height) from the coarsest power-of-two
    reduction at least min_width wide up to the full image."""
    out: list[tuple[int, int, int]] = []
    w = int(width)
    scale = 1
    while w // (scale * 2) >= min_width:
        scale *= 2
    level = 0
    while scale >= 1:
        out.append((level, max(1, width // scale), max(1, height // scale)))
        level += 1
        scale //= 2
    return out


def generate_progressive_tiles(width: int, height: int, tile_size: int = 64,
                               min_width: int = 480) -> Iterator[RenderTile]:
    """tiles.py:54-57."""
    for level, w, h in progressive_levels(width, height, min_width):
        yield from generate_tiles(w, h, tile_size, level)


def tile_views(view: View, tiles: Sequence[RenderTile]) -> list[View]:
    """The tiles of one view as crops (the renderer packs them back to back)."""
    return [replace(view, crop=(t.x0, t.y0, t.width, t.height)) for t in tiles]


def progressive_render(brick: DeviceBrick, view: View, *, min_width: int = 480, config: RenderConfig | None = None,
                       precision: str = "fp32") -> Iterator[tuple[int, torch.Tensor]]:
    """Yield (level, (h, w, 4) image on the device) coarse to fine.  All levels
    are queued at once; each is yielded when its own launch has completed."""
    levels = progressive_levels(view.width, view.height, min_width)
    queued = []
    for level, w, h in levels:
        r = Renderer(brick, [replace(view, width=w, height=h, crop=None)], config=config, precision=precision)
        r.launch()
        done = torch.cuda.Event()
        done.record()
        queued.append((level, r, done))
    for level, r, done in queued:
        done.synchronize()
        yield level, r.result().image(0)
