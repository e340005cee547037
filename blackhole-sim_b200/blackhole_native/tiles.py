"""Tiled and progressive (coarse-to-fine) rendering.

``generate_tiles`` / ``progressive_levels`` / ``generate_progressive_tiles``
give the same tiles and levels as the reference's scheduling helpers
(python/blackhole_sim/tiles.py:9-57).
``progressive_render`` is their GPU use: every level of the coarse-to-fine
ladder is one persistent launch on the current stream, queued back to back,
and each level's image is handed out as soon as its own launch has finished
(an event per level), so a viewer shows the coarse image while the finer
levels still render.
"""

from __future__ import annotations

import itertools
import math
from dataclasses import dataclass, replace
from typing import Iterator, Sequence

import torch

from .render import DeviceBrick, RenderConfig, Renderer, View


@dataclass(frozen=True, order=True)
class RenderTile:
    """One rectangle [x0, x1) x [y0, y1) of the image at a progressive level.

    Field order and ordering are the reference's (python/blackhole_sim/tiles.py:9-27):
    tiles sort by level, then row, then column."""

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


def _spans(extent: int, size: int) -> list[tuple[int, int]]:
    """[start, stop) pieces of at most ``size`` covering range(extent)."""
    starts = range(0, int(extent), int(size))
    return [(s, min(s + size, extent)) for s in starts]


def generate_tiles(width: int, height: int, tile_size: int = 64, level: int = 0) -> list[RenderTile]:
    """Row-major tiles of at most ``tile_size`` pixels a side covering a
    width x height image; edge tiles are clipped (tiles.py:30-35)."""
    rows, cols = _spans(height, tile_size), _spans(width, tile_size)
    return [RenderTile(level, y0=y0, x0=x0, x1=x1, y1=y1) for (y0, y1), (x0, x1) in itertools.product(rows, cols)]


def progressive_levels(width: int, height: int, min_width: int = 480) -> list[tuple[int, int, int]]:
    """(level, width, height) of the coarse-to-fine ladder (tiles.py:38-51).

    Level 0 is the image reduced by 2**k, k the largest power whose reduced
    width ``width // 2**k`` is still at least ``min_width`` (k = 0 when the
    image is narrower than that); every further level halves the reduction,
    the last being the full image.  ``width // 2**k >= m`` holds exactly when
    2**k <= width // ceil(m), so k is the bit length of that quotient less one.
    """
    m = math.ceil(min_width)
    if m < 1:
        raise ValueError("min_width must be at least 1")
    quotient = int(width) // m
    k = quotient.bit_length() - 1 if quotient >= 1 else 0
    return [(level, max(1, width // 2 ** (k - level)), max(1, height // 2 ** (k - level))) for level in range(k + 1)]


def generate_progressive_tiles(width: int, height: int, tile_size: int = 64,
                               min_width: int = 480) -> Iterator[RenderTile]:
    """The tiles of every progressive level, coarsest level first (tiles.py:54-57)."""
    return itertools.chain.from_iterable(generate_tiles(w, h, tile_size, level)
                                         for level, w, h in progressive_levels(width, height, min_width))


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
